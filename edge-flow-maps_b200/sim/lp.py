"""Drop-in for the reference's sim/lp.py laden-particle kernels (same names
and arguments) on libedgeb200.so.  Particle arrays are (max_num, 3) float32
tensors (ti.Vector.field(3, float, shape=max_num)); the radius array is
(max_num,)."""
from edgeb200 import ops
from edgeb200.fields import dims_from_faces


def update_particles_acc(u_x, u_y, u_z, laden_particles_vel, laden_particles_pos, laden_particles_acc, dx, curr_dt,
                         laden_particle_num, St, gravity):
    """lp.py:6-29 (G2P of velocity, drag + gravity acceleration)."""
    ops.lp_acc((u_x, u_y, u_z), dx, laden_particles_vel, laden_particles_pos, laden_particles_acc,
               laden_particle_num, curr_dt, St, gravity)


def update_particles_velocity(laden_particles_acc, laden_particles_vel, laden_particles_pos, curr_dt, dx,
                              laden_particle_num, domain_range_x, domain_range_y, domain_range_z):
    """lp.py:32-70."""
    ops.lp_velocity(laden_particles_acc, laden_particles_vel, laden_particles_pos, curr_dt, dx, laden_particle_num,
                    (domain_range_x, domain_range_y, domain_range_z))


def calculate_velocity_diff(u_x, u_y, u_z, laden_particles_vel, laden_particles_vel_diff, laden_particles_pos, dx,
                            laden_particle_num, St, density_ratio, epiral_radius_ratio):
    """lp.py:73-97."""
    ops.lp_vel_diff((u_x, u_y, u_z), dx, laden_particles_vel, laden_particles_vel_diff, laden_particles_pos,
                    laden_particle_num, St, density_ratio, epiral_radius_ratio)


def laden_particles_back_with_computing_particle(drag_x, drag_y, drag_z, u_x, u_y, u_z, laden_particles_vel,
                                                 laden_particles_vel_diff, laden_particles_pos,
                                                 laden_particle_ref_radius, dx, laden_particle_num, laden_radius,
                                                 domain_range_x, domain_range_y, domain_range_z, res_x, res_y, res_z):
    """lp.py:100-156 (P2G scatter of the drag onto the face grids)."""
    ops.lp_p2g((res_x, res_y, res_z), dx, (drag_x, drag_y, drag_z), laden_particles_vel_diff, laden_particles_pos,
               laden_particle_ref_radius, laden_particle_num, laden_radius,
               (domain_range_x, domain_range_y, domain_range_z))


def update_particles_position(laden_particles_vel, laden_particles_pos, curr_dt, laden_particle_num, domain_range_x,
                              domain_range_y, domain_range_z):
    """lp.py:158-181."""
    ops.lp_position(laden_particles_vel, laden_particles_pos, curr_dt, laden_particle_num,
                    (domain_range_x, domain_range_y, domain_range_z))


def calculate_viscous_force(u_x, u_y, u_z, vis_x, vis_y, vis_z, dx, Re):
    """lp.py:183-219."""
    dims_from_faces(u_x, u_y, u_z)
    ops.lp_viscous((u_x, u_y, u_z), dx, Re, (vis_x, vis_y, vis_z))
