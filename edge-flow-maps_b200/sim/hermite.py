"""Drop-in for the reference's sim/hermite.py host entry points (the flow-map
marches, the semi-Lagrangian advection and the map resets), running the
sm_100a kernels of libedgeb200.so.

Fields are torch float32 CUDA tensors in the reference's layout: a
``ti.Vector.field(3, float, shape=(nx, ny, nz))`` becomes a tensor of shape
(nx, ny, nz, 3).  Arguments keep the reference's order and meaning; the cell
and face coordinate fields (X, X_x, ...) are accepted for signature
compatibility but positions are computed exactly in-kernel as
(I + 0.5) * dx, as center_coords_func / x_coords_func do
(util/taichi_utils.py:23-44).  Scratch fields of the reference's unfused
pipelines (psi_0..psi_3, psi_000..psi_111) hold the marched results before
they are copied into the accumulated map, as the reference's temporaries do.
"""
import torch

from edgeb200 import _native as N
from edgeb200 import ops
from edgeb200.fields import require

__all__ = [
    "advect_psi_garm_ed4_fusion_unroll", "advect_ps_hermite_ed4_fd_unroll", "advect_ps_hermite_ed8",
    "advect_ps_garm", "calc_fd_3_from_grad", "advect_u_semi_lagrangian", "reset_to_identity_1", "reset_to_identity_2", "reset_to_identity_3",
    "reset_to_identity_ed4", "reset_to_identity_ed8", "interp_hermite_points",
]

_ED4_OFF = ((-1, -1, -1), (1, 1, -1), (-1, 1, 1), (1, -1, 1))                        # hermite.py:737-742
_ED8_OFF = ((-1, -1, -1), (1, -1, -1), (-1, 1, -1), (1, 1, -1),                      # hermite.py:716-723
            (-1, -1, 1), (1, -1, 1), (-1, 1, 1), (1, 1, 1))


def advect_psi_garm_ed4_fusion_unroll(psi_tmp, T_x_tmp, T_y_tmp, T_z_tmp, dT_x_tmp, dT_y_tmp, dT_z_tmp,
                                      psi, T_x, T_y, T_z, dT_x, dT_y, dT_z, u_x, u_y, u_z, X, dx, dt, epsilon):
    """hermite.py:1495-1521: EDGE march into the *_tmp fields, then copied
    into the accumulated map."""
    ops.march_edge((u_x, u_y, u_z), dx, dt, epsilon, psi, (T_x, T_y, T_z), (dT_x, dT_y, dT_z), psi_tmp,
                   (T_x_tmp, T_y_tmp, T_z_tmp), (dT_x_tmp, dT_y_tmp, dT_z_tmp))
    for d, s in ((psi, psi_tmp), (T_x, T_x_tmp), (T_y, T_y_tmp), (T_z, T_z_tmp), (dT_x, dT_x_tmp),
                 (dT_y, dT_y_tmp), (dT_z, dT_z_tmp)):
        ops.copy(s, d)


def advect_ps_hermite_ed4_fd_unroll(psi_0, psi_1, psi_2, psi_3, psi, T_x, T_y, T_z, u_x, u_y, u_z, X, dx, dt,
                                    epsilon):
    """hermite.py:1375-1395: ED4 march (the four scratch fields receive the new
    psi, T_x, T_y, T_z before the copy back)."""
    ops.march_ed4((u_x, u_y, u_z), dx, dt, epsilon, psi, (T_x, T_y, T_z), psi_0, (psi_1, psi_2, psi_3))
    for d, s in ((psi, psi_0), (T_x, psi_1), (T_y, psi_2), (T_z, psi_3)):
        ops.copy(s, d)


def advect_ps_hermite_ed8(psi_000, psi_001, psi_010, psi_011, psi_100, psi_101, psi_110, psi_111,
                          psi, T_x, T_y, T_z, dT_x, dT_y, dT_z, d2T_x, d2T_y, d2T_z, u_x, u_y, u_z, X, dx, dt,
                          epsilon):
    """hermite.py:1290-1338: ED8 march."""
    d2 = [torch.empty_like(d2T_x) for _ in range(3)]
    ops.march_ed8((u_x, u_y, u_z), dx, dt, epsilon, psi, (T_x, T_y, T_z), (dT_x, dT_y, dT_z), (d2T_x, d2T_y, d2T_z),
                  psi_000, (psi_001, psi_010, psi_011), (psi_100, psi_101, psi_110), d2)
    for d, s in ((psi, psi_000), (T_x, psi_001), (T_y, psi_010), (T_z, psi_011), (dT_x, psi_100),
                 (dT_y, psi_101), (dT_z, psi_110), (d2T_x, d2[0]), (d2T_y, d2[1]), (d2T_z, d2[2])):
        ops.copy(s, d)


def advect_ps_garm(psi_tmp, T_x_tmp, T_y_tmp, T_z_tmp, psi, T_x, T_y, T_z, dT_x, dT_y, dT_z, d2T_x, d2T_y, d2T_z,
                   u_x, u_y, u_z, X, dx, dt):
    """hermite.py:1398-1424: GE march.  As in the reference, the new psi and T
    are left in the _tmp fields as well as in psi, T."""
    dn = [torch.empty_like(dT_x) for _ in range(3)]
    d2n = [torch.empty_like(d2T_x) for _ in range(3)]
    ops.march_ge((u_x, u_y, u_z), dx, dt, psi, (T_x, T_y, T_z), (dT_x, dT_y, dT_z), (d2T_x, d2T_y, d2T_z),
                 psi_tmp, (T_x_tmp, T_y_tmp, T_z_tmp), dn, d2n)
    for d, s in ((psi, psi_tmp), (T_x, T_x_tmp), (T_y, T_y_tmp), (T_z, T_z_tmp), (dT_x, dn[0]), (dT_y, dn[1]),
                 (dT_z, dn[2]), (d2T_x, d2n[0]), (d2T_y, d2n[1]), (d2T_z, d2n[2])):
        ops.copy(s, d)


def calc_fd_3_from_grad(T_x, T_y, T_z, dT_x, dT_y, dT_z, d2T_x, d2T_y, d2T_z, dx):
    """hermite.py:1180-1256."""
    ops.calc_fd_3_from_grad(dx, (T_x, T_y, T_z), (dT_x, dT_y, dT_z), (d2T_x, d2T_y, d2T_z))


def advect_u_semi_lagrangian(u_x0, u_y0, u_z0, u_x1, u_y1, u_z1, dx, dt, X_x, X_y, X_z):
    """hermite.py:1578-1621."""
    ops.advect_u_sl((u_x0, u_y0, u_z0), dx, dt, (u_x1, u_y1, u_z1))


def _dx_from_X(X):
    require(X, "X")
    # X[0,0,0] = 0.5*dx (center_coords_func)
    return float(X[0, 0, 0, 0].item()) * 2.0


def reset_to_identity_1(psi, T_x, T_y, T_z, X):
    """hermite.py:642-654."""
    ops.reset_cells(_dx_from_X(X), psi, (T_x, T_y, T_z))


def reset_to_identity_2(psi, T_x, T_y, T_z, dT_x, dT_y, dT_z, X):
    """hermite.py:657-674."""
    ops.reset_cells(_dx_from_X(X), psi, (T_x, T_y, T_z), (dT_x, dT_y, dT_z))


def reset_to_identity_3(psi, T_x, T_y, T_z, dT_x, dT_y, dT_z, d2T_x, d2T_y, d2T_z, X):
    """hermite.py:676-700."""
    ops.reset_cells(_dx_from_X(X), psi, (T_x, T_y, T_z), (dT_x, dT_y, dT_z), (d2T_x, d2T_y, d2T_z))


def reset_to_identity_ed4(psi_0, psi_1, psi_2, psi_3, X, epsilon):
    """hermite.py:727-742: the four tetrahedral epsilon points around X."""
    for p, off in zip((psi_0, psi_1, psi_2, psi_3), _ED4_OFF):
        p.copy_(X + torch.tensor(off, dtype=torch.float32, device=X.device) * float(epsilon))


def reset_to_identity_ed8(psi_000, psi_001, psi_010, psi_011, psi_100, psi_101, psi_110, psi_111, X, epsilon):
    """hermite.py:703-723: the eight cube-corner epsilon points around X."""
    for p, off in zip((psi_000, psi_001, psi_010, psi_011, psi_100, psi_101, psi_110, psi_111), _ED8_OFF):
        p.copy_(X + torch.tensor(off, dtype=torch.float32, device=X.device) * float(epsilon))


def interp_hermite_points(variant, psi, T, dT, d2T, dx, pts):
    """Evaluate the Hermite interpolants of hermite.py (variant:
    'fd' -> interp_(grad_)hermite_fd_unroll, 'garm' -> *_garm_fd_unroll,
    'full' -> interp_(grad_)hermite) for all three components at points.
    Returns (value, value_of_grad_variant, grad rows)."""
    v = {"fd": N.HERMITE_FD, "garm": N.HERMITE_GARM, "full": N.HERMITE_FULL}[variant]
    return ops.points_hermite(v, psi, T, dT, d2T, dx, pts)
