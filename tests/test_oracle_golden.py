"""The C restatement oracle against golden vectors produced by the reference's
own sources (tests/golden/make_golden.py).  CPU only.

Tolerances: float32 paths agree to ~1e-7 relative; outputs that the reference
forms as epsilon differences of marched points lose digits by construction:
an ulp-level difference d ~ 2^-23 |psi| in the marched positions becomes
d/eps in T, d/eps^2 in dT and d/eps^3 in d2T (eps = 0.025 dx here), so their
tolerances scale accordingly.
"""
import numpy as np
import pytest

from conftest import load_golden, rel_l2
from oracle import edge_oracle as O

TOL = 2e-6          # plain float32 kernels
TOL_T = 1e-4        # first epsilon difference
TOL_DT = 5e-3       # second
TOL_D2T = 3e-2      # third


def test_interp_points():
    d = load_golden("interp_points")
    u = [d["u_x"], d["u_y"], d["u_z"]]
    dx = float(d["meta_dx"])
    v, vg, g = O.points_mac(u, dx, d["pts"])
    assert rel_l2(v, d["mac_v"]) < TOL
    assert rel_l2(vg, d["macg_v"]) < TOL
    assert rel_l2(g, np.stack([d["macg_gx"], d["macg_gy"], d["macg_gz"]], 1)) < TOL
    lin, mn, mx = O.points_dye(d["smoke"], dx, d["pts"])
    assert rel_l2(lin, d["lin"]) < TOL
    np.testing.assert_array_equal(mn, d["minv"])
    np.testing.assert_array_equal(mx, d["maxv"])
    T = [d["T_x"], d["T_y"], d["T_z"]]
    dT = [d["dT_x"], d["dT_y"], d["dT_z"]]
    d2T = [d["d2T_x"], d["d2T_y"], d["d2T_z"]]
    for var, name in [(O.HV_FD, "fd"), (O.HV_GARM, "garm"), (O.HV_FULL, "full")]:
        val, gval, grad = O.points_hermite(var, d["psi"], T, dT, d2T, dx, d["pts"])
        assert rel_l2(val, d["herm_" + name]) < TOL, name
        assert rel_l2(gval, d[f"hermg_{name}_v"]) < TOL, name
        ref = np.stack([d[f"hermg_{name}_x"], d[f"hermg_{name}_y"], d[f"hermg_{name}_z"]], 1)
        assert rel_l2(grad, ref) < TOL, name


def test_march_edge():
    d = load_golden("march_edge")
    u = [d["u_x"], d["u_y"], d["u_z"]]
    psi, T, dT = O.march_edge(u, d["in_psi"], [d["in_T_" + a] for a in "xyz"], [d["in_dT_" + a] for a in "xyz"],
                              float(d["meta_dx"]), d["meta_dt"], d["meta_eps"])
    assert rel_l2(psi, d["out_psi"]) < TOL
    for i, a in enumerate("xyz"):
        assert rel_l2(T[i], d["out_T_" + a]) < TOL
        assert rel_l2(dT[i], d["out_dT_" + a]) < TOL_T


def test_march_ed4():
    d = load_golden("march_ed4")
    u = [d["u_x"], d["u_y"], d["u_z"]]
    psi, T = O.march_ed4(u, d["in_psi"], [d["in_T_" + a] for a in "xyz"], float(d["meta_dx"]), d["meta_dt"],
                         d["meta_eps"])
    assert rel_l2(psi, d["out_psi"]) < TOL
    for i, a in enumerate("xyz"):
        assert rel_l2(T[i], d["out_T_" + a]) < TOL_T


def test_march_ed8_and_split():
    d = load_golden("march_ed8")
    u = [d["u_x"], d["u_y"], d["u_z"]]
    psi, T, dT, d2T = O.march_ed8(u, d["in_psi"], [d["in_T_" + a] for a in "xyz"],
                                  [d["in_dT_" + a] for a in "xyz"], [d["in_d2T_" + a] for a in "xyz"],
                                  float(d["meta_dx"]), d["meta_dt"], d["meta_eps"])
    assert rel_l2(psi, d["out_psi"]) < TOL
    for i, a in enumerate("xyz"):
        assert rel_l2(T[i], d["out_T_" + a]) < TOL_T
        assert rel_l2(dT[i], d["out_dT_" + a]) < TOL_DT
        assert rel_l2(d2T[i], d["out_d2T_" + a]) < TOL_D2T
    # the face split is evaluated on the reference's own marched state
    pf, tf = O.split_psi_hermite(d["out_psi"], [d["out_T_" + a] for a in "xyz"], [d["out_dT_" + a] for a in "xyz"],
                                 [d["out_d2T_" + a] for a in "xyz"], float(d["meta_dx"]))
    for i, a in enumerate("xyz"):
        assert rel_l2(pf[i], d["face_psi_" + a]) < TOL
        assert rel_l2(tf[i], d["face_T_" + a]) < TOL


def test_march_ge_and_split():
    d = load_golden("march_ge")
    u = [d["u_x"], d["u_y"], d["u_z"]]
    psi, T, dT, d2T = O.march_ge(u, d["in_psi"], [d["in_T_" + a] for a in "xyz"], [d["in_dT_" + a] for a in "xyz"],
                                 [d["in_d2T_" + a] for a in "xyz"], float(d["meta_dx"]), d["meta_dt"])
    assert rel_l2(psi, d["out_psi"]) < TOL
    for i, a in enumerate("xyz"):
        # no epsilon differences: the Jacobian is marched and composed, dT and
        # d2T are grid differences of it
        assert rel_l2(T[i], d["out_T_" + a]) < TOL
        assert rel_l2(dT[i], d["out_dT_" + a]) < 1e-5
        assert rel_l2(d2T[i], d["out_d2T_" + a]) < 1e-5
    # calc_fd_3_from_grad alone on the reference's marched Jacobian
    dT2, d2T2 = O.calc_fd_3_from_grad([d["out_T_" + a] for a in "xyz"], float(d["meta_dx"]))
    for i, a in enumerate("xyz"):
        assert rel_l2(dT2[i], d["out_dT_" + a]) < TOL
        assert rel_l2(d2T2[i], d["out_d2T_" + a]) < TOL
    pf, tf = O.split_psi_hermite(d["out_psi"], [d["out_T_" + a] for a in "xyz"], [d["out_dT_" + a] for a in "xyz"],
                                 [d["out_d2T_" + a] for a in "xyz"], float(d["meta_dx"]))
    for i, a in enumerate("xyz"):
        assert rel_l2(pf[i], d["face_psi_" + a]) < TOL
        assert rel_l2(tf[i], d["face_T_" + a]) < TOL


def test_efm_backtrack():
    d = load_golden("efm_backtrack")
    nsteps = len(d["dts"])
    cache = [[d[f"u{s}_{a}"] for a in "xyz"] for s in range(nsteps)]
    psi, T = O.efm_backtrack(cache, d["dts"], float(d["meta_dx"]))
    for i, a in enumerate("xyz"):
        assert rel_l2(psi[i], d["out_psi_" + a]) < TOL
        assert rel_l2(T[i], d["out_T_" + a]) < TOL


def test_face_kernels():
    d = load_golden("advect_faces")
    u = [d["u_x"], d["u_y"], d["u_z"]]
    dx, dt = float(d["meta_dx"]), d["meta_dt"]
    sl = O.advect_u_semi_lagrangian(u, dx, np.float32(0.5) * dt)
    for i, a in enumerate("xyz"):
        assert rel_l2(sl[i], d["sl_" + a]) < TOL
        phi, F = d["phi_in_" + a].copy(), d["F_in_" + a].copy()
        O.advance_map(u, phi, F, i, dx, dt)
        assert rel_l2(phi, d["phi_out_" + a]) < TOL
        assert rel_l2(F, d["F_out_" + a]) < TOL
        np.testing.assert_array_equal(O.clamp_u(d["clamp_in_" + a], u[i]), d["clamp_" + a])
    m = O.map_u(u, [d["F_out_" + a] for a in "xyz"], [d["phi_out_" + a] for a in "xyz"], dx)
    for i, a in enumerate("xyz"):
        assert rel_l2(m[i], d["mapu_" + a]) < TOL
    assert O.calc_max_speed(u) == pytest.approx(float(d["meta_max_speed"]), rel=1e-6)


@pytest.mark.parametrize("name,variant", [("pullback_edge", O.HV_GARM), ("pullback_ed4", O.HV_FD)])
def test_pullbacks(name, variant):
    d = load_golden(name)
    dx = float(d["meta_dx"])
    u0 = [d["u0_x"], d["u0_y"], d["u0_z"]]
    T = [d["T_x"], d["T_y"], d["T_z"]]
    dT = [d["dT_x"], d["dT_y"], d["dT_z"]] if "dT_x" in d else None
    u1 = O.map_u_psi(variant, u0, d["psi"], T, dT, dx)
    for i, a in enumerate("xyz"):
        assert rel_l2(u1[i], d["u1_" + a]) < TOL
    s1 = O.map_smoke_psi(variant, d["smoke0"], d["psi"], T, dT, dx)
    assert rel_l2(s1, d["smoke1"]) < TOL
    sc = d["smoke_cur"].copy()
    O.clamp_smoke_psi(variant, d["smoke0"], sc, d["psi"], T, dT, dx)
    assert rel_l2(sc, d["smoke_clamped"]) < TOL
    phi = [d["phi_x"], d["phi_y"], d["phi_z"]]
    assert rel_l2(O.map_smoke(d["smoke0"], phi, dx), d["smoke_fwd"]) < TOL
    sc = d["smoke_cur"].copy()
    O.clamp_smoke(d["smoke0"], sc, phi, dx)
    np.testing.assert_allclose(sc, d["smoke_fwd_clamped"], rtol=0, atol=1e-6)


def test_mgpcg_plain():
    d = load_golden("mgpcg_plain")
    u = [d["u_in_x"].copy(), d["u_in_y"].copy(), d["u_in_z"].copy()]
    it, div, p, rtr = O.poisson(u, base_level=1)
    assert rel_l2(div, d["div"]) < TOL
    assert abs(it - int(d["meta_iters"])) <= 1
    for i, a in enumerate("xyz"):
        assert rel_l2(u[i], d["u_out_" + a]) < 1e-5
    # pressure is defined up to the all-Neumann null space: compare mean-free
    assert rel_l2(p - p.mean(), d["pressure"] - d["pressure"].mean()) < 1e-4
    z, Ap, L = O.vcycle(d["vc_rhs"], base_level=1)
    assert L == int(d["meta_levels"])
    assert rel_l2(z, d["vc_z"]) < TOL
    assert rel_l2(Ap, d["ap_out"]) < TOL


def test_mgpcg_solid():
    d = load_golden("mgpcg_solid")
    u = [d["u_in_x"].copy(), d["u_in_y"].copy(), d["u_in_z"].copy()]
    it, div, p, bm1, bm2, dsum = O.poisson_solid(u, d["mask"], d["bvel"], base_level=1)
    np.testing.assert_array_equal(bm1, d["bm1"])
    np.testing.assert_array_equal(bm2, d["bm2"])
    assert rel_l2(div, d["div"]) < 1e-5
    assert abs(it - int(d["meta_iters"])) <= 1
    for i, a in enumerate("xyz"):
        assert rel_l2(u[i], d["u_out_" + a]) < 1e-4


def test_particles():
    d = load_golden("particles")
    res = tuple(int(v) for v in d["res"])
    dx = float(d["meta_dx"])
    num = int(d["meta_num"])
    dt, St, grav, dens, erad, Re, lrad = (float(v) for v in d["meta_params"])
    u = [d["u_x"], d["u_y"], d["u_z"]]
    L = [r * dx for r in res]
    vel = d["vel_in"].copy()
    pos = d["pos_in"].copy()
    acc = O.lp_acc(u, dx, vel, pos, num, dt, St, grav)
    assert rel_l2(acc, d["acc"]) < TOL
    O.lp_velocity(acc, vel, pos, dt, dx, num, L)
    assert rel_l2(vel, d["vel1"]) < TOL
    vd = O.lp_vel_diff(u, dx, vel, pos, num, St, dens, erad)
    assert rel_l2(vd, d["vel_diff"]) < TOL
    drag = O.lp_p2g(res, dx, vd, pos, d["rad"], num, lrad, L)
    for i, a in enumerate("xyz"):
        assert rel_l2(drag[i], d["drag_" + a]) < TOL
    O.lp_position(vel, pos, dt, num, L)
    assert rel_l2(pos, d["pos_out"]) < TOL
    vis = O.lp_viscous(u, dx, Re)
    for i, a in enumerate("xyz"):
        assert rel_l2(vis[i], d["vis_" + a]) < TOL


def test_init_rings():
    d = load_golden("init_rings")
    res = tuple(int(v) for v in d["res"])
    dx = float(d["meta_dx"])
    u = np.zeros(res + (3,), np.float32)
    smoke = np.zeros(res + (4,), np.float32)
    O.add_vortex_ring(res, dx, 0.1, 0.25, 0.06, [0.6, 0.5, 0.5], [0, 0, -1], [0, 1, 0], u, smoke, [1, 0, 0], 64)
    assert rel_l2(u, d["u_center"]) < 1e-5
    np.testing.assert_array_equal(smoke, d["smoke"])
    f = O.split_central_vector(d["u_center"])
    for i, a in enumerate("xyz"):
        assert rel_l2(f[i], d["u_" + a]) < TOL


def test_output_fields():
    """get_central_vector and curl (taichi_utils.py:69-100), bit for bit."""
    d = load_golden("output_fields")
    vc = O.get_central_vector([d["u_x"], d["u_y"], d["u_z"]])
    np.testing.assert_array_equal(vc, d["u_center"])
    np.testing.assert_array_equal(O.curl(d["u_center"], float(d["meta_dx"])), d["curl"])


def test_edge_steps():
    """Two full EDGE substeps of the driver loop (run_edge.py:588-712)."""
    d = load_golden("edge_steps")
    res = tuple(int(v) for v in d["res"])
    st = O.EdgeState(res, float(d["meta_dx"]), [d["u_in_x"], d["u_in_y"], d["u_in_z"]], d["smoke_in"])
    for i in range(2):
        dt, its = O.edge_substep(st, cfl=float(d["meta_cfl"]), reinit_every=int(d["meta_reinit"]),
                                 ed_eps=float(d["meta_eps"]), base_level=1)
        assert dt == pytest.approx(float(d[f"s{i}_meta_dt"]), rel=1e-5)
        for c, a in enumerate("xyz"):
            assert rel_l2(st.u[c], d[f"s{i}_u_{a}"]) < 1e-4, (i, a)
            assert rel_l2(st.T[c], d[f"s{i}_T_{a}"]) < 1e-5
            assert rel_l2(st.phi[c], d[f"s{i}_phi_{a}"]) < 1e-5
            assert rel_l2(st.dT[c], d[f"s{i}_dT_{a}"]) < TOL_T
        assert rel_l2(st.psi, d[f"s{i}_psi"]) < 1e-6
        assert rel_l2(st.smoke, d[f"s{i}_smoke"]) < 1e-4
