"""CUDA kernels of libedgeb200.so against the golden vectors (reference
sources) and the C oracle, through the C ABI.

Tolerances: the device kernels evaluate the B-spline separably on its 27
non-zero taps and the Hermite interpolants as a tensor-product contraction
(the reference sums 64 / 8x8 terms in loop order) and contract with FMA, so
float32 results differ from the reference's by rounding only: 1e-5 relative
L2 on plain outputs; epsilon-difference outputs carry the conditioning noted
in test_oracle_golden.py.
"""
import numpy as np
import pytest
import torch

from conftest import load_golden, rel_l2
from oracle import edge_oracle as O

pytestmark = pytest.mark.gpu

TOL = 1e-5
TOL_T = 2e-4
TOL_DT = 1e-2
TOL_D2T = 5e-2


def T_(a):
    return torch.from_numpy(np.ascontiguousarray(a, dtype=np.float32)).cuda()


def N_(t):
    torch.cuda.synchronize()
    return t.detach().cpu().numpy()


@pytest.fixture(scope="module")
def ops():
    from edgeb200 import ops as _ops
    return _ops


def test_points(ops):
    d = load_golden("interp_points")
    u = [T_(d["u_x"]), T_(d["u_y"]), T_(d["u_z"])]
    dx = float(d["meta_dx"])
    pts = T_(d["pts"])
    v, vg, g = ops.points_mac(u, dx, pts)
    assert rel_l2(N_(v), d["mac_v"]) < TOL
    assert rel_l2(N_(vg), d["macg_v"]) < TOL
    assert rel_l2(N_(g), np.stack([d["macg_gx"], d["macg_gy"], d["macg_gz"]], 1)) < TOL
    lin, mn, mx = ops.points_dye(T_(d["smoke"]), dx, pts)
    assert rel_l2(N_(lin), d["lin"]) < TOL
    np.testing.assert_array_equal(N_(mn), d["minv"])
    np.testing.assert_array_equal(N_(mx), d["maxv"])
    psi = T_(d["psi"])
    T = [T_(d["T_" + a]) for a in "xyz"]
    dT = [T_(d["dT_" + a]) for a in "xyz"]
    d2T = [T_(d["d2T_" + a]) for a in "xyz"]
    for var, name in [(0, "fd"), (1, "garm"), (2, "full")]:
        val, gval, grad = ops.points_hermite(var, psi, T, dT, d2T, dx, pts)
        assert rel_l2(N_(val), d["herm_" + name]) < TOL, name
        assert rel_l2(N_(gval), d[f"hermg_{name}_v"]) < TOL, name
        ref = np.stack([d[f"hermg_{name}_x"], d[f"hermg_{name}_y"], d[f"hermg_{name}_z"]], 1)
        assert rel_l2(N_(grad), ref) < TOL, name


def test_clamp_bound_rounding(ops):
    """At dim >= 64 the reference's clamp bound dim-2-1e-6 rounds to dim-2 in
    float32, so a coordinate can reach the last Hermite corner and the FD
    neighbour index is clamped by sample(); points on and beyond the upper
    faces of a 128-long axis exercise that."""
    rng = np.random.default_rng(7)
    res = (128, 6, 5)
    dx = 1.0 / 32.0
    psi = (O.center_coords(res, dx) + rng.normal(size=res + (3,)) * 0.01).astype(np.float32)
    T = [(np.eye(3)[c] + 0.1 * rng.normal(size=res + (3,))).astype(np.float32) for c in range(3)]
    dT = [(0.3 * rng.normal(size=res + (3,))).astype(np.float32) for _ in range(3)]
    L = np.array(res) * dx
    pts = np.stack([np.linspace(L[0] - 2 * dx, L[0] + dx, 40), rng.uniform(0, L[1], 40), rng.uniform(0, L[2], 40)],
                   -1).astype(np.float32)
    for var in (0, 1):
        ov, og, ogr = O.points_hermite(var, psi, T, dT, None, dx, pts)
        gv, gg, ggr = ops.points_hermite(var, T_(psi), [T_(t) for t in T], [T_(t) for t in dT], None, dx, T_(pts))
        assert rel_l2(N_(gv), ov) < TOL
        assert rel_l2(N_(ggr), ogr) < 1e-4


def test_march_edge(ops):
    d = load_golden("march_edge")
    u = [T_(d[k]) for k in ("u_x", "u_y", "u_z")]
    psi, T, dT = T_(d["in_psi"]), [T_(d["in_T_" + a]) for a in "xyz"], [T_(d["in_dT_" + a]) for a in "xyz"]
    opsi = torch.empty_like(psi)
    oT = [torch.empty_like(t) for t in T]
    odT = [torch.empty_like(t) for t in dT]
    ops.march_edge(u, float(d["meta_dx"]), float(d["meta_dt"]), float(d["meta_eps"]), psi, T, dT, opsi, oT, odT)
    assert rel_l2(N_(opsi), d["out_psi"]) < TOL
    for i, a in enumerate("xyz"):
        assert rel_l2(N_(oT[i]), d["out_T_" + a]) < TOL
        assert rel_l2(N_(odT[i]), d["out_dT_" + a]) < TOL_T


def test_march_edge_identity_matches_reset(ops):
    """The identity shortcut after a reinitialisation equals marching from a
    map reset by reset_to_identity_2 (hermite.py:657-674)."""
    rng = np.random.default_rng(3)
    res = (24, 16, 12)
    dx = 1.0 / 16
    u = [T_(0.5 * rng.normal(size=s)) for s in O.face_shapes(res)]
    psi = torch.empty(res + (3,), device="cuda")
    T = [torch.empty_like(psi) for _ in range(3)]
    dT = [torch.empty_like(psi) for _ in range(3)]
    ops.reset_cells(dx, psi, T, dT)
    outs = []
    for ident in (False, True):
        o = [torch.empty_like(psi) for _ in range(7)]
        ops.march_edge(u, dx, 0.02, 0.025 * dx, psi, T, dT, o[0], o[1:4], o[4:7], identity=ident)
        outs.append([N_(t) for t in o])
    # the analytic composition rounds once where the Hermite sum rounds ~30 times
    for a, b in zip(outs[0][:4], outs[1][:4]):
        assert rel_l2(a, b) < 1e-5
    for a, b in zip(outs[0][4:], outs[1][4:]):
        assert rel_l2(a, b) < 1e-3


def test_march_ed4(ops):
    d = load_golden("march_ed4")
    u = [T_(d[k]) for k in ("u_x", "u_y", "u_z")]
    psi, T = T_(d["in_psi"]), [T_(d["in_T_" + a]) for a in "xyz"]
    opsi = torch.empty_like(psi)
    oT = [torch.empty_like(t) for t in T]
    ops.march_ed4(u, float(d["meta_dx"]), float(d["meta_dt"]), float(d["meta_eps"]), psi, T, opsi, oT)
    assert rel_l2(N_(opsi), d["out_psi"]) < TOL
    for i, a in enumerate("xyz"):
        assert rel_l2(N_(oT[i]), d["out_T_" + a]) < TOL_T


def test_march_ed8_and_split(ops):
    d = load_golden("march_ed8")
    u = [T_(d[k]) for k in ("u_x", "u_y", "u_z")]
    psi = T_(d["in_psi"])
    T = [T_(d["in_T_" + a]) for a in "xyz"]
    dT = [T_(d["in_dT_" + a]) for a in "xyz"]
    d2T = [T_(d["in_d2T_" + a]) for a in "xyz"]
    o = [torch.empty_like(psi) for _ in range(7)] + [torch.empty_like(d2T[0]) for _ in range(3)]
    ops.march_ed8(u, float(d["meta_dx"]), float(d["meta_dt"]), float(d["meta_eps"]), psi, T, dT, d2T, o[0], o[1:4],
                  o[4:7], o[7:10])
    assert rel_l2(N_(o[0]), d["out_psi"]) < TOL
    for i, a in enumerate("xyz"):
        assert rel_l2(N_(o[1 + i]), d["out_T_" + a]) < TOL_T
        assert rel_l2(N_(o[4 + i]), d["out_dT_" + a]) < TOL_DT
        assert rel_l2(N_(o[7 + i]), d["out_d2T_" + a]) < TOL_D2T
    # split_psi_hermite on the reference's marched state
    res = tuple(int(v) for v in d["res"])
    fpsi = [torch.empty(s + (3,), device="cuda") for s in O.face_shapes(res)]
    fcol = [torch.empty(s + (3,), device="cuda") for s in O.face_shapes(res)]
    ops.face_map(2, float(d["meta_dx"]), T_(d["out_psi"]), [T_(d["out_T_" + a]) for a in "xyz"],
                 [T_(d["out_dT_" + a]) for a in "xyz"], [T_(d["out_d2T_" + a]) for a in "xyz"], fpsi, fcol)
    for i, a in enumerate("xyz"):
        assert rel_l2(N_(fpsi[i]), d["face_psi_" + a]) < TOL
        assert rel_l2(N_(fcol[i]), d["face_T_" + a]) < TOL


def test_face_kernels(ops):
    d = load_golden("advect_faces")
    u = [T_(d[k]) for k in ("u_x", "u_y", "u_z")]
    dx, dt = float(d["meta_dx"]), float(d["meta_dt"])
    sl = [torch.empty_like(t) for t in u]
    ops.advect_u_sl(u, dx, float(np.float32(0.5) * np.float32(dt)), sl)
    phi = [T_(d["phi_in_" + a]) for a in "xyz"]
    F = [T_(d["F_in_" + a]) for a in "xyz"]
    ops.advance_map(u, dx, dt, phi, F)
    mapped = [torch.empty_like(t) for t in u]
    ops.pullback_u(u, dx, [T_(d["phi_out_" + a]) for a in "xyz"], [T_(d["F_out_" + a]) for a in "xyz"], mapped)
    cl = [torch.empty_like(t) for t in u]
    ops.clamp_u([T_(d["clamp_in_" + a]) for a in "xyz"], u, cl)
    ms = torch.zeros(1, device="cuda")
    ops.max_speed(u, ms)
    for i, a in enumerate("xyz"):
        assert rel_l2(N_(sl[i]), d["sl_" + a]) < TOL
        assert rel_l2(N_(phi[i]), d["phi_out_" + a]) < TOL
        assert rel_l2(N_(F[i]), d["F_out_" + a]) < TOL
        assert rel_l2(N_(mapped[i]), d["mapu_" + a]) < TOL
        np.testing.assert_array_equal(N_(cl[i]), d["clamp_" + a])
    assert float(N_(ms)[0]) == pytest.approx(float(d["meta_max_speed"]), rel=1e-6)


@pytest.mark.parametrize("name,variant", [("pullback_edge", 1), ("pullback_ed4", 0)])
def test_pullbacks(ops, name, variant):
    d = load_golden(name)
    dx = float(d["meta_dx"])
    res = tuple(int(v) for v in d["res"])
    u0 = [T_(d["u0_" + a]) for a in "xyz"]
    psi = T_(d["psi"])
    T = [T_(d["T_" + a]) for a in "xyz"]
    dT = [T_(d["dT_" + a]) for a in "xyz"] if "dT_x" in d else None
    smoke0 = T_(d["smoke0"])
    # direct kernels (map_u_psi, map_smoke_psi, clamp_smoke_psi)
    u1 = [torch.empty_like(t) for t in u0]
    ops.map_u_psi(variant, u0, u1, dx, psi, T, dT)
    s1 = torch.empty_like(smoke0)
    ops.smoke_psi(variant, 0, smoke0, s1, dx, psi, T, dT)
    sc = T_(d["smoke_cur"])
    ops.smoke_psi(variant, 1, smoke0, sc, dx, psi, T, dT)
    for i, a in enumerate("xyz"):
        assert rel_l2(N_(u1[i]), d["u1_" + a]) < TOL
    assert rel_l2(N_(s1), d["smoke1"]) < TOL
    assert rel_l2(N_(sc), d["smoke_clamped"]) < TOL
    # the deduplicated path: Hermite once per face, then the pullbacks
    fpsi = [torch.empty(s + (3,), device="cuda") for s in O.face_shapes(res)]
    fcol = [torch.empty(s + (3,), device="cuda") for s in O.face_shapes(res)]
    ops.face_map(variant, dx, psi, T, dT, None, fpsi, fcol)
    u2 = [torch.empty_like(t) for t in u0]
    ops.pullback_u(u0, dx, fpsi, fcol, u2)
    s2 = torch.empty_like(smoke0)
    ops.pullback_dye(smoke0, dx, fpsi, s2)
    sc2 = T_(d["smoke_cur"])
    ops.pullback_dye(None, dx, fpsi, sc2, clampsrc=smoke0, inplace_clamp=True)
    for i, a in enumerate("xyz"):
        assert rel_l2(N_(u2[i]), d["u1_" + a]) < TOL
    assert rel_l2(N_(s2), d["smoke1"]) < TOL
    assert rel_l2(N_(sc2), d["smoke_clamped"]) < TOL
    # forward-map dye pullback and clamp (map_smoke / clamp_smoke)
    phi = [T_(d["phi_" + a]) for a in "xyz"]
    s3 = torch.empty_like(smoke0)
    ops.pullback_dye(smoke0, dx, phi, s3)
    sc3 = T_(d["smoke_cur"])
    ops.pullback_dye(None, dx, phi, sc3, clampsrc=smoke0, inplace_clamp=True)
    assert rel_l2(N_(s3), d["smoke_fwd"]) < TOL
    np.testing.assert_allclose(N_(sc3), d["smoke_fwd_clamped"], rtol=0, atol=1e-6)


def test_fused_bfecc_arithmetic(ops):
    """err = scale*(F.u(phi) - init) and out = sub - col.e(pos) equal the
    reference's separate add_fields / scale_field passes."""
    rng = np.random.default_rng(11)
    res = (16, 12, 10)
    dx = 1 / 12
    u = [T_(rng.normal(size=s)) for s in O.face_shapes(res)]
    init = [T_(rng.normal(size=s)) for s in O.face_shapes(res)]
    pos = [T_(O.face_coords(res, dx, a) + 0.2 * dx * rng.normal(size=s + (3,))) for a, s in
           enumerate(O.face_shapes(res))]
    col = [T_(np.eye(3)[a] + 0.1 * rng.normal(size=s + (3,))) for a, s in enumerate(O.face_shapes(res))]
    plain = [torch.empty_like(t) for t in u]
    ops.pullback_u(u, dx, pos, col, plain)
    fused = [torch.empty_like(t) for t in u]
    ops.pullback_u(u, dx, pos, col, fused, init=init, scale=0.5)
    sub = [torch.empty_like(t) for t in u]
    ops.pullback_u(u, dx, pos, col, sub, sub=init)
    for p, f, s, i in zip(plain, fused, sub, init):
        np.testing.assert_allclose(N_(f), 0.5 * (N_(p) - N_(i)), rtol=1e-6, atol=1e-6)
        np.testing.assert_allclose(N_(s), N_(i) - N_(p), rtol=1e-6, atol=1e-6)


def test_larger_grid_vs_oracle(ops):
    """A 48x32x24 grid with a non-trivial map: marches and pullbacks against
    the oracle (sizes the oracle finishes in seconds)."""
    rng = np.random.default_rng(5)
    res = (48, 32, 24)
    dx = 1.0 / 32
    u = [(0.8 * np.sin(np.indices(s)[0] * 0.2 + a) * np.cos(np.indices(s)[1] * 0.15)).astype(np.float32)
         for a, s in enumerate(O.face_shapes(res))]
    psi = (O.center_coords(res, dx) + 0.3 * dx * rng.uniform(-1, 1, size=res + (3,))).astype(np.float32)
    T = [(np.eye(3)[c] + 0.05 * rng.normal(size=res + (3,))).astype(np.float32) for c in range(3)]
    dT = [(0.2 * rng.normal(size=res + (3,))).astype(np.float32) for _ in range(3)]
    dt, eps = 0.01, 0.025 * dx
    opsi, oT, odT = O.march_edge(u, psi, T, dT, dx, dt, eps)
    gu = [T_(a) for a in u]
    g = [torch.empty(res + (3,), device="cuda") for _ in range(7)]
    ops.march_edge(gu, dx, dt, eps, T_(psi), [T_(t) for t in T], [T_(t) for t in dT], g[0], g[1:4], g[4:7])
    assert rel_l2(N_(g[0]), opsi) < TOL
    # dT is an epsilon difference of four marched Jacobians: an error of a few
    # ulp in T (~1e-6 here) becomes ~1e-6 / (8 eps) absolute, i.e. ~1e-3 of
    # this rough random map's dT
    for i in range(3):
        assert rel_l2(N_(g[1 + i]), oT[i]) < TOL
        assert rel_l2(N_(g[4 + i]), odT[i]) < 2e-3
    ou = O.map_u_psi(1, u, opsi, oT, odT, dx)
    gu1 = [torch.empty_like(t) for t in gu]
    ops.map_u_psi(1, gu, gu1, dx, g[0], g[1:4], g[4:7])
    for i in range(3):
        assert rel_l2(N_(gu1[i]), ou[i]) < 1e-4


@pytest.mark.parametrize("variant", [0, 1, 2])
def test_packed_layout_roundtrip_and_march(ops, variant):
    """pack -> unpack is the identity, and the packed march / face map equal
    the reference-layout ones."""
    rng = np.random.default_rng(21 + variant)
    res = (24, 16, 12)
    dx = 1.0 / 16
    planes = 8  # every packed map (edge_packed_planes)
    psi = T_(O.center_coords(res, dx) + 0.3 * dx * rng.uniform(-1, 1, size=res + (3,)))
    T = [T_(np.eye(3)[c] + 0.05 * rng.normal(size=res + (3,))) for c in range(3)]
    dT = [T_(0.2 * rng.normal(size=res + (3,))) for _ in range(3)] if variant else None
    d2T = [T_(0.2 * rng.normal(size=res)) for _ in range(3)] if variant == 2 else None
    packed = torch.zeros((planes,) + res + (4,), device="cuda")
    ops.map_pack(variant, psi, T, dT, d2T, packed)
    psi2 = torch.empty_like(psi)
    T2 = [torch.empty_like(t) for t in T]
    dT2 = [torch.empty_like(t) for t in dT] if dT else None
    d2T2 = [torch.empty_like(t) for t in d2T] if d2T else None
    ops.map_unpack(variant, packed, psi2, T2, dT2, d2T2)
    np.testing.assert_array_equal(N_(psi2), N_(psi))
    for a, b in zip(T2, T):
        np.testing.assert_array_equal(N_(a), N_(b))
    u = [T_(0.5 * rng.normal(size=s)) for s in O.face_shapes(res)]
    out = torch.zeros_like(packed)
    ops.march_packed(variant, u, dx, 0.02, 0.025 * dx, packed, out, res)
    o = [torch.empty_like(psi) for _ in range(7)] + [torch.empty(res, device="cuda") for _ in range(3)]
    if variant == 1:
        ops.march_edge(u, dx, 0.02, 0.025 * dx, psi, T, dT, o[0], o[1:4], o[4:7])
    elif variant == 0:
        ops.march_ed4(u, dx, 0.02, 0.025 * dx, psi, T, o[0], o[1:4])
    else:
        ops.march_ed8(u, dx, 0.02, 0.025 * dx, psi, T, dT, d2T, o[0], o[1:4], o[4:7], o[7:10])
    p2 = torch.empty_like(psi)
    T3 = [torch.empty_like(t) for t in T]
    dT3 = [torch.empty_like(t) for t in T] if dT else None
    d2T3 = [torch.empty(res, device="cuda") for _ in range(3)] if d2T else None
    ops.map_unpack(variant, out, p2, T3, dT3, d2T3)
    assert rel_l2(N_(p2), N_(o[0])) < 1e-6
    for a, b in zip(T3, o[1:4]):
        assert rel_l2(N_(a), N_(b)) < 1e-5
    fp = [torch.empty(s + (3,), device="cuda") for s in O.face_shapes(res)]
    fc = [torch.empty(s + (3,), device="cuda") for s in O.face_shapes(res)]
    fp2 = [torch.empty_like(t) for t in fp]
    fc2 = [torch.empty_like(t) for t in fc]
    ops.face_map(variant, dx, psi, T, dT, d2T, fp, fc)
    ops.face_map_packed(variant, dx, packed, res, fp2, fc2)
    for a, b in zip(fp + fc, fp2 + fc2):
        assert rel_l2(N_(b), N_(a)) < 1e-6


def test_march_ge_and_split(ops):
    """GE march advect_ps_garm against the reference's own output."""
    d = load_golden("march_ge")
    u = [T_(d[k]) for k in ("u_x", "u_y", "u_z")]
    psi = T_(d["in_psi"])
    T = [T_(d["in_T_" + a]) for a in "xyz"]
    dT = [T_(d["in_dT_" + a]) for a in "xyz"]
    d2T = [T_(d["in_d2T_" + a]) for a in "xyz"]
    o = [torch.empty_like(psi) for _ in range(7)] + [torch.empty_like(d2T[0]) for _ in range(3)]
    ops.march_ge(u, float(d["meta_dx"]), float(d["meta_dt"]), psi, T, dT, d2T, o[0], o[1:4], o[4:7], o[7:10])
    assert rel_l2(N_(o[0]), d["out_psi"]) < TOL
    for i, a in enumerate("xyz"):
        # T is marched and composed (no epsilon difference); dT, d2T are grid
        # differences of T over 4 dx and 6 dx
        assert rel_l2(N_(o[1 + i]), d["out_T_" + a]) < TOL
        assert rel_l2(N_(o[4 + i]), d["out_dT_" + a]) < 1e-4
        assert rel_l2(N_(o[7 + i]), d["out_d2T_" + a]) < 1e-4
    # calc_fd_3_from_grad alone, on the reference's T: same float32 expressions
    dT2 = [torch.empty_like(t) for t in T]
    d2T2 = [torch.empty_like(t) for t in d2T]
    ops.calc_fd_3_from_grad(float(d["meta_dx"]), [T_(d["out_T_" + a]) for a in "xyz"], dT2, d2T2)
    for i, a in enumerate("xyz"):
        assert rel_l2(N_(dT2[i]), d["out_dT_" + a]) < 1e-6
        assert rel_l2(N_(d2T2[i]), d["out_d2T_" + a]) < 1e-6


def test_march_ge_larger_grid_and_packed(ops):
    """48x32x24 GE march against the oracle, and the packed-plane march equal
    to the reference-layout one."""
    rng = np.random.default_rng(55)
    res = (48, 32, 24)
    dx = 1.0 / 32
    u = [(0.8 * np.sin(np.indices(s)[0] * 0.2 + a) * np.cos(np.indices(s)[1] * 0.15)).astype(np.float32)
         for a, s in enumerate(O.face_shapes(res))]
    psi = (O.center_coords(res, dx) + 0.3 * dx * rng.uniform(-1, 1, size=res + (3,))).astype(np.float32)
    T = [(np.eye(3)[c] + 0.05 * rng.normal(size=res + (3,))).astype(np.float32) for c in range(3)]
    dT = [(0.2 * rng.normal(size=res + (3,))).astype(np.float32) for _ in range(3)]
    d2T = [(0.2 * rng.normal(size=res)).astype(np.float32) for _ in range(3)]
    dt = 0.01
    opsi, oT, odT, od2T = O.march_ge(u, psi, T, dT, d2T, dx, dt)
    gu = [T_(a) for a in u]
    g = [torch.empty(res + (3,), device="cuda") for _ in range(7)] + [torch.empty(res, device="cuda") for _ in range(3)]
    gin = (T_(psi), [T_(t) for t in T], [T_(t) for t in dT], [T_(t) for t in d2T])
    ops.march_ge(gu, dx, dt, *gin, g[0], g[1:4], g[4:7], g[7:10])
    assert rel_l2(N_(g[0]), opsi) < TOL
    for i in range(3):
        assert rel_l2(N_(g[1 + i]), oT[i]) < TOL
        assert rel_l2(N_(g[4 + i]), odT[i]) < 1e-4
        assert rel_l2(N_(g[7 + i]), od2T[i]) < 1e-4
    packed = torch.zeros((8,) + res + (4,), device="cuda")
    ops.map_pack(2, *gin, packed)
    out = torch.zeros_like(packed)
    ops.march_ge_packed(gu, dx, dt, packed, out, res)
    p = [torch.empty_like(t) for t in g]
    ops.map_unpack(2, out, p[0], p[1:4], p[4:7], p[7:10])
    for a, b in zip(p, g):
        assert rel_l2(N_(a), N_(b)) < 1e-6


def test_dropin_hermite_marches():
    """The sim/hermite.py drop-in entry points, called with the reference's
    arguments (fields in place, scratch fields, X), reproduce the reference's
    marches on its golden vectors."""
    from sim import hermite as H
    for name in ("march_ed8", "march_ge", "march_edge"):
        d = load_golden(name)
        res = tuple(int(v) for v in d["res"])
        dx, dt = float(d["meta_dx"]), float(d["meta_dt"])
        X = T_(O.center_coords(res, dx))
        u = [T_(d[k]) for k in ("u_x", "u_y", "u_z")]
        psi = T_(d["in_psi"])
        T = [T_(d["in_T_" + a]) for a in "xyz"]
        dT = [T_(d["in_dT_" + a]) for a in "xyz"]
        if name == "march_edge":
            tmp = [torch.empty_like(psi) for _ in range(7)]
            H.advect_psi_garm_ed4_fusion_unroll(*tmp, psi, *T, *dT, *u, X, dx, dt, float(d["meta_eps"]))
        else:
            d2T = [T_(d["in_d2T_" + a]) for a in "xyz"]
            if name == "march_ed8":
                tmp = [torch.empty_like(psi) for _ in range(8)]
                H.advect_ps_hermite_ed8(*tmp, psi, *T, *dT, *d2T, *u, X, dx, dt, float(d["meta_eps"]))
            else:
                tmp = [torch.empty_like(psi) for _ in range(4)]
                H.advect_ps_garm(*tmp, psi, *T, *dT, *d2T, *u, X, dx, dt)
            for i, a in enumerate("xyz"):
                assert rel_l2(N_(d2T[i]), d["out_d2T_" + a]) < TOL_D2T, name
        assert rel_l2(N_(psi), d["out_psi"]) < TOL, name
        for i, a in enumerate("xyz"):
            assert rel_l2(N_(T[i]), d["out_T_" + a]) < TOL_T, name
            assert rel_l2(N_(dT[i]), d["out_dT_" + a]) < TOL_DT, name


def test_efm_backtrack(ops):
    """EFM backward face map through cached velocities: against the
    reference's backtrack_psi_grid, and against the oracle at 48x32x24 with
    twelve cached steps (one launch for the whole chain)."""
    d = load_golden("efm_backtrack")
    n = len(d["dts"])
    res = tuple(int(v) for v in d["res"])
    cache = [[T_(d[f"u{s}_{a}"]) for a in "xyz"] for s in range(n)]
    psi = [torch.empty(s + (3,), device="cuda") for s in O.face_shapes(res)]
    T = [torch.empty(s + (3,), device="cuda") for s in O.face_shapes(res)]
    ops.efm_backtrack(cache, [float(x) for x in d["dts"]], float(d["meta_dx"]), psi, T)
    for i, a in enumerate("xyz"):
        assert rel_l2(N_(psi[i]), d["out_psi_" + a]) < TOL
        assert rel_l2(N_(T[i]), d["out_T_" + a]) < TOL
    rng = np.random.default_rng(77)
    res = (48, 32, 24)
    dx = 1.0 / 32
    cache = []
    for s in range(12):
        cache.append([(0.6 * np.sin(np.indices(sh)[0] * 0.2 + a + 0.1 * s) * np.cos(np.indices(sh)[1] * 0.15)
                       + 0.05 * rng.normal(size=sh)).astype(np.float32) for a, sh in enumerate(O.face_shapes(res))])
    dts = [np.float32(0.4 * dx / 0.7) for _ in cache]
    opsi, oT = O.efm_backtrack(cache, dts, dx)
    psi = [torch.empty(s + (3,), device="cuda") for s in O.face_shapes(res)]
    T = [torch.empty(s + (3,), device="cuda") for s in O.face_shapes(res)]
    ops.efm_backtrack([[T_(a) for a in c] for c in cache], [float(x) for x in dts], dx, psi, T)
    for i in range(3):
        assert rel_l2(N_(psi[i]), opsi[i]) < TOL
        assert rel_l2(N_(T[i]), oT[i]) < 1e-4
