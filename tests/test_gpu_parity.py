"""Step-level parity of the device driver (edgeb200.sim.EdgeSim) with the
oracle's substep, with the projection's stopping point taken out of the
comparison.

The reference stops CG when r.r < max(abs_tol, rel_tol z.r0) on the
recursion's residual (mgpcg.py:224-254), and its dot products are float32
atomics whose order is not reproducible; on the benchmark's flows the
absolute 1e-12 binds while the right-hand side is small, so the solve stops
at a loose relative residual and two implementations that sum in another
order can stop one iteration apart; the velocity then differs by the last CG
update and every later kernel carries that difference.  The tests here take
that out:

  * every kernel outside the projection is compared when the device, the
    oracle and the oracle's twin are all handed the device's projected
    velocity;
  * whole steps are compared when the projections run a fixed number of CG
    iterations, past the point where the solution stops changing in float32;
  * the configuration-0 flow (64x32x32 leapfrogging rings, 4 levels, reinit
    every 12 steps) runs 24 steps, across two reinitialisations, both ways.

What remains is float32 rounding, amplified by the reference's epsilon
differences; the oracle's twin build measures it per case (K_FLOOR below).
"""
import numpy as np
import pytest
import torch

from conftest import load_golden, rel_l2
from oracle import edge_oracle as O

pytestmark = pytest.mark.gpu

TOL = 1e-5


def T_(a):
    return torch.from_numpy(np.ascontiguousarray(a, dtype=np.float32)).cuda()


def N_(t):
    torch.cuda.synchronize()
    return t.cpu().numpy()


# ---------------------------------------------------------------------------
# set-up kernels against the reference-source goldens
# ---------------------------------------------------------------------------
def test_vortex_ring_and_split_vs_golden():
    """add_vortex_ring_and_smoke (init_conditions.py:11-36) and
    split_central_vector (taichi_utils.py:103-116) on the device."""
    from edgeb200 import ops
    from edgeb200.fields import zeros_cells, zeros_faces
    d = load_golden("init_rings")
    res = tuple(int(v) for v in d["res"])
    dx = float(d["meta_dx"])
    u = zeros_cells(res, 3)
    smoke = zeros_cells(res, 4)
    ops.add_vortex_ring(dx, 0.1, 0.25, 0.06, (0.6, 0.5, 0.5), (0., 0., -1.), (0., 1., 0.), u, smoke, (1., 0., 0.),
                        64)
    assert rel_l2(N_(u), d["u_center"]) < TOL
    np.testing.assert_array_equal(N_(smoke), d["smoke"])
    f = zeros_faces(res)
    ops.split_central_vector(T_(d["u_center"]), f)
    for i, a in enumerate("xyz"):
        np.testing.assert_array_equal(N_(f[i]), d["u_" + a])


def test_output_helpers_vs_golden():
    """get_central_vector and curl (taichi_utils.py:69-100) on the device,
    bit for bit."""
    from util.taichi_utils import curl, get_central_vector
    d = load_golden("output_fields")
    res = tuple(int(v) for v in d["res"])
    vc = torch.empty(res + (3,), device="cuda")
    get_central_vector(T_(d["u_x"]), T_(d["u_y"]), T_(d["u_z"]), vc)
    np.testing.assert_array_equal(N_(vc), d["u_center"])
    w = torch.empty(res + (3,), device="cuda")
    curl(T_(d["u_center"]), w, float(d["meta_dx"]))
    np.testing.assert_array_equal(N_(w), d["curl"])


# ---------------------------------------------------------------------------
# whole steps
# ---------------------------------------------------------------------------
# Two float32 evaluations of the reference algorithm that differ only in
# rounding disagree by more than 1e-5 on these flows: the ED4/ED8 maps and
# the EDGE mixed derivatives are epsilon differences (eps = dx/40), which
# turn one ulp of psi into ulp/eps in the gradient, and the BFECC clamps and
# solid boundaries pass such differences on.  The oracle's twin build
# (oracle/_build/libedge_oracle_fma.so: the same source with multiply-adds
# fused) measures that floor on every case below; the device must agree with
# the oracle to 1e-5, or to within K times the floor where the floor itself
# exceeds 1e-5 / K.
K_FLOOR = 8.0


def _bound(floor):
    return max(TOL, K_FLOOR * floor)


def _hook_projection(sim):
    """Record the velocity before and after every projection of `sim`."""
    rec = []
    orig = sim.proj.poisson

    def poisson(ux, uy, uz, f=None, **kw):
        pre = [t.clone() for t in (ux, uy, uz)]
        orig(ux, uy, uz, f=f, **kw)
        rec.append((pre, [t.clone() for t in (ux, uy, uz)], None if f is None else [t.clone() for t in f]))
    sim.proj.poisson = poisson
    return rec


def _replay(rec, seen):
    """An oracle projection that records the oracle's velocity before the
    projection and continues from the device's projected velocity (and
    force), so that the solver's stopping point is out of the comparison."""
    q = list(rec)

    def project(u, force):
        pre, post, f = q.pop(0)
        seen.append([a.copy() for a in u])
        for a, p in zip(u, post):
            a[...] = N_(p)
        if force is not None:
            for a, p in zip(force, f):
                a[...] = N_(p)
        return 0
    return project


def _fields(src, names):
    out = {}
    for n in names:
        if n == "smoke":
            out[n] = [src["smoke"]]
        elif n == "psi":
            out[n] = [src["psi"]]
        elif n == "T":
            out[n] = list(src["T"])
        elif n == "phi":
            out[n] = list(src["phi"])
        elif n == "init_smoke":
            out[n] = [src["init_smoke"]]
        elif n in ("pos", "vel"):
            out[n] = [src[n]]
    return out


def _sim_fields(sim, names):
    m = sim.map if any(n in names for n in ("psi", "T")) else None
    src = {"smoke": N_(sim.smoke), "init_smoke": N_(sim.init_smoke), "phi": [N_(t) for t in sim.phi]}
    if m is not None:
        src["psi"] = N_(m["psi"])
        src["T"] = [N_(t) for t in m["T"]]
    if sim.particles is not None:
        src["pos"], src["vel"] = N_(sim.particles["pos"]), N_(sim.particles["vel"])
    return _fields(src, names)


def _orc_fields(st, names, P=None):
    src = {"smoke": st.smoke, "init_smoke": st.init_smoke, "phi": st.phi, "psi": st.psi, "T": st.T}
    if P is not None:
        src["pos"], src["vel"] = P["pos"], P["vel"]
    return _fields(src, names)


def _err(a, b):
    return max(rel_l2(x, y) for x, y in zip(a, b))


def _isolated(sim, u, smoke, steps, names, particles=None, **kw):
    """Step the device, the oracle and the oracle's twin, all three from the
    device's projected velocities; returns per quantity the worst
    device-vs-oracle and twin-vs-oracle differences over the steps: the
    velocity entering each projection ("u_pre") and `names` after each step."""
    res, dx = sim.res, sim.dx
    rec = _hook_projection(sim)
    A = O.EdgeState(res, dx, [N_(t) for t in u], N_(smoke))
    B = O.EdgeState(res, dx, [N_(t) for t in u], N_(smoke))
    PA = PB = None
    if particles is not None:
        PA = {k: (v.copy() if isinstance(v, np.ndarray) else v) for k, v in particles.items()}
        PB = {k: (v.copy() if isinstance(v, np.ndarray) else v) for k, v in particles.items()}
    dev, floor = {}, {}
    for i in range(steps):
        rec.clear()
        dt = sim.step()
        seen_a, seen_b = [], []
        O.edge_substep(A, dt=dt, project=_replay(rec, seen_a), particles=PA, **kw)
        with O.fma_twin():
            O.edge_substep(B, dt=dt, project=_replay(rec, seen_b), particles=PB, **kw)
        for (pre, _, _), a, b in zip(rec, seen_a, seen_b):
            dev["u_pre"] = max(dev.get("u_pre", 0.0), _err([N_(t) for t in pre], a))
            floor["u_pre"] = max(floor.get("u_pre", 0.0), _err(b, a))
        fa, fb, fd = _orc_fields(A, names, PA), _orc_fields(B, names, PB), _sim_fields(sim, names)
        for n in names:
            dev[n] = max(dev.get(n, 0.0), _err(fd[n], fa[n]))
            floor[n] = max(floor.get(n, 0.0), _err(fb[n], fa[n]))
    return dev, floor


def _check(dev, floor, tag):
    bad = {n: (dev[n], floor[n], _bound(floor[n])) for n in dev if dev[n] > _bound(floor[n])}
    assert not bad, (tag, bad)


@pytest.mark.parametrize("variant", ["edge", "ed4", "ed8", "ge", "efm"])
def test_step_kernels_outside_projection(variant):
    """Every kernel of the substep except the projection: the velocity
    entering each projection, the dye, the forward map and the backward
    map."""
    from edgeb200.sim import EdgeSim, leapfrog_init
    res, dx = (32, 16, 16), 1.0 / 16
    u, smoke = leapfrog_init(res, dx, radii=(0.21, 0.28), sigma=0.06, circulation=0.2, num_samples=200)
    sim = EdgeSim(res, dx, variant=variant, reinit_every=3, base_level=2, visualize_dt=1e9)
    sim.set_velocity(*u)
    sim.set_smoke(smoke)
    names = ("smoke", "phi") if variant == "efm" else ("smoke", "phi", "psi")
    dev, floor = _isolated(sim, u, smoke, 6, names, reinit_every=3, base_level=2, variant=variant)
    _check(dev, floor, variant)
    if variant == "edge":
        assert max(dev.values()) < TOL, dev


@pytest.mark.parametrize("variant", ["edge", "ed4", "ed8", "ge", "efm"])
def test_steps_with_fixed_iteration_projection(variant):
    """Whole substeps (velocity and dye) when the projections run the same
    fixed number of CG iterations (tolerances 0): the stopping point no
    longer depends on the order of the dot products."""
    from edgeb200.sim import EdgeSim, leapfrog_init
    res, dx = (32, 16, 16), 1.0 / 16
    u, smoke = leapfrog_init(res, dx, radii=(0.21, 0.28), sigma=0.06, circulation=0.2, num_samples=200)
    A = O.EdgeState(res, dx, [N_(t) for t in u], N_(smoke))
    B = O.EdgeState(res, dx, [N_(t) for t in u], N_(smoke))
    sim = EdgeSim(res, dx, variant=variant, reinit_every=3, base_level=2, visualize_dt=1e9, abs_tol=0.0,
                  rel_tol=0.0)
    sim.max_iters = 16
    sim.set_velocity(*u)
    sim.set_smoke(smoke)
    kw = dict(reinit_every=3, base_level=2, variant=variant, abs_tol=0.0, rel_tol=0.0, max_iters=16)
    dev, floor = {}, {}
    for i in range(6):
        dt = sim.step()
        O.edge_substep(A, dt=dt, **kw)
        with O.fma_twin():
            O.edge_substep(B, dt=dt, **kw)
        for n, d, a, b in (("u", [N_(t) for t in sim.u], A.u, B.u), ("smoke", [N_(sim.smoke)], [A.smoke], [B.smoke])):
            dev[n] = max(dev.get(n, 0.0), _err(d, a))
            floor[n] = max(floor.get(n, 0.0), _err(b, a))
    _check(dev, floor, variant)
    if variant == "edge":
        assert max(dev.values()) < TOL, dev


def _config0(res=(64, 32, 32)):
    from edgeb200.sim import leapfrog_init
    dx = 1.0 / res[1]
    u, smoke = leapfrog_init(res, dx, radii=(0.21, 0.28), sigma=0.03, circulation=1.0, x_start=0.3)
    return res, dx, u, smoke


def test_config0_leapfrog_24_steps_outside_projection():
    """The 64x32x32 leapfrogging rings (4 levels, reinit every 12) for 24
    EDGE steps, two reinitialisations: every non-solver kernel."""
    from edgeb200.sim import EdgeSim
    res, dx, u, smoke = _config0()
    sim = EdgeSim(res, dx, variant="edge", reinit_every=12, base_level=2, visualize_dt=1e9)
    sim.set_velocity(*u)
    sim.set_smoke(smoke)
    dev, floor = _isolated(sim, u, smoke, 24, ("smoke", "psi", "T"), reinit_every=12, base_level=2)
    _check(dev, floor, "config0")


def test_config0_leapfrog_24_steps_fixed_iterations():
    """The same 24 steps with both projections at a fixed 12 CG iterations:
    velocity and dye at every step."""
    from edgeb200.sim import EdgeSim
    res, dx, u, smoke = _config0()
    A = O.EdgeState(res, dx, [N_(t) for t in u], N_(smoke))
    B = O.EdgeState(res, dx, [N_(t) for t in u], N_(smoke))
    sim = EdgeSim(res, dx, variant="edge", reinit_every=12, base_level=2, visualize_dt=1e9, abs_tol=0.0,
                  rel_tol=0.0)
    sim.max_iters = 12
    sim.set_velocity(*u)
    sim.set_smoke(smoke)
    kw = dict(reinit_every=12, base_level=2, abs_tol=0.0, rel_tol=0.0, max_iters=12)
    dev, floor = {}, {}
    for i in range(24):
        dt = sim.step()
        O.edge_substep(A, dt=dt, **kw)
        with O.fma_twin():
            O.edge_substep(B, dt=dt, **kw)
        for n, d, a, b in (("u", [N_(t) for t in sim.u], A.u, B.u), ("smoke", [N_(sim.smoke)], [A.smoke], [B.smoke])):
            dev[n] = max(dev.get(n, 0.0), _err(d, a))
            floor[n] = max(floor.get(n, 0.0), _err(b, a))
    _check(dev, floor, "config0 fixed")


def test_step_128x64x64_outside_projection():
    """Two EDGE steps on a 128x64x64 grid (two levels outside the
    shared-memory coarse group), non-solver kernels."""
    from edgeb200.sim import EdgeSim
    res, dx, u, smoke = _config0((128, 64, 64))
    sim = EdgeSim(res, dx, variant="edge", reinit_every=12, base_level=2, visualize_dt=1e9)
    sim.set_velocity(*u)
    sim.set_smoke(smoke)
    dev, floor = _isolated(sim, u, smoke, 2, ("smoke", "psi"), reinit_every=12, base_level=2)
    _check(dev, floor, "128x64x64")


def test_solid_and_particle_steps_outside_projection():
    """The solid (MGPCG_Solid_3) path with dye emitters, and the two-way
    coupled particle path (Poisson_with_buffer), non-solver parts."""
    from edgeb200.sim import EdgeSim, delta_emitters, leapfrog_init, uniform_flow, wedge_mask
    res, dx = (32, 16, 16), 1.0 / 16
    mask, bvel = wedge_mask(res, dx, apex=(0.35, 0.5, 0.4), chord=0.6, thickness_cells=2)
    u = uniform_flow(res, (0.6 * 0.94, 0.0, 0.6 * 0.34))
    em = delta_emitters(offset=(0.3, 0.5, 0.45), radius=0.1)
    sim = EdgeSim(res, dx, variant="edge", reinit_every=4, base_level=2, visualize_dt=1e9, solid=(mask, bvel),
                  emitters=em)
    sim.set_velocity(*u)
    zero = torch.zeros(res + (4,), device="cuda")
    dev, floor = _isolated(sim, u, zero, 5, ("smoke", "init_smoke"), reinit_every=4, base_level=2,
                           solid=(N_(mask), N_(bvel)), emitters=em)
    _check(dev, floor, "solid")

    rng = np.random.default_rng(9)
    dxp = 1.0
    L = tuple(r * dxp for r in res)
    u, smoke = leapfrog_init(res, 1.0 / 16, radii=(0.21, 0.28), sigma=0.06, circulation=0.2, num_samples=200)
    n = 2000
    pos = rng.uniform(0.2, 0.8, size=(n, 3)) * np.array(L)
    vel = rng.normal(size=(n, 3)) * 0.05
    rad = rng.uniform(0.005, 0.015, size=n)
    params = dict(St=6.6e-2, gravity=0.01, density_ratio=2.0 / 3, epiral_radius_ratio=35.0, Re=5.5,
                  laden_radius=0.01)
    sim = EdgeSim(res, dxp, variant="edge", reinit_every=3, base_level=2, visualize_dt=1e9)
    sim.set_velocity(*u)
    sim.set_smoke(smoke)
    sim.add_particles(T_(pos), T_(vel), T_(rad), L, **params)
    P = dict(pos=pos.astype(np.float32), vel=vel.astype(np.float32), rad=rad.astype(np.float32), num=n, L=L,
             St=params["St"], gravity=params["gravity"], density_ratio=params["density_ratio"],
             erad=params["epiral_radius_ratio"], Re=params["Re"], lrad=params["laden_radius"])
    dev, floor = _isolated(sim, u, smoke, 4, ("smoke", "pos", "vel"), particles=P, reinit_every=3, base_level=2)
    _check(dev, floor, "particles")


# ---------------------------------------------------------------------------
# the projection alone
# ---------------------------------------------------------------------------
def _div(u):
    ux, uy, uz = (np.asarray(a, np.float64) for a in u)
    return (ux[1:] - ux[:-1]) + (uy[:, 1:] - uy[:, :-1]) + (uz[:, :, 1:] - uz[:, :, :-1])


def _div_floor(u):
    """The float32 storage floor of the divergence: one rounding of each
    stored face value, summed over a cell's six faces, in the 2-norm."""
    ux, uy, uz = (np.abs(np.asarray(a, np.float64)) for a in u)
    s = (ux[1:] + ux[:-1]) + (uy[:, 1:] + uy[:, :-1]) + (uz[:, :, 1:] + uz[:, :, :-1])
    return 2.0 ** -24 * float(np.sqrt((s * s).sum()))


@pytest.mark.parametrize("amp", [1.0, 1e-4])
def test_divergence_after_projection_at_solver_tolerance(amp):
    """The divergence the projection leaves is the CG residual, whose
    recursion the solver stops below its tolerance (r.r < 1e-12 absolute,
    or 1e-12 of z.r at the start, mgpcg.py:224-254), plus one float32
    rounding of each stored face.  At amplitude 1e-4 the absolute tolerance
    binds: ||div||_2 < 1e-6."""
    from edgeb200.projection import Projection
    res = (64, 32, 32)
    rng = np.random.default_rng(3)
    u = [(amp * rng.normal(size=s)).astype(np.float32) for s in O.face_shapes(res)]
    P = Projection(res, base_level=2)
    ug = [T_(a) for a in u]
    P.poisson(*ug)
    it, rtr, st = P.result()
    assert st == 0
    uo = [a.copy() for a in u]
    O.poisson(uo, base_level=2)
    got = [N_(t) for t in ug]
    d = float(np.sqrt((_div(got) ** 2).sum()))
    d_o = float(np.sqrt((_div(uo) ** 2).sum()))
    floor = _div_floor(got)
    assert d <= np.sqrt(rtr) + 4 * floor, (d, rtr, floor)
    assert d <= 2 * d_o + 4 * floor, (d, d_o, floor)
    if amp < 1e-3:
        assert d < 1e-6 + 4 * floor, (d, floor)
