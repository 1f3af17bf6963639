"""Whole substeps of the device driver (edgeb200.sim.EdgeSim) against the
golden two-step run of the reference driver loop and the oracle's substep."""
import numpy as np
import pytest
import torch

from conftest import load_golden, rel_l2
from oracle import edge_oracle as O

pytestmark = pytest.mark.gpu


def T_(a):
    return torch.from_numpy(np.ascontiguousarray(a, dtype=np.float32)).cuda()


def N_(t):
    torch.cuda.synchronize()
    return t.cpu().numpy()


def test_edge_steps_golden():
    from edgeb200.sim import EdgeSim
    d = load_golden("edge_steps")
    res = tuple(int(v) for v in d["res"])
    sim = EdgeSim(res, float(d["meta_dx"]), variant="edge", cfl=float(d["meta_cfl"]),
                  reinit_every=int(d["meta_reinit"]), ed_eps=float(d["meta_eps"]), base_level=1, visualize_dt=1e9)
    sim.set_velocity(*[T_(d["u_in_" + a]) for a in "xyz"])
    sim.set_smoke(T_(d["smoke_in"]))
    for i in range(2):
        dt = sim.step()
        assert dt == pytest.approx(float(d[f"s{i}_meta_dt"]), rel=1e-5)
        for c, a in enumerate("xyz"):
            assert rel_l2(N_(sim.u[c]), d[f"s{i}_u_{a}"]) < 2e-4, (i, a)
            assert rel_l2(N_(sim.phi[c]), d[f"s{i}_phi_{a}"]) < 1e-5
            assert rel_l2(N_(sim.map["T"][c]), d[f"s{i}_T_{a}"]) < 1e-5
        assert rel_l2(N_(sim.map["psi"]), d[f"s{i}_psi"]) < 1e-6
        assert rel_l2(N_(sim.smoke), d[f"s{i}_smoke"]) < 2e-4


@pytest.mark.parametrize("packed", [False, True])
@pytest.mark.parametrize("variant", ["edge", "ed4", "ed8", "ge", "efm"])
def test_steps_vs_oracle(variant, packed):
    from edgeb200.sim import EdgeSim, leapfrog_init
    res = (32, 16, 16)
    dx = 1.0 / 16
    u, smoke = leapfrog_init(res, dx, radii=(0.21, 0.28), sigma=0.06, circulation=0.2, num_samples=200)
    st = O.EdgeState(res, dx, [N_(t) for t in u], N_(smoke))
    sim = EdgeSim(res, dx, variant=variant, reinit_every=3, base_level=2, visualize_dt=1e9, packed=packed)
    sim.set_velocity(*u)
    sim.set_smoke(smoke)
    for i in range(4):
        dt = sim.step()
        dto, _ = O.edge_substep(st, reinit_every=3, base_level=2, dt=dt, variant=variant)
        for c in range(3):
            assert rel_l2(N_(sim.u[c]), st.u[c]) < 5e-4, (variant, i, c)
        assert rel_l2(N_(sim.smoke), st.smoke) < 5e-4, (variant, i)
        if variant == "efm":
            for c in range(3):  # the backtracked face map
                assert rel_l2(N_(sim.fpsi[c]), O.efm_backtrack(
                    [st.u_cache[s] for s in range(i % 3 + 1)], [st.dts[s] for s in range(i % 3 + 1)], dx)[0][c]) < 1e-5
        else:
            assert rel_l2(N_(sim.map["psi"]), st.psi) < 1e-5


def test_solid_emitter_steps_vs_oracle():
    """The solid-obstacle (MGPCG_Solid_3) and dye-emitter path of the delta
    case (run_edge.py:643-648, 704-710) against the oracle's substep."""
    from edgeb200.sim import EdgeSim, delta_emitters, uniform_flow, wedge_mask
    res = (32, 16, 16)
    dx = 1.0 / 16
    mask, bvel = wedge_mask(res, dx, apex=(0.35, 0.5, 0.4), chord=0.6, thickness_cells=2)
    u = uniform_flow(res, (0.6 * 0.94, 0.0, 0.6 * 0.34))
    em = delta_emitters(offset=(0.3, 0.5, 0.45), radius=0.1)
    sim = EdgeSim(res, dx, variant="edge", reinit_every=4, base_level=2, visualize_dt=1e9, solid=(mask, bvel),
                  emitters=em)
    sim.set_velocity(*u)
    st = O.EdgeState(res, dx, [N_(t) for t in u], np.zeros(res + (4,), np.float32))
    m_h, b_h = N_(mask), N_(bvel)
    for i in range(3):
        dt = sim.step()
        O.edge_substep(st, reinit_every=4, base_level=2, dt=dt, solid=(m_h, b_h), emitters=em)
        for c in range(3):
            assert rel_l2(N_(sim.u[c]), st.u[c]) < 1e-3, (i, c)
        assert rel_l2(N_(sim.init_smoke), st.init_smoke) < 1e-4, i
        assert rel_l2(N_(sim.smoke), st.smoke) < 1e-3, i
        assert sim.proj.result()[2] == 0


def test_particle_coupled_steps_vs_oracle():
    """Two-way laden-particle coupling (run_edge.py:627-667, 704-708)."""
    from edgeb200.sim import EdgeSim, leapfrog_init
    rng = np.random.default_rng(9)
    res = (32, 16, 16)
    dx = 1.0
    L = tuple(r * dx for r in res)
    u, smoke = leapfrog_init(res, 1.0 / 16, radii=(0.21, 0.28), sigma=0.06, circulation=0.2, num_samples=200)
    n = 2000
    pos = rng.uniform(0.2, 0.8, size=(n, 3)) * np.array(L)
    vel = rng.normal(size=(n, 3)) * 0.05
    rad = rng.uniform(0.005, 0.015, size=n)
    params = dict(St=6.6e-2, gravity=0.01, density_ratio=2.0 / 3, epiral_radius_ratio=35.0, Re=5.5,
                  laden_radius=0.01)
    sim = EdgeSim(res, dx, variant="edge", reinit_every=3, base_level=2, visualize_dt=1e9)
    sim.set_velocity(*u)
    sim.set_smoke(smoke)
    sim.add_particles(T_(pos), T_(vel), T_(rad), L, **params)
    P = dict(pos=pos.astype(np.float32), vel=vel.astype(np.float32), rad=rad.astype(np.float32), num=n, L=L,
             St=params["St"], gravity=params["gravity"], density_ratio=params["density_ratio"],
             erad=params["epiral_radius_ratio"], Re=params["Re"], lrad=params["laden_radius"])
    st = O.EdgeState(res, dx, [N_(t) for t in u], N_(smoke))
    for i in range(3):
        dt = sim.step()
        O.edge_substep(st, reinit_every=3, base_level=2, dt=dt, particles=P)
        assert rel_l2(N_(sim.particles["pos"]), P["pos"]) < 1e-5, i
        assert rel_l2(N_(sim.particles["vel"]), P["vel"]) < 1e-4, i
        for c in range(3):
            assert rel_l2(N_(sim.u[c]), st.u[c]) < 1e-3, (i, c)
            assert rel_l2(N_(sim.particles["vis"][c]), P["vis"][c]) < 1e-3, (i, c)


@pytest.mark.parametrize("variant,packed", [("edge", True), ("ed8", False), ("efm", False)])
def test_state_dict_resume_is_exact(variant, packed):
    """Saving the state in the middle of a reinitialisation interval and
    loading it into a fresh simulation continues bit for bit."""
    from edgeb200.sim import EdgeSim, leapfrog_init
    res = (32, 16, 16)
    dx = 1.0 / 16
    u, smoke = leapfrog_init(res, dx, radii=(0.21, 0.28), sigma=0.06, circulation=0.2, num_samples=200)

    def make():
        s = EdgeSim(res, dx, variant=variant, reinit_every=4, base_level=2, visualize_dt=0.05, packed=packed)
        s.set_velocity(*u)
        s.set_smoke(smoke)
        return s

    a = make()
    for _ in range(2):
        a.step()
    state = a.state_dict()
    for _ in range(3):
        a.step()
    b = make()
    b.load_state_dict(state)
    for _ in range(3):
        b.step()
    for c in range(3):
        assert torch.equal(a.u[c], b.u[c])
    assert torch.equal(a.smoke, b.smoke)
    assert (a.i, a.frame_idx, a.sub_t) == (b.i, b.frame_idx, b.sub_t)


@pytest.mark.parametrize("variant", ["edge", "ed8"])
def test_step_host_matches_device_steps(variant):
    """step_host (state round-tripping through pinned host buffers, copies
    overlapped with the step) gives the device-resident steps' results, also
    across a reinitialisation."""
    from edgeb200.sim import EdgeSim, leapfrog_init
    res = (32, 16, 16)
    dx = 1.0 / 16
    u, smoke = leapfrog_init(res, dx, radii=(0.21, 0.28), sigma=0.06, circulation=0.2, num_samples=200)
    a = EdgeSim(res, dx, variant=variant, reinit_every=3, base_level=2, visualize_dt=1e9)
    b = EdgeSim(res, dx, variant=variant, reinit_every=3, base_level=2, visualize_dt=1e9)
    for s in (a, b):
        s.set_velocity(*u)
        s.set_smoke(smoke)
    hu = [torch.empty(t.shape, pin_memory=True) for t in u]
    hs = torch.empty(smoke.shape, pin_memory=True)
    for h, d in zip(hu, u):
        h.copy_(d)
    hs.copy_(smoke)
    for _ in range(5):
        a.step()
        b.step_host(hu, hs)
    torch.cuda.synchronize()
    for c in range(3):
        assert torch.equal(a.u[c].cpu(), hu[c])
    assert torch.equal(a.smoke.cpu(), hs)


def test_random_potential_init_is_seeded_and_scaled():
    """The 512x256x256 workload's initial velocity (curl of a seeded random
    vector potential), on a small grid: deterministic per seed, scaled to
    max |u_cell| = 1, and nearly divergence-free (the clamped central curl)."""
    from edgeb200.sim import random_potential_init
    res, dx = (32, 16, 16), 1.0 / 16
    a = random_potential_init(res, dx, seed=3)
    b = random_potential_init(res, dx, seed=3)
    c = random_potential_init(res, dx, seed=4)
    for x, y in zip(a, b):
        assert torch.equal(x, y)
    assert any(not torch.equal(x, y) for x, y in zip(a, c))
    ux, uy, uz = (N_(t).astype(np.float64) for t in a)
    assert np.isfinite(ux).all() and np.abs(ux).max() <= 1.0 + 1e-6
    div = (ux[1:] - ux[:-1]) + (uy[:, 1:] - uy[:, :-1]) + (uz[:, :, 1:] - uz[:, :, :-1])
    mag = np.abs(ux[1:]) + np.abs(uy[:, 1:]) + np.abs(uz[:, :, 1:])
    assert np.sqrt((div[1:-1, 1:-1, 1:-1] ** 2).mean()) < 0.5 * np.sqrt((mag ** 2).mean())


@pytest.mark.parametrize("precision", [1, 2])
def test_mixed_precision_steps_track_fp32(precision):
    """EdgeSim(precision=1/2): BF16/FP16 V-cycle storage and the float64
    Jacobian composition; the steps stay within the solver tolerance's reach
    of the float32 steps and every projection converges."""
    from edgeb200.sim import EdgeSim, leapfrog_init
    res, dx = (64, 32, 32), 1.0 / 32
    u, smoke = leapfrog_init(res, dx, radii=(0.21, 0.28), sigma=0.03, circulation=1.0)
    sims = [EdgeSim(res, dx, variant="edge", reinit_every=12, base_level=2, visualize_dt=1e9, precision=p)
            for p in (0, precision)]
    for s in sims:
        s.set_velocity(*u)
        s.set_smoke(smoke)
    for i in range(6):
        dts = [s.step() for s in sims]
        assert dts[0] == pytest.approx(dts[1], rel=1e-3)
        assert sims[1].proj.result()[2] == 0
        for c in range(3):
            assert rel_l2(N_(sims[1].u[c]), N_(sims[0].u[c])) < 2e-3, (i, c)
