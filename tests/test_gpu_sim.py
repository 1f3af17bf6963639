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


@pytest.mark.parametrize("variant", ["edge", "ed4", "ed8"])
def test_steps_vs_oracle(variant):
    from edgeb200.sim import EdgeSim, leapfrog_init
    res = (32, 16, 16)
    dx = 1.0 / 16
    u, smoke = leapfrog_init(res, dx, radii=(0.21, 0.28), sigma=0.06, circulation=0.2, num_samples=200)
    st = O.EdgeState(res, dx, [N_(t) for t in u], N_(smoke))
    sim = EdgeSim(res, dx, variant=variant, reinit_every=3, base_level=2, visualize_dt=1e9)
    sim.set_velocity(*u)
    sim.set_smoke(smoke)
    for i in range(4):
        dt = sim.step()
        dto, _ = O.edge_substep(st, reinit_every=3, base_level=2, dt=dt, variant=variant)
        for c in range(3):
            assert rel_l2(N_(sim.u[c]), st.u[c]) < 5e-4, (variant, i, c)
        assert rel_l2(N_(sim.smoke), st.smoke) < 5e-4, (variant, i)
        assert rel_l2(N_(sim.map["psi"]), st.psi) < 1e-5
