"""sim/lp.py kernels on the device against the golden vectors."""
import numpy as np
import pytest
import torch

from conftest import load_golden, rel_l2

pytestmark = pytest.mark.gpu


def T_(a):
    return torch.from_numpy(np.ascontiguousarray(a, dtype=np.float32)).cuda()


def N_(t):
    torch.cuda.synchronize()
    return t.cpu().numpy()


def test_particles_golden():
    import sim.lp as LP
    d = load_golden("particles")
    res = tuple(int(v) for v in d["res"])
    dx = float(d["meta_dx"])
    num = int(d["meta_num"])
    dt, St, grav, dens, erad, Re, lrad = (float(v) for v in d["meta_params"])
    u = [T_(d["u_" + a]) for a in "xyz"]
    vel, pos = T_(d["vel_in"]), T_(d["pos_in"])
    acc = torch.zeros_like(vel)
    vd = torch.zeros_like(vel)
    L = [r * dx for r in res]
    LP.update_particles_acc(*u, vel, pos, acc, dx, dt, num, St, grav)
    assert rel_l2(N_(acc), d["acc"]) < 1e-5
    LP.update_particles_velocity(acc, vel, pos, dt, dx, num, *L)
    assert rel_l2(N_(vel), d["vel1"]) < 1e-5
    LP.calculate_velocity_diff(*u, vel, vd, pos, dx, num, St, dens, erad)
    assert rel_l2(N_(vd)[:num], d["vel_diff"][:num]) < 1e-5
    drag = [torch.zeros_like(t) for t in u]
    LP.laden_particles_back_with_computing_particle(*drag, *u, vel, vd, pos, T_(d["rad"]), dx, num, lrad, *L, *res)
    for i, a in enumerate("xyz"):
        assert rel_l2(N_(drag[i]), d["drag_" + a]) < 1e-5
    LP.update_particles_position(vel, pos, dt, num, *L)
    assert rel_l2(N_(pos), d["pos_out"]) < 1e-6
    vis = [torch.zeros_like(t) for t in u]
    LP.calculate_viscous_force(*u, *vis, dx, Re)
    for i, a in enumerate("xyz"):
        assert rel_l2(N_(vis[i]), d["vis_" + a]) < 1e-5
