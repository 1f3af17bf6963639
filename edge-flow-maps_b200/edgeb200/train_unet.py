"""Train the learned preconditioner on the GPU from plain-MGPCG solves.

    python -m edgeb200.train_unet --res 128 64 64 --solves 1000 --out weights.npz

Training pairs are (r_k, x* - x_k): every iterate of a plain preconditioned
CG solve (flexible CG with the MGPCG V-cycle) gives its residual and the
correction still missing from it.  The right-hand sides alternate between
the divergence of a running four-vortex EDGE simulation (the configuration
the step solves) and seeded N(0,1) mean-removed fields (the evaluation
family).  Each pair is used for one Adam step of the library's own forward
and backward kernels and then discarded, so memory stays at one solve.
"""
import argparse
import math
import os
import sys
import time

import numpy as np
import torch

from .projection import Projection
from .sim import EdgeSim, four_vortex_init
from .unet import LAYERS, BIASES, LearnedCoarsePCG, LearnedPCG, UNet


def random_rhs(res, seed):
    g = torch.Generator().manual_seed(seed)
    b = torch.randn(res, generator=g)
    return (b - b.mean()).cuda()


def save_params(params, path):
    np.savez(path, **{k: v.detach().cpu().numpy() for k, v in params.items()})


def load_params(path, device="cuda"):
    d = np.load(path)
    names = [n for n, _, _ in LAYERS] + ["b" + n[1:] for n in BIASES]
    return {k: torch.from_numpy(np.ascontiguousarray(d[k])).to(device) for k in names}


def train(res=(128, 64, 64), solves=1000, lr=1e-3, seed=0, base_level=1, log=print, params=None):
    """Returns the trained parameters (float32 CUDA tensors) and the number
    of pairs used."""
    P = Projection(res, base_level=base_level)
    net = UNet(res, params=params, seed=seed)
    pcg = LearnedPCG(P, net)
    dx = 1.0 / res[1]
    sim = EdgeSim(res, dx, variant="edge", cfl=0.5, reinit_every=12, ed_eps=0.025 * dx, base_level=base_level,
                  bfecc_clamp=True, visualize_dt=0.1, packed=True)
    u, smoke = four_vortex_init(res, dx)
    sim.set_velocity(*u)
    sim.set_smoke(smoke)
    sim.proj.poisson(*sim.u)
    pairs = 0
    t0 = time.time()
    x = torch.zeros(res, device="cuda")
    for it in range(solves):
        if it % 2 == 0:
            b = random_rhs(res, 100000 + it)
        else:
            sim.step()
            b = (-sim.proj.get("div")).contiguous()
        rec = []
        pcg.solve(b, x, rel_tol=1e-7, max_iters=40, mode="vcycle", record=rec)
        for rk, xk in rec:
            if float(torch.linalg.vector_norm(rk)) == 0.0:
                continue
            loss = net.train_step(rk.contiguous(), (x - xk).contiguous(), lr=lr)
            pairs += 1
        if it % 50 == 0:
            log(f"solve {it} pairs {pairs} loss {float(loss):.4g} {time.time() - t0:.1f}s")
    if net.timed_out():
        raise RuntimeError("a tensor-core wait gave up during training")
    return net.params, pairs


def evaluate(params, sizes=((96, 96, 96), (128, 64, 64), (256, 128, 128)), seeds=(1, 2, 3), rel_tol=1e-6):
    """Iterations of flexible CG to rel_tol on seeded N(0,1) right-hand sides
    with the plain V-cycle, the V-cycle warm-started by the network, and the
    network alone."""
    out = {}
    for res in sizes:
        lg = int(math.log2(min(res)))
        P = Projection(res, base_level=max(1, lg - 5))  # 6 levels where the grid allows
        net = UNet(res, params=params)
        pcg = LearnedPCG(P, net)
        x = torch.zeros(res, device="cuda")
        row = {}
        for mode in ("vcycle", "warm", "net"):
            row[mode] = [pcg.solve(random_rhs(res, s), x, rel_tol=rel_tol, mode=mode)[0] for s in seeds]
        out["x".join(map(str, res))] = row
        P.close()
    return out


# ---- the learned coarse-grid solver (LearnedCoarsePCG) ---------------------------
def coarse_residuals(P, b, rel=1e-6, max_iters=40):
    """The level-lc residuals of every V-cycle of a plain MGPCG solve of
    A x = b (the stepwise solve with the built-in coarse group)."""
    level, dims = P.coarse_shape()
    r = torch.empty(dims, device="cuda")
    bb = float((b.double() ** 2).sum())
    out = []
    P.solve_begin(b, abs_tol=rel * rel * bb, rel_tol=0.0, max_iters=max_iters)
    while True:
        P.coarse_get_r(r)
        out.append(r.clone())
        P.coarse_default()
        P.solve_iter()
        if not P.progress()[2]:
            break
    return out


class ExactCoarse:
    """Solutions of the level-lc residual equation A_lc z = r (the same
    7-point operator with walls on the coarse grid) to 1e-7 of the
    preconditioned initial residual; the tolerance is relative, so one
    captured solve graph serves every call."""

    def __init__(self, dims):
        lg = int(math.log2(min(dims)))
        self.P = Projection(dims, base_level=max(1, lg - 2))
        self.z = torch.empty(dims, device="cuda")
        self.r = torch.empty(dims, device="cuda")

    def __call__(self, r):
        self.r.copy_(r)
        self.P.solve(self.r, self.z, abs_tol=0.0, rel_tol=1e-14, max_iters=400)
        return self.z


def _config_sims(res, base_level):
    """The two workloads whose projections give the training right-hand
    sides: the four-vortex collision (configuration 1) and the solid wedge
    in a uniform inflow (configuration 2, its divergence fields solved with
    the plain operator)."""
    from .sim import delta_emitters, uniform_flow, wedge_mask
    dx = 1.0 / res[1]
    a = EdgeSim(res, dx, variant="edge", cfl=0.5, reinit_every=12, ed_eps=0.025 * dx, base_level=base_level,
                bfecc_clamp=True, visualize_dt=1e9, packed=True)
    u, smoke = four_vortex_init(res, dx)
    a.set_velocity(*u)
    a.set_smoke(smoke)
    half = math.degrees(math.atan2(0.2, 0.3))
    mask, bvel = wedge_mask(res, dx, apex=(0.5, 0.5, 0.45), chord=0.3, half_angle_deg=half, aoa_deg=20.0,
                            thickness_cells=4, shell_vel=(1.0, 0.0, 0.0))
    c = EdgeSim(res, dx, variant="edge", cfl=0.5, reinit_every=12, ed_eps=0.025 * dx, base_level=base_level,
                bfecc_clamp=True, visualize_dt=1e9, solid=(mask, bvel),
                emitters=delta_emitters(offset=(0.5, 0.5, 0.47), half_angle_deg=half, radius=0.02), packed=True)
    c.set_velocity(*uniform_flow(res, (1.0, 0.0, 0.0)))
    return a, c


def train_coarse(sizes=((128, 64, 64), (256, 128, 128)), steps_per_source=1000, lr=1e-3, seed=0, params=None,
                 log=print):
    """Train the coarse-level network on (r_lc, exact z_lc) pairs from plain
    MGPCG solves of the projections of configurations 1 and 2 at each size.
    Returns (parameters, pairs used)."""
    pairs = 0
    net = None
    t0 = time.time()
    # The exact coarse solution is tens of times larger than its right-hand
    # side (1/lambda_min of the coarse operator); the network learns it
    # divided by a fixed gain, folded into the last layer afterwards.
    gain = None
    for res in sizes:
        P = Projection(res, base_level=2)
        level, dims = P.coarse_shape()
        if net is None or net.res != dims:
            net = UNet(dims, params=params if net is None else net.params, seed=seed)
        exact = ExactCoarse(dims)
        sims = _config_sims(res, 2)
        for k in range(steps_per_source):
            for sim in sims:
                sim.step()
                b = (-sim.proj.get("div")).contiguous()
                if float(b.abs().max()) == 0.0:
                    continue
                for r in coarse_residuals(P, b):
                    z = exact(r)
                    if gain is None:
                        gain = float(z.norm() / r.norm())
                    loss = net.train_step(r, z / gain, lr=lr)
                    pairs += 1
            if k % 100 == 0:
                log(f"{res} step {k} pairs {pairs} loss {float(loss):.4g} {time.time() - t0:.1f}s")
        params = net.params
        del sims
        P.close()
        torch.cuda.empty_cache()
    if net.timed_out():
        raise RuntimeError("a tensor-core wait gave up during training")
    params = {k: v.clone() for k, v in net.params.items()}
    params["W5"] *= gain
    params["b5"] *= gain
    log(f"output gain {gain:.4g}")
    return params, pairs


def evaluate_coarse(params, sizes=((96, 96, 96), (128, 64, 64), (256, 128, 128)), seeds=(1, 2, 3), rel_tol=1e-6,
                    precision=0, timing=True):
    """Iterations (and wall time of the stepwise loop) of MGPCG to rel_tol on
    seeded N(0,1) right-hand sides never seen in training, with the built-in
    coarse group, with the network as the coarse solver, and with the
    coarse-level equation solved exactly (the bound on what any coarse
    solver can gain)."""
    out = {}
    for res in sizes:
        lg = int(math.log2(min(res)))
        P = Projection(res, base_level=max(1, lg - 5), precision=precision)  # 6 levels where the grid allows
        L = LearnedCoarsePCG(P, params)
        x = torch.zeros(res, device="cuda")
        row = {"coarse_dims": list(L.dims)}
        for mode in ("vcycle", "net", "exact"):
            its, ms, fb = [], [], []
            for sd in seeds:
                b = random_rhs(res, sd)
                bb = float((b.double() ** 2).sum())
                L.solve(b, x, abs_tol=rel_tol * rel_tol * bb, rel_tol=0.0, mode=mode)  # warm-up / capture
                e0 = torch.cuda.Event(enable_timing=True)
                e1 = torch.cuda.Event(enable_timing=True)
                e0.record()
                it, rtr, st, fell = L.solve(b, x, abs_tol=rel_tol * rel_tol * bb, rel_tol=0.0, mode=mode)
                e1.record()
                torch.cuda.synchronize()
                its.append(it)
                ms.append(e0.elapsed_time(e1))
                fb.append(fell)
            row[mode] = {"iters": its, "ms": ms, "fell_back": fb}
        out["x".join(map(str, res))] = row
        P.close()
    return out


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--res", type=int, nargs=3, default=[128, 64, 64])
    ap.add_argument("--solves", type=int, default=1000)
    ap.add_argument("--lr", type=float, default=1e-3)
    ap.add_argument("--seed", type=int, default=0)
    ap.add_argument("--base-level", type=int, default=1)
    ap.add_argument("--init", default=None, help="start from these weights (.npz)")
    ap.add_argument("--out", default=None)
    ap.add_argument("--eval", action="store_true", help="report iterations to 1e-6 (with --init: no training)")
    ap.add_argument("--coarse", action="store_true", help="train the coarse-level network (LearnedCoarsePCG)")
    ap.add_argument("--steps-per-source", type=int, default=1000)
    a = ap.parse_args(argv)
    if a.coarse:
        params = load_params(a.init) if a.init else None
        if not (a.eval and a.out is None):
            params, pairs = train_coarse(steps_per_source=a.steps_per_source, lr=a.lr, seed=a.seed, params=params)
            save_params(params, a.out)
            print(f"saved {a.out} after {pairs} pairs")
        if a.eval:
            print(evaluate_coarse(params))
        return 0
    params = load_params(a.init) if a.init else None
    if a.eval and a.out is None:
        print(evaluate(params))
        return 0
    p, pairs = train(tuple(a.res), a.solves, a.lr, a.seed, a.base_level, params=params)
    save_params(p, a.out)
    print(f"saved {a.out} after {pairs} pairs")
    if a.eval:
        print(evaluate(p))


if __name__ == "__main__":
    sys.exit(main())
