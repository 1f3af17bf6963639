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
from .unet import LAYERS, BIASES, LearnedPCG, UNet


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
    a = ap.parse_args(argv)
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
