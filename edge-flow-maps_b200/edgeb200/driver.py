"""Shared body of the run_edge.py / run_ed4.py / run_ed8.py / run_ge.py drop-in drivers:
the reference's per-case configuration and its frame loop (run_edge.py:17-145,
522-746) around the device substep ``EdgeSim.step``.

Output: instead of VTK files (util/io_utils.py, vtk/pyevtk are not installed)
each output frame writes the reference's velocity checkpoints
ckpts/vel_{x,y,z}_numpy_<frame>.npy (run_edge.py:731-737) and also the dye
(smoke_numpy_<frame>.npy, which the reference's resume path reads at
run_edge.py:565-566 but never writes) plus the map state needed for an exact
mid-interval resume (mapstate_<frame>.pt).
"""
import argparse
import os
import time

import numpy as np
import torch

from .sim import EdgeSim, four_vortex_init, leapfrog_init

CASES = {
    # run_edge.py:25-77 (case 0 leapfrog, case 1 four vortices)
    0: dict(init="leapfrog", res=(384, 128, 128), visualize_dt=0.1, reinit_every=20, cfl=0.5, total_frames=500,
            bfecc_clamp=False, ed_eps_frac=0.01),
    1: dict(init="fourvorts", res=(128, 128, 256), visualize_dt=0.1, reinit_every=20, cfl=0.5, total_frames=500,
            bfecc_clamp=True, ed_eps_frac=0.025),
}


class SimpleTimer:
    """CUDA-event phase timer with the reference's names and skip rule
    (util/timer.py:4-51)."""

    def __init__(self):
        self.open, self.acc, self.count, self.rec = {}, {}, {}, {}
        self.pending = []

    def start(self, k):
        e = torch.cuda.Event(enable_timing=True)
        e.record()
        self.open[k] = e
        self.count[k] = self.count.get(k, 0) + 1

    def stop(self, k, skip_count=5):
        e = torch.cuda.Event(enable_timing=True)
        e.record()
        s = self.open.pop(k)
        if skip_count >= self.count[k]:
            return
        self.pending.append((k, s, e))

    def print_times(self, log=print):
        torch.cuda.synchronize()
        for k, s, e in self.pending:
            self.acc[k] = self.acc.get(k, 0.0) + s.elapsed_time(e) / 1000.0
            self.rec[k] = self.rec.get(k, 0) + 1
        self.pending = []
        for k, t in self.acc.items():
            c = self.rec[k]
            log(f"'{k}' execution time: {t:.8f} seconds, average: {t / c:.8f} seconds, count: {c}")


def parse(variant):
    ap = argparse.ArgumentParser()
    ap.add_argument("-n", "--name", help="Experiment name")
    ap.add_argument("-c", "--case", type=int, default=0, help="Demo case number")
    ap.add_argument("--res", type=int, nargs=3, default=None, help="override the case's grid")
    ap.add_argument("--frames", type=int, default=None, help="override total_frames")
    ap.add_argument("--max-steps", type=int, default=None, help="stop after this many substeps")
    ap.add_argument("--reinit", type=int, default=None)
    ap.add_argument("--base-level", type=int, default=3)
    ap.add_argument("--logdir", default="logs")
    return ap.parse_args()


def main(variant):
    args = parse(variant)
    if args.case not in CASES:
        raise SystemExit(f"case {args.case} is not on this driver's path (cases {sorted(CASES)})")
    cfg = dict(CASES[args.case])
    res = tuple(args.res) if args.res else cfg["res"]
    dx = 1.0 / res[1]  # run_edge.py:30 dx = 1/res_y
    reinit = args.reinit or cfg["reinit_every"]
    exp = args.name or f"{cfg['init']}-{variant}-" + time.strftime("%Y-%m-%d-%H-%M-%S")
    logsdir = os.path.join(args.logdir, exp)
    ckptdir = os.path.join(logsdir, "ckpts")
    os.makedirs(ckptdir, exist_ok=True)
    logf = open(os.path.join(logsdir, "log.txt"), "a")

    def log(msg):
        print(msg)
        logf.write(msg + "\n")
        logf.flush()

    sim = EdgeSim(res, dx, variant=variant, cfl=cfg["cfl"], reinit_every=reinit,
                  ed_eps=cfg["ed_eps_frac"] * dx, base_level=args.base_level, bfecc_clamp=cfg["bfecc_clamp"],
                  visualize_dt=cfg["visualize_dt"])
    if cfg["init"] == "leapfrog":
        # init_vorts_leapfrog geometry (init_conditions.py:70-86)
        rad = 0.21
        u, smoke = leapfrog_init(res, dx, radii=(rad, rad), sigma=0.08 * rad, circulation=rad * 0.1,
                                 x_start=0.16, num_samples=2000)
    else:
        u, smoke = four_vortex_init(res, dx)
    sim.set_velocity(*u)
    sim.set_smoke(smoke)
    sim.proj.poisson(*sim.u)  # run_edge.py:557

    def save(frame):
        for c, a in enumerate("xyz"):
            np.save(os.path.join(ckptdir, f"vel_{a}_numpy_{frame}"), sim.u[c].cpu().numpy())
        np.save(os.path.join(ckptdir, f"smoke_numpy_{frame}"), sim.smoke.cpu().numpy())

    save(0)
    timer = SimpleTimer()
    total_frames = args.frames or cfg["total_frames"]
    t0 = time.time()
    last = 0
    i = 0
    while True:
        frame_before = sim.frame_idx
        sim.step(timers=timer)
        j = i % reinit
        relstep = int(sim.visualize_dt / sim.last_dt) if sim.last_dt > 0 else 0
        log(f"[Simulate] Done step {i} substep {j} relstep 1/{relstep}")
        if sim.frame_idx != frame_before:
            save(sim.frame_idx)
            torch.cuda.synchronize()
            log(f"[Simulate] Done Frame {sim.frame_idx} substep {i - last} time {time.time() - t0:.2f}s\n")
            last = i
            if sim.frame_idx >= total_frames:
                break
        i += 1
        if args.max_steps and i >= args.max_steps:
            break
    timer.print_times(log)
    log("[Main] Complete")
