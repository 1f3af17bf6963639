"""Shared body of the run_edge.py / run_ed4.py / run_ed8.py / run_ge.py / run_efm.py drop-in drivers:
the reference's per-case configuration and its frame loop (run_edge.py:17-145,
522-746) around the device substep ``EdgeSim.step``.

Output per frame, as the reference: vtks/field_<frame>.vti (|curl u| and the
4-channel dye, written by util/io_utils.py's own VTK XML writer since
vtk/pyevtk are not installed), particle/field_<frame>.vtu for the laden
particle cases, the velocity checkpoints ckpts/vel_{x,y,z}_numpy_<frame>.npy
(run_edge.py:719-737); and also the dye (smoke_numpy_<frame>.npy, which the
reference's resume path reads at run_edge.py:565-566 but never writes) and
with --save-state the whole simulation state (mapstate_<frame>.pt) for an
exact resume in the middle of a reinitialisation interval (--from-frame).
Checkpoints follow the case's ckpt_every (run_edge.py:731).
"""
import argparse
import math
import os
import time

import numpy as np
import torch

from util.io_utils import write_to_vtks_lp, write_vtks_4channel_smoke
from util.taichi_utils import curl, get_central_vector

from .sim import EdgeSim, delta_emitters, four_vortex_init, ink_init, leapfrog_init, uniform_flow, wedge_mask

CASES = {
    # run_edge.py:25-77 (case 0 leapfrog, case 1 four vortices; the same two
    # cases in run_ed4.py, run_ed8.py, run_ge.py, run_efm.py)
    0: dict(init="leapfrog", res=(384, 128, 128), visualize_dt=0.1, reinit_every=20, cfl=0.5, total_frames=500,
            bfecc_clamp=False, ed_eps_frac=0.01, ckpt_every=1),
    1: dict(init="fourvorts", res=(128, 128, 256), visualize_dt=0.1, reinit_every=20, cfl=0.5, total_frames=500,
            bfecc_clamp=True, ed_eps_frac=0.025, ckpt_every=1),
    # run_edge.py:78-95: delta wing (solid obstacle, MGPCG_Solid_3, dye emitters)
    2: dict(init="delta", res=(256, 128, 128), visualize_dt=0.05, reinit_every=10, cfl=0.5, total_frames=120,
            bfecc_clamp=True, ed_eps_frac=0.02, only="edge", ckpt_every=1),
    # run_edge.py:96-127 / 128-159: ink circle and ink drop (two-way coupled
    # laden particles); dx = domain_range_y / res_y
    3: dict(init="inkcircle", res=(128, 256, 128), visualize_dt=10.0, reinit_every=60, cfl=0.25, total_frames=300,
            bfecc_clamp=True, ed_eps_frac=0.02, only="edge", ckpt_every=100, lp=dict(
                case=0, Re=5.5, St=6.6e-5, gravity=1.0, density_ratio=2.0 / 3, erad=35.0, num=1000000,
                laden_radius=0.01)),
    4: dict(init="inkdrop", res=(256, 512, 256), visualize_dt=10.0, reinit_every=80, cfl=0.25, total_frames=120,
            bfecc_clamp=True, ed_eps_frac=0.02, only="edge", ckpt_every=1, lp=dict(
                case=1, Re=1000.0, St=5e-5, gravity=1.0, density_ratio=0.6, erad=35.0, num=4000000,
                laden_radius=0.01)),
}
DOMAIN_Y = 256.0  # domain_range_y of the laden-particle cases


class SimpleTimer:
    """CUDA-event phase timer with the reference's names and skip rule
    (util/timer.py:4-51)."""

    def __init__(self, skip_count=5):
        self.open, self.acc, self.count, self.rec = {}, {}, {}, {}
        self.pending = []
        self.skip_count = skip_count

    def start(self, k):
        e = torch.cuda.Event(enable_timing=True)
        e.record()
        self.open[k] = e
        self.count[k] = self.count.get(k, 0) + 1

    def stop(self, k, skip_count=None):
        e = torch.cuda.Event(enable_timing=True)
        e.record()
        s = self.open.pop(k)
        if (self.skip_count if skip_count is None else skip_count) >= self.count[k]:
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
    ap.add_argument("--from-frame", type=int, default=0,
                    help="resume from this frame's checkpoint in the experiment's ckpts/ (exact with mapstate)")
    ap.add_argument("--save-state", action="store_true",
                    help="also write the whole simulation state (mapstate_<frame>.pt) with each checkpoint")
    return ap.parse_args()


def main(variant):
    args = parse(variant)
    cases = sorted(c for c, v in CASES.items() if v.get("only", variant) == variant)
    if args.case not in cases:
        raise SystemExit(f"case {args.case} is not on this driver's path (cases {cases})")
    cfg = dict(CASES[args.case])
    res = tuple(args.res) if args.res else cfg["res"]
    lp = cfg.get("lp")
    # run_edge.py:30 dx = 1/res_y; run_edge.py:101-104 dx = domain_range_y/res_y
    dx = DOMAIN_Y / res[1] if lp else 1.0 / res[1]
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

    solid = emitters = None
    if cfg["init"] == "delta":
        # set_boundary_mask_delta (init_conditions.py:139-167): the plate's
        # apex at cell (0.1 // dx, centre, 0.2 // dx), four cells thick
        apex = ((0.1 // dx) * dx, 0.5, (0.2 // dx) * dx)
        solid = wedge_mask(res, dx, apex=apex)
        emitters = delta_emitters()
    sim = EdgeSim(res, dx, variant=variant, cfl=cfg["cfl"], reinit_every=reinit,
                  ed_eps=cfg["ed_eps_frac"] * dx, base_level=args.base_level, bfecc_clamp=cfg["bfecc_clamp"],
                  visualize_dt=cfg["visualize_dt"], solid=solid, emitters=emitters)
    if lp:
        u, pos, vel, rad = ink_init(lp["case"], res, dx, lp["num"], lp["laden_radius"], DOMAIN_Y)
        smoke = torch.zeros(res + (4,), dtype=torch.float32, device="cuda")
        domain = tuple(DOMAIN_Y / res[1] * n for n in res)
        sim.add_particles(pos, vel, rad, domain, St=lp["St"], gravity=lp["gravity"],
                          density_ratio=lp["density_ratio"], epiral_radius_ratio=lp["erad"], Re=lp["Re"],
                          laden_radius=lp["laden_radius"])
    elif cfg["init"] == "delta":
        # init_delta (init_conditions.py:170-175)
        v, ang = 0.6, math.radians(20)
        u = uniform_flow(res, (v * math.cos(ang), 0.0, v * math.sin(ang)))
        smoke = torch.zeros(res + (4,), dtype=torch.float32, device="cuda")
    elif cfg["init"] == "leapfrog":
        # init_vorts_leapfrog geometry (init_conditions.py:70-86)
        rad = 0.21
        u, smoke = leapfrog_init(res, dx, radii=(rad, rad), sigma=0.08 * rad, circulation=rad * 0.1,
                                 x_start=0.16, num_samples=2000)
    else:
        u, smoke = four_vortex_init(res, dx)
    sim.set_velocity(*u)
    sim.set_smoke(smoke)
    sim.proj.poisson(*sim.u)  # run_edge.py:557
    start = args.from_frame
    if start > 0:
        state = os.path.join(ckptdir, f"mapstate_{start}.pt")
        if os.path.exists(state):
            sim.load_state_dict(torch.load(state, map_location="cuda", weights_only=False))
        else:
            # run_edge.py:559-566: velocity and dye only; the maps restart
            sim.set_velocity(*[torch.from_numpy(np.load(os.path.join(ckptdir, f"vel_{a}_numpy_{start}.npy"))).cuda()
                               for a in "xyz"])
            sim.set_smoke(torch.from_numpy(np.load(os.path.join(ckptdir, f"smoke_numpy_{start}.npy"))).cuda())
            sim.frame_idx = start

    vtkdir = os.path.join(logsdir, "vtks")
    os.makedirs(vtkdir, exist_ok=True)
    pdir = os.path.join(logsdir, "particle")
    uc = torch.empty(res + (3,), device="cuda")
    w = torch.empty(res + (3,), device="cuda")

    def save(frame):
        # run_edge.py:719-737: |curl u| and the dye as field_####.vti, the
        # particles as particle/field_###.vtu, velocity checkpoints
        get_central_vector(*sim.u, uc)
        curl(uc, w, dx)
        write_vtks_4channel_smoke(torch.linalg.vector_norm(w, dim=-1).cpu().numpy(), sim.smoke.cpu().numpy(),
                                  vtkdir, frame)
        if sim.particles is not None:
            os.makedirs(pdir, exist_ok=True)
            write_to_vtks_lp(sim.particles["pos"].cpu().numpy(), {}, {}, os.path.join(pdir, "field_{:03d}".format(frame)))
        if frame % cfg["ckpt_every"] != 0:
            return
        for c, a in enumerate("xyz"):
            np.save(os.path.join(ckptdir, f"vel_{a}_numpy_{frame}"), sim.u[c].cpu().numpy())
        # the reference's resume path reads this file (run_edge.py:565-566)
        # but never writes it
        np.save(os.path.join(ckptdir, f"smoke_numpy_{frame}"), sim.smoke.cpu().numpy())
        # the whole state, for an exact resume in the middle of an interval
        if args.save_state:
            torch.save(sim.state_dict(), os.path.join(ckptdir, f"mapstate_{frame}.pt"))

    if start <= 0:
        save(0)
    # the EFM driver skips a whole reinitialisation interval (run_efm.py:356, 404, 408)
    timer = SimpleTimer(reinit + 1 if variant == "efm" else 5)
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
