#!/usr/bin/env python
"""EDGE steps/s at 256x128x128 on B200 (four-vortex collision, EDGE variant).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

A step is one substep of the EDGE driver loop (run_edge.py:588-712): CFL dt,
map reinitialisation every 12 steps, semi-Lagrangian midpoint advection,
MGPCG projection, EDGE flow-map march, forward-map march, BFECC pullback of
velocity and dye with clamps, second projection.  Workload: 256x128x128 MAC
grid (dx = 1/128), four vortex rings of init_four_vorts rotated to travel
along x, CFL 0.5, epsilon 0.025 dx, 6-level MGPCG (base_level 2) to the
reference tolerance (r.r < 1e-12 or 1e-12 z0.r0), BFECC clamp on.  Synthetic
seeded input (no dataset); the step's working set (~1.7 GB) exceeds L2, so L2
is not warm between timed steps.

Multi-GPU: the solver does not shard (one grid per GPU); N ranks run N
independent replicas, value = N x K / max-over-ranks time ("scaling": "weak").

--impl reference times the reference's CPU restatement (the oracle, OpenMP on
all host cores) on the same workload, rank 0 only, a bounded number of steps.
"""
import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
PKG = os.path.join(ROOT, "edge-flow-maps_b200")
for _p in (PKG, ROOT):
    if _p not in sys.path:
        sys.path.insert(0, _p)

RES = (256, 128, 128)
DX = 1.0 / 128
CFL = 0.5
REINIT = 12
BASE_LEVEL = 2
EPS_FRAC = 0.025
METRIC = "EDGE steps/s at 256x128x128"
UNIT = "steps/s"

# algorithmic work per unit (cells Nc, faces Nf; float32)
NC = RES[0] * RES[1] * RES[2]
NF = (RES[0] + 1) * RES[1] * RES[2] + RES[0] * (RES[1] + 1) * RES[2] + RES[0] * RES[1] * (RES[2] + 1)
# MGPCG: per CG iteration 117 B per fine cell; set-up 100 B per cell plus
# divergence / gradient update 36 B per face
MG_ITER_BYTES = 117 * NC
MG_SETUP_BYTES = 100 * NC + 36 * NF


def peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.gpu = str(gpu_index)
        self.proc = None
        self.lines = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", self.gpu, f"--query-gpu={self.FIELDS}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            p = [x.strip() for x in ln.split(",")]
            if len(p) < 9:
                continue
            try:
                sm.append(float(p[1]))
                mx.append(float(p[2]))
            except ValueError:
                continue
            for nm, v in zip(names, p[5:9]):
                if v.lower() == "active":
                    reasons.add(nm)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": max(mx), "reasons": sorted(reasons),
                "samples": len(sm)}


def max_over_ranks(value, world, device):
    """Max of a per-rank float over all ranks (the job's time is its slowest
    rank's)."""
    import torch
    import torch.distributed as dist
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    if world > 1:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t[0])


def replica_throughput(world, steps, ms_max):
    """Whole-job steps/s of `world` independent replicas, each timing `steps`
    steps, bounded by the slowest rank."""
    return world * steps * 1000.0 / ms_max


def make_sim(variant="edge", res=None, packed=False):
    from edgeb200.sim import EdgeSim, four_vortex_init
    res = tuple(res) if res else RES
    dx = 1.0 / res[1]
    base = BASE_LEVEL - (int(math.log2(RES[1])) - int(math.log2(res[1])))  # keep the coarsest level's size
    sim = EdgeSim(res, dx, variant=variant, cfl=CFL, reinit_every=REINIT, ed_eps=EPS_FRAC * dx,
                  base_level=max(base, 1), bfecc_clamp=True, visualize_dt=0.1, packed=packed)
    u, smoke = four_vortex_init(res, dx)
    sim.set_velocity(*u)
    sim.set_smoke(smoke)
    sim.proj.poisson(*sim.u)  # run_edge.py:557 projection of the initial field
    return sim


class EventTimers:
    """CUDA-event phase timers with the reference SimpleTimer's names."""

    def __init__(self):
        import torch
        self.torch = torch
        self.open = {}
        self.done = []

    def start(self, k):
        e = self.torch.cuda.Event(enable_timing=True)
        e.record()
        self.open[k] = e

    def stop(self, k, skip=0):
        e = self.torch.cuda.Event(enable_timing=True)
        e.record()
        self.done.append((k, self.open.pop(k), e))

    def totals(self):
        self.torch.cuda.synchronize()
        out = {}
        for k, a, b in self.done:
            out[k] = out.get(k, 0.0) + a.elapsed_time(b)
        return out


def instrumented_step(sim):
    """One step with CUDA events around every kernel family (outside the timed
    region).  Returns {stage: ms} and the two solves' iteration counts."""
    import torch

    from edgeb200 import ops
    evs = []

    def mark(name):
        e = torch.cuda.Event(enable_timing=True)
        e.record()
        evs.append((name, e))

    dx = sim.dx
    sim.i += 1
    j = sim.i % sim.reinit_every
    dt = sim.next_dt()
    if j == 0:
        ops.reset_faces(sim.res, dx, sim.phi, sim.F)
        for a, b in zip(sim.init_u, sim.u):
            ops.copy(b, a)
        ops.copy(sim.smoke, sim.init_smoke)
    mark("start")
    ops.advect_u_sl(sim.u, dx, 0.5 * dt, sim.tmp_u)
    sim.u, sim.tmp_u = sim.tmp_u, sim.u
    mark("advect_u_semi_lagrangian")
    sim.proj.poisson(*sim.u)
    mark("mgpcg_solve_1")
    it1 = sim.proj.result()[0]
    mark("_sync1")
    sim._march(dt, j == 0, j)
    mark("march_edge")
    ops.advance_map(sim.u, dx, dt, sim.phi, sim.F)
    mark("advance_map")
    if sim.variant == "efm":
        pass  # the backtrack (march_edge stage) wrote the face map
    elif sim.packed:
        ops.face_map_packed(sim.hv, dx, sim.pmaps[sim.cur], sim.res, sim.fpsi, sim.fcol)
    else:
        m = sim.map
        ops.face_map(sim.hv, dx, m["psi"], m["T"], m.get("dT"), m.get("d2T"), sim.fpsi, sim.fcol)
    mark("face_map")
    ops.pullback_u(sim.init_u, dx, sim.fpsi, sim.fcol, sim.u)
    ops.pullback_u(sim.u, dx, sim.phi, sim.F, sim.err_u, init=sim.init_u, scale=0.5)
    ops.pullback_u(sim.err_u, dx, sim.fpsi, sim.fcol, sim.tmp_u, sub=sim.u)
    mark("pullback_u")
    ops.pullback_dye(sim.init_smoke, dx, sim.fpsi, sim.smoke)
    ops.pullback_dye(sim.smoke, dx, sim.phi, sim.err_smoke, init=sim.init_smoke, scale=0.5)
    ops.pullback_dye(sim.err_smoke, dx, sim.fpsi, sim.smoke, sub=sim.smoke, clampsrc=sim.init_smoke)
    mark("pullback_dye")
    ops.clamp_u(sim.tmp_u, sim.u, sim.tmp_u)
    sim.u, sim.tmp_u = sim.tmp_u, sim.u
    mark("clamp_u")
    sim.proj.poisson(*sim.u)
    mark("mgpcg_solve_2")
    torch.cuda.synchronize()
    it2 = sim.proj.result()[0]
    out = {}
    for (a, ea), (b, eb) in zip(evs[:-1], evs[1:]):
        if b.startswith("_") or a.startswith("_") and b != "march_edge":
            continue
        name = b
        if a == "_sync1":
            name = "march_edge"
        out[name] = out.get(name, 0.0) + ea.elapsed_time(eb)
    return out, (it1, it2)


def cpu_reference_steps(k, warm):
    """The oracle substep on the host cores; returns (seconds per step, cores,
    steps timed)."""
    import numpy as np

    from oracle import edge_oracle as O
    cores = os.cpu_count() or 1
    os.environ.setdefault("OMP_NUM_THREADS", str(cores))
    u_c = np.zeros(RES + (3,), np.float32)
    smoke = np.zeros(RES + (4,), np.float32)
    tmp = np.zeros(RES + (4,), np.float32)
    # init_four_vorts geometry with the long axis along x (see edgeb200.sim.four_vortex_init)
    c45 = math.cos(math.pi / 4)
    mid = RES[0] * DX / 2
    perm = lambda v: [v[2], v[1], v[0]]  # noqa: E731
    rings = [(2.e-2, (0.34, 0.34, mid), (-c45, c45, 0.), (1, 0, 0)), (-2.e-2, (0.66, 0.34, mid), (c45, c45, 0.), (0, 1, 0)),
             (2.e-2, (0.34, 0.66, mid), (c45, c45, 0.), (0, 0, 1)), (-2.e-2, (0.66, 0.66, mid), (-c45, c45, 0.), (0, 0, 0))]
    for q, (w, c, ex, col) in enumerate(rings):
        n = math.sqrt(sum(v * v for v in ex))
        ex = [v / n for v in ex]
        tgt = smoke if q == 0 else tmp
        if q:
            tmp[...] = 0
        O.add_vortex_ring(RES, DX, w, 0.15, 0.024, perm(c), perm(ex), perm((0., 0., 1.)), u_c, tgt, col, 500)
        if q:
            smoke += tmp
    u = O.split_central_vector(u_c)
    O.poisson(u, BASE_LEVEL)
    st = O.EdgeState(RES, DX, u, smoke)
    for _ in range(warm):
        O.edge_substep(st, cfl=CFL, reinit_every=REINIT, ed_eps=EPS_FRAC * DX, base_level=BASE_LEVEL)
    t0 = time.perf_counter()
    for _ in range(k):
        O.edge_substep(st, cfl=CFL, reinit_every=REINIT, ed_eps=EPS_FRAC * DX, base_level=BASE_LEVEL)
    return (time.perf_counter() - t0) / k, int(os.environ.get("OMP_NUM_THREADS", cores)), k


def run_reference(args, rank, world):
    if rank != 0:
        return 0
    k = max(1, min(args.steps, args.ref_max_steps))
    warm = min(args.warmup, 1)
    sec, cores, k = cpu_reference_steps(k, warm)
    v = 1.0 / sec
    line = {
        "impl": "reference", "metric": METRIC, "value": v, "unit": UNIT, "n_gpus": args.gpus, "steps": k,
        "warmup": warm, "ms_per_step": 1000 * sec, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded four-vortex rings)",
        "config": {"workload": "four-vortex collision 256x128x128, EDGE, CFL 0.5, reinit 12, 6-level MGPCG",
                   "res": list(RES)},
        "cpu_baseline": {"value": v, "unit": UNIT, "cores": cores, "kind": "port",
                         "sample": f"{k} full substep(s) of the same workload after {warm} warm-up, "
                                   f"C/OpenMP restatement of the reference kernels (Taichi is not installable)"},
        "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


# "PCG time to 1e-6": the plain MGPCG solve of A x = b (6 levels, all walls)
# for a seeded N(0,1) mean-removed right-hand side, run until the CG residual
# satisfies ||r|| <= 1e-6 ||b|| (r.r <= 1e-12 b.b)
PCG_REL = 1e-6
# DRAM bytes (dram__bytes_read.sum + dram__bytes_write.sum) summed over the
# launches of that solve (4 CG iterations), one ncu capture of
# `bench.py --pcg-only` with the host-driven solver loop (EDGE_MGPCG_EAGER=1);
# ncu flushes the caches before every launch, so this is the cold-L2 figure
PCG_TRAFFIC = 1379416320


def _event_ms(fn, reps):
    import torch
    times = []
    for _ in range(reps):
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record()
        fn()
        e1.record()
        torch.cuda.synchronize()
        times.append(e0.elapsed_time(e1))
    return statistics.median(times)


def _solve_stats(res, b, bb, tol, precision, reps, ref):
    """One Projection solving A x = b to r.r <= tol (graph-captured solve):
    median CUDA-event time, iterations, the recursion's and the true relative
    residual, and the error against the FP64 solve `ref`."""
    import torch
    from edgeb200.precision import rel_error
    from edgeb200.projection import Projection
    P = Projection(res, base_level=BASE_LEVEL, precision=precision)
    x = torch.zeros(res, device="cuda")
    P.solve(b, x, abs_tol=tol, rel_tol=0.0)  # captures the solve graph
    torch.cuda.synchronize()
    ms = _event_ms(lambda: P.solve(b, x, abs_tol=tol, rel_tol=0.0), reps)
    it, rtr, st = P.result()
    Ax = torch.empty_like(x)
    P.apply_A(x, Ax)
    true_rel = float((Ax.double() - b.double()).norm() / b.double().norm())
    out = {"ms": ms, "iters": it, "status": st, "rel_residual": math.sqrt(rtr / bb), "true_rel_residual": true_rel,
           "fp64_rel_error": rel_error(x, ref) if ref is not None else None}
    return out, P


def _refined_stats(P, b, reps, ref, inner_rel):
    """Iterative refinement around P (float64 residual and iterate) to a
    TRUE relative residual of 1e-6."""
    from edgeb200.precision import RefinedSolver, rel_error
    R = RefinedSolver(P, inner_rel=inner_rel)
    b64 = b.double()
    R.solve(b64, rel_tol=PCG_REL)
    ms = _event_ms(lambda: R.solve(b64, rel_tol=PCG_REL), reps)
    x = R.solve(b64, rel_tol=PCG_REL)
    return {"ms": ms, "outer": R.stats["outer"], "inner_iters": R.stats["inner_iters"],
            "true_rel_residual": R.stats["true_rel_residual"], "inner_rel": inner_rel,
            "fp64_rel_error": rel_error(x.float(), ref) if ref is not None else None}


def pcg_measure(res, reps=5, variants=True):
    """Pressure solve to 1e-6 relative residual on a seeded N(0,1)
    mean-removed right-hand side: the plain float32 solver (the roofline
    line),
    the BF16 and FP16 mixed-precision solvers, and iterative refinement that
    brings the TRUE residual to 1e-6 (float64 residual and iterate around
    float32 or FP16 inner solves); errors against an FP64 solve."""
    import torch
    from edgeb200.precision import fp64_solve, rel_error
    g = torch.Generator().manual_seed(1)
    b = torch.randn(res, generator=g, dtype=torch.float64)
    b -= b.mean()
    bb = float((b * b).sum())
    b = b.float().cuda()
    tol = PCG_REL * PCG_REL * bb
    nc = res[0] * res[1] * res[2]
    out, P = _solve_stats(res, b, bb, tol, 0, reps, None)
    ref = fp64_solve(P, b)
    x = torch.zeros(res, device="cuda")
    P.solve(b, x, abs_tol=tol, rel_tol=0.0)
    out["fp64_rel_error"] = rel_error(x, ref)
    it = out["iters"]
    # set-up + one preconditioned iteration each (+1: the set-up V-cycle)
    out["algorithmic_bytes"] = 100 * nc + (it + 1) * 117 * nc
    out["res"] = list(res)
    out["rhs"] = "N(0,1) seed 1, mean removed"
    if not variants:
        P.close()
        return out
    out["refined"] = {"fp32": _refined_stats(P, b, reps, ref, 1e-2)}
    P.close()
    out["mixed"] = {}
    for name, prec in (("bf16", 1), ("fp16", 2)):
        m, Pm = _solve_stats(res, b, bb, tol, prec, reps, ref)
        m["speedup_vs_fp32"] = out["ms"] / m["ms"]
        m["refined"] = _refined_stats(Pm, b, reps, ref, 1e-2)
        Pm.close()
        out["mixed"][name] = m
    return out


# FLOPs per cell of the marches, counted from the reference's arithmetic
# (EDGE: 5 trajectories x (RK4 with Jacobian + Hermite value/gradient); GE: one
# trajectory with Jacobian, 3 full Hermite value/gradient, 3x3 compose and the
# grid differences of calc_fd_3_from_grad)
MARCH_FLOP_PER_CELL = {"edge": 27400, "ed4": 8400, "ed8": 16800, "ge": 5500}


# EFM: RK4 of the face map with its Jacobian column through each cached field
EFM_FLOP_PER_FACE_STEP = 3000


def march_roofline(stages, variant, peak_tflops, ncells, flop_per_cell=None):
    ms = stages.get("march_edge", 0.0)
    if ms <= 0 or not peak_tflops:
        return None
    fpc = MARCH_FLOP_PER_CELL[variant] if flop_per_cell is None else flop_per_cell
    ach = fpc * ncells / (ms * 1e-3) / 1e12
    kernel = "k_backtrack_faces" if variant == "efm" else f"k_march_{variant}_p"
    return {"kernel": kernel, "bound": "fp32", "achieved": ach, "peak": peak_tflops,
            "unit": "TFLOP/s", "frac": ach / peak_tflops, "flop_per_cell": round(fpc, 1),
            "peak_source": "measured here (edge_fma_peak, FP32 FMA chains)"}


COARSE_WEIGHTS = os.path.join(PKG, "edgeb200", "weights", "unet_coarse.npz")
WEIGHTS = os.path.join(PKG, "edgeb200", "weights", "unet_pcg.npz")


def learned_measure(res, reps=3):
    """The learned coarse-grid solver (LearnedCoarsePCG: the U-Net as the
    V-cycle's coarse group, everything else the plain solver's kernels) on
    the plain solve's right-hand side, to the same 1e-6: float32 and FP16
    V-cycle storage (learned + mixed), next to the same stepwise loop with
    the built-in coarse group; CUDA-event time of the whole solve (graph
    replays of one iteration, the host reading the status between them).
    Plus the iteration counts on held-out right-hand sides at 96^3,
    128x64x64 and 256x128x128."""
    import torch
    from edgeb200.projection import Projection
    from edgeb200.train_unet import evaluate_coarse, load_params
    from edgeb200.unet import LearnedCoarsePCG
    if not os.path.exists(COARSE_WEIGHTS):
        return None
    params = load_params(COARSE_WEIGHTS)
    g = torch.Generator().manual_seed(1)
    b = torch.randn(res, generator=g, dtype=torch.float64)
    b -= b.mean()
    bb = float((b * b).sum())
    b = b.float().cuda()
    tol = PCG_REL * PCG_REL * bb
    x = torch.zeros(res, device="cuda")
    out = {}
    for prec in (0, 2):
        P = Projection(res, base_level=BASE_LEVEL, precision=prec)
        L = LearnedCoarsePCG(P, params)
        row = {"coarse_dims": list(L.dims)}
        for mode in ("vcycle", "net"):
            L.solve(b, x, abs_tol=tol, rel_tol=0.0, mode=mode)
            res_ = []
            ms = _event_ms(lambda: res_.append(L.solve(b, x, abs_tol=tol, rel_tol=0.0, mode=mode)), reps)
            it, rtr, st, fell = res_[-1]
            row[mode] = {"ms": ms, "iters": it, "status": st, "rel_residual": math.sqrt(rtr / bb), "fell_back": fell}
        # one network application at the coarse level
        r = torch.randn(L.dims, device="cuda")
        row["unet_forward_ms"] = _event_ms(lambda: L.net.forward(r, L.z), 10)
        row["unet_timed_out"] = L.net.timed_out()
        out["fp32" if prec == 0 else "fp16_mixed"] = row
        P.close()
    out["held_out_iters"] = evaluate_coarse(params, timing=False)
    out["note"] = ("the plain graph-captured solve of the same system is pcg.ms; learned = network as the coarse "
                   "solver of the V-cycle (trained on exact coarse solutions from configurations 1-2)")
    return out


def run_learned_only(args):
    import torch
    torch.cuda.set_device(0)
    res = tuple(args.res) if args.res else RES
    print(json.dumps({"learned": learned_measure(res, reps=1)}), flush=True)
    return 0


def c2_measure(steps=5, warm=3, per_cell=8):
    """Configuration 2: solid wedge (chord 0.3, span 0.4, 20 degrees angle of
    attack) in a uniform inflow u = (1, 0, 0) carried by the solid outer
    shell, MGPCG_Solid_3 projection, dye emitters, and laden particles at
    `per_cell` per fluid cell (jittered per octant, seed 0) two-way coupled
    through the lp.py G2P/P2G kernels; EDGE at 256x128x128."""
    import torch
    from edgeb200.sim import EdgeSim, delta_emitters, uniform_flow, wedge_mask
    res, dx = RES, DX
    half = math.degrees(math.atan2(0.2, 0.3))
    mask, bvel = wedge_mask(res, dx, apex=(0.5, 0.5, 0.45), chord=0.3, half_angle_deg=half, aoa_deg=20.0,
                            thickness_cells=4, shell_vel=(1.0, 0.0, 0.0))
    sim = EdgeSim(res, dx, variant="edge", cfl=CFL, reinit_every=REINIT, ed_eps=EPS_FRAC * dx, base_level=BASE_LEVEL,
                  bfecc_clamp=True, visualize_dt=1e9, solid=(mask, bvel),
                  emitters=delta_emitters(offset=(0.5, 0.5, 0.47), half_angle_deg=half, radius=0.02), packed=True)
    sim.set_velocity(*uniform_flow(res, (1.0, 0.0, 0.0)))
    g = torch.Generator(device="cuda").manual_seed(0)
    fluid = torch.nonzero(mask.reshape(-1) <= 0).squeeze(1)
    nf = fluid.numel()
    cell = fluid.repeat_interleave(per_cell)
    octant = torch.arange(per_cell, device="cuda").repeat(nf)
    i = cell // (res[1] * res[2])
    j = (cell // res[2]) % res[1]
    k = cell % res[2]
    base = torch.stack([i, j, k], 1).float()
    sub = torch.stack([(octant >> 2) & 1, (octant >> 1) & 1, octant & 1], 1).float() * 0.5
    pos = ((base + sub + torch.rand(base.shape, generator=g, device="cuda") * 0.5) * dx).contiguous()
    vel = torch.zeros_like(pos)
    rad = (0.001 + 0.002 * torch.rand(pos.shape[0], generator=g, device="cuda")).contiguous()
    sim.add_particles(pos, vel, rad, tuple(n * dx for n in res), St=6.6e-2, gravity=0.0, density_ratio=2.0 / 3,
                      epiral_radius_ratio=35.0, Re=5.5, laden_radius=0.01)
    for _ in range(warm):
        sim.step()
    torch.cuda.synchronize()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(steps):
        sim.step()
    e1.record()
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / steps
    it, rtr, st = sim.proj.result()
    # per-step solve results over a few more (untimed) steps: the solid
    # projection stops at r.r < 1e-12 or 100 iterations (mgpcg_solid.py:413-416),
    # which is at the float32 floor of this grid, so an occasional solve
    # stagnates just above it and runs to the cap, as the reference's would;
    # which one varies from run to run with the order of the particle
    # scatter-adds (float atomics)
    hist = []
    for _ in range(steps):
        sim.step()
        hist.append(sim.proj.result())
    out = {"workload": "solid wedge + laden particles 256x128x128, EDGE, MGPCG_Solid_3", "ms_per_step": ms,
           "steps_per_s": 1e3 / ms, "particles": int(pos.shape[0]), "solid_cells": int((mask > 0).sum()),
           "last_solve_iters": it, "last_solve_status": st,
           "solve_iters_next_steps": [h[0] for h in hist], "solve_rtr_next_steps": [h[1] for h in hist],
           "solve_tolerance": "r.r < 1e-12 absolute, at most 100 iterations (the reference's)"}
    del sim
    torch.cuda.empty_cache()
    return out


C0_RES = (64, 32, 32)


def c0_measure(steps=100):
    """Configuration 0 in full: the 64x32x32 leapfrogging rings (4 levels,
    reinit every 12, CFL 0.5) for `steps` EDGE steps from t = 0, on the
    device (CUDA events around all steps; a separate 3-step run first warms
    the kernels and captures the solve graphs) and on the host cores (the
    oracle, C/OpenMP, every step timed), each choosing its own dt.  Also the
    relative L2 difference of velocity and dye after the last step between
    the two, next to the same difference between the oracle and its FMA twin
    (the oracle compiled with contracted multiply-adds): how far two float32
    evaluation orders drift apart over the run."""
    import numpy as np
    import torch
    from edgeb200.sim import EdgeSim, leapfrog_init
    from oracle import edge_oracle as O
    res = C0_RES
    dx = 1.0 / res[1]
    u, smoke = leapfrog_init(res, dx, radii=(0.21, 0.28), sigma=0.03, circulation=1.0, x_start=0.3)
    kw = dict(variant="edge", cfl=CFL, reinit_every=REINIT, ed_eps=EPS_FRAC * dx, base_level=2, bfecc_clamp=True,
              visualize_dt=1e9)
    warm = EdgeSim(res, dx, **kw)
    warm.set_velocity(*u)
    warm.set_smoke(smoke)
    for _ in range(3):
        warm.step()
    del warm
    sim = EdgeSim(res, dx, **kw)
    sim.set_velocity(*u)
    sim.set_smoke(smoke)
    torch.cuda.synchronize()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(steps):
        sim.step()
    e1.record()
    torch.cuda.synchronize()
    gpu_s = e0.elapsed_time(e1) / 1e3 / steps
    cores = os.cpu_count() or 1
    os.environ.setdefault("OMP_NUM_THREADS", str(cores))
    u0 = [t.cpu().numpy() for t in u]
    sm0 = smoke.cpu().numpy()
    okw = dict(cfl=CFL, reinit_every=REINIT, ed_eps=EPS_FRAC * dx, base_level=2)
    A = O.EdgeState(res, dx, [a.copy() for a in u0], sm0.copy())
    t0 = time.perf_counter()
    for _ in range(steps):
        O.edge_substep(A, **okw)
    cpu_s = (time.perf_counter() - t0) / steps
    B = O.EdgeState(res, dx, [a.copy() for a in u0], sm0.copy())
    with O.fma_twin():
        for _ in range(steps):
            O.edge_substep(B, **okw)

    def rel(x, y):
        x = np.asarray(x, np.float64)
        y = np.asarray(y, np.float64)
        return float(np.linalg.norm(x - y) / max(np.linalg.norm(y), 1e-30))

    return {"workload": "leapfrogging rings 64x32x32, EDGE, CFL 0.5, reinit 12, 4-level MGPCG", "steps": steps,
            "gpu_ms_per_step": 1e3 * gpu_s, "gpu_steps_per_s": 1.0 / gpu_s,
            "cpu_ms_per_step": 1e3 * cpu_s, "cpu_steps_per_s": 1.0 / cpu_s,
            "cpu_cores": int(os.environ["OMP_NUM_THREADS"]),
            "cpu_kind": "port (C/OpenMP restatement of the reference kernels)",
            "final_rel_l2": {"u_device_vs_oracle": max(rel(t.cpu().numpy(), a) for t, a in zip(sim.u, A.u)),
                             "u_twin_vs_oracle": max(rel(b, a) for b, a in zip(B.u, A.u)),
                             "smoke_device_vs_oracle": rel(sim.smoke.cpu().numpy(), A.smoke),
                             "smoke_twin_vs_oracle": rel(B.smoke, A.smoke)}}


C4_RES = (512, 256, 256)


def fp64_projection_error(P, u_pre, u_out):
    """Relative L2 error over all faces of the projected velocity u_out
    against the FP64 projection of the same pre-projection velocity u_pre
    (MGPCG_3.Poisson's steps, mgpcg.py:440-445, in float64: walls zeroed,
    divergence, A p = -div solved by float64 flexible CG, u - grad p)."""
    from edgeb200.precision import fp64_solve
    ux, uy, uz = (t.double().clone() for t in u_pre)
    ux[0] = 0.0
    ux[-1] = 0.0
    uy[:, 0] = 0.0
    uy[:, -1] = 0.0
    uz[:, :, 0] = 0.0
    uz[:, :, -1] = 0.0
    div = (ux[1:] - ux[:-1]) + (uy[:, 1:] - uy[:, :-1]) + (uz[:, :, 1:] - uz[:, :, :-1])
    p = fp64_solve(P, -div, rel_tol=1e-12)
    del div
    ux[1:-1] -= p[1:] - p[:-1]
    uy[:, 1:-1] -= p[:, 1:] - p[:, :-1]
    uz[:, :, 1:-1] -= p[:, :, 1:] - p[:, :, :-1]
    num = sum(float(((o.double() - r) ** 2).sum()) for o, r in zip(u_out, (ux, uy, uz)))
    den = sum(float((r ** 2).sum()) for r in (ux, uy, uz))
    return math.sqrt(num / den)


def c4_measure(steps=100, precision=2, warm=2):
    """Configuration 4: 512x256x256, initial velocity = curl of a seeded
    random vector potential (modes 1 <= |m| <= 8, amplitude |m|^(-17/6)),
    EDGE with FP16 V-cycle storage and the float64 Jacobian composition.
    Pass 1 times `steps` steps with CUDA events; pass 2 (untimed) repeats the
    same deterministic steps from the same initial state and measures after
    every step the error of its final projection against an FP64 projection
    of the same velocity, and the step's MGPCG iterations."""
    import torch
    from edgeb200.sim import EdgeSim, random_potential_init
    res = C4_RES
    dx = 1.0 / res[1]

    def fresh():
        sim = EdgeSim(res, dx, variant="edge", cfl=CFL, reinit_every=REINIT, ed_eps=EPS_FRAC * dx,
                      base_level=BASE_LEVEL, bfecc_clamp=True, visualize_dt=1e9, packed=True, precision=precision)
        sim.set_velocity(*random_potential_init(res, dx, seed=0))
        sim.proj.poisson(*sim.u)  # run_edge.py:557
        for _ in range(warm):
            sim.step()
        torch.cuda.synchronize()
        return sim

    torch.cuda.empty_cache()
    torch.cuda.reset_peak_memory_stats()
    sim = fresh()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(steps):
        sim.step()
    e1.record()
    torch.cuda.synchronize()
    total_ms = e0.elapsed_time(e1)
    peak = torch.cuda.max_memory_allocated()
    levels = sim.proj.levels
    del sim
    torch.cuda.empty_cache()
    sim = fresh()
    rec = []
    orig = sim.proj.poisson

    def poisson(ux, uy, uz, **kw):
        rec.append([t.clone() for t in (ux, uy, uz)])
        orig(ux, uy, uz, **kw)
    sim.proj.poisson = poisson
    errs, iters = [], []
    for _ in range(steps):
        rec.clear()
        sim.step()
        iters.append(sim.proj.result()[0])
        errs.append(fp64_projection_error(sim.proj, rec[-1], sim.u))
    del sim, rec
    torch.cuda.empty_cache()
    return {"workload": f"curl of a seeded random vector potential (1 <= |m| <= 8, |m|^-17/6) 512x256x256, EDGE, "
                        f"{'FP16' if precision == 2 else 'BF16'} V-cycle storage, float64 Jacobian composition, "
                        f"reinit 12, {levels}-level MGPCG",
            "steps": steps, "ms_per_step": total_ms / steps, "steps_per_s": 1e3 * steps / total_ms,
            "peak_device_bytes": int(peak), "second_projection_iters": iters,
            "fp64_projection_rel_error": [float(f"{e:.4g}") for e in errs],
            "fp64_projection_rel_error_max": max(errs)}


def mixed_learned_steps(steps=12, warm=3):
    """EDGE steps/s of the headline workload with the FP16 V-cycle and the
    float64 Jacobian composition (precision 2), and with the learned
    coarse-level solver on top (both projections of every step), next to
    the float32 steps; CUDA events around `steps` steps after `warm`."""
    import torch
    from edgeb200.sim import EdgeSim, four_vortex_init
    from edgeb200.train_unet import load_params
    params = load_params(COARSE_WEIGHTS) if os.path.exists(COARSE_WEIGHTS) else None
    out = {}
    for name, prec, learned in (("fp32", 0, None), ("mixed_fp16", 2, None), ("learned_fp32", 0, params),
                                ("learned_mixed_fp16", 2, params)):
        if name.startswith("learned") and params is None:
            continue
        sim = EdgeSim(RES, DX, variant="edge", cfl=CFL, reinit_every=REINIT, ed_eps=EPS_FRAC * DX,
                      base_level=BASE_LEVEL, bfecc_clamp=True, visualize_dt=0.1, packed=True, precision=prec,
                      learned=learned)
        u, smoke = four_vortex_init(RES, DX)
        sim.set_velocity(*u)
        sim.set_smoke(smoke)
        sim.proj.poisson(*sim.u)
        for _ in range(warm):
            sim.step()
        torch.cuda.synchronize()
        ms = _event_ms(lambda: [sim.step() for _ in range(steps)], 1) / steps
        out[name] = {"ms_per_step": ms, "steps_per_s": 1e3 / ms, "last_solve_iters": sim.proj.result()[0]}
        if learned is not None:
            out[name]["fell_back_last_solve"] = bool(sim.learned.fell_back)
        del sim
        torch.cuda.empty_cache()
    return out


def run_c4_only(args):
    import torch
    torch.cuda.set_device(0)
    print(json.dumps({"c4_mixed": c4_measure(steps=args.c4_steps)}), flush=True)
    return 0


def run_pcg_only(args):
    import torch
    torch.cuda.set_device(0)
    res = tuple(args.res) if args.res else RES
    print(json.dumps({"pcg": pcg_measure(res, reps=1)}), flush=True)
    return 0


def run_ours(args, rank, world, local_rank):
    import torch
    import torch.distributed as dist

    torch.cuda.set_device(local_rank)
    if world > 1:
        dist.init_process_group("nccl", timeout=__import__("datetime").timedelta(seconds=120),
                                device_id=torch.device("cuda", local_rank))
    from edgeb200 import ops
    sim = make_sim(args.variant, args.res, packed=not args.unpacked)
    mg_levels = sim.proj.levels
    if args.res and tuple(args.res) != RES:
        args.no_cpu_baseline = True  # profiling runs on a smaller grid
    for _ in range(args.warmup):
        sim.step()
    torch.cuda.synchronize()
    # per-stage breakdown (outside the timed region)
    stages, iters = instrumented_step(sim)
    # timed region
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    from edgeb200 import ops as _ops
    launches0 = _ops.launch_count()
    with ClockSampler(local_rank) as clk:
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(args.steps):
            sim.step()
        e1.record()
        torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    launches = _ops.launch_count() - launches0
    ms_max = max_over_ranks(e0.elapsed_time(e1), world, "cuda")
    value = replica_throughput(world, args.steps, ms_max)
    # end to end through the public API with host buffers: every step copies
    # the velocity and dye in from pinned host memory and reads them back
    # (EdgeSim.step_host: the copies on a copy stream beside the computation)
    e2e = None
    if args.e2e_steps < 0:
        args.e2e_steps = args.steps
    if args.e2e_steps > 0:
        host_u = [torch.empty(t_.shape, dtype=torch.float32, pin_memory=True) for t_ in sim.u]
        host_s = torch.empty(sim.smoke.shape, dtype=torch.float32, pin_memory=True)
        for h, d in zip(host_u, sim.u):
            h.copy_(d)
        host_s.copy_(sim.smoke)
        torch.cuda.synchronize()
        if world > 1:
            dist.barrier()
        e2 = torch.cuda.Event(enable_timing=True)
        e3 = torch.cuda.Event(enable_timing=True)
        e2.record()
        for _ in range(args.e2e_steps):
            sim.step_host(host_u, host_s)
        torch.cuda.current_stream().wait_stream(sim.copy_stream)
        e3.record()
        torch.cuda.synchronize()
        t2 = max_over_ranks(e2.elapsed_time(e3), world, "cuda")
        nbytes = sum(h.numel() * 4 for h in host_u) + host_s.numel() * 4
        e2e = {"value": replica_throughput(world, args.e2e_steps, t2), "unit": UNIT, "h2d_bytes_per_step": nbytes,
               "d2h_bytes_per_step": nbytes}
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        sec, cores, k = cpu_reference_steps(1, 1)
        cpu = {"value": 1.0 / sec, "unit": UNIT, "cores": cores, "kind": "port",
               "sample": "1 full substep of the same workload in the middle of a reinitialisation interval (after "
                         "one untimed substep), C/OpenMP restatement of the reference kernels"}
    # ED4 / ED8 / GE / EFM steps of the same workload (a few steps each, outside the
    # timed region of the EDGE line)
    variants = {}
    fp32_peak = ops.fma_peak_tflops() if not args.no_extras else None
    if args.no_extras:
        args.no_variants = True
    if not args.no_variants and args.variant == "edge" and not args.res:
        del sim
        torch.cuda.empty_cache()
        for v in ("ed4", "ed8", "ge", "efm"):
            vs = make_sim(v, args.res, packed=not args.unpacked)
            for _ in range(3):
                vs.step()
            torch.cuda.synchronize()
            # EFM's cost grows with the number of cached steps: time one whole
            # reinitialisation interval
            nsteps = REINIT if v == "efm" else 6
            a0 = torch.cuda.Event(enable_timing=True)
            a1 = torch.cuda.Event(enable_timing=True)
            a0.record()
            for _ in range(nsteps):
                vs.step()
            a1.record()
            torch.cuda.synchronize()
            vst, _ = instrumented_step(vs)
            if v == "efm":
                # the instrumented step backtracks through j + 1 cached fields
                flop = EFM_FLOP_PER_FACE_STEP * NF * (vs.i % vs.reinit_every + 1)
                roof = march_roofline(vst, v, fp32_peak, NC, flop_per_cell=flop / NC)
            else:
                roof = march_roofline(vst, v, fp32_peak, NC)
            variants[v] = {"ms_per_step": a0.elapsed_time(a1) / nsteps,
                           "steps_per_s": nsteps * 1e3 / a0.elapsed_time(a1),
                           "march_ms": round(vst.get("march_edge", 0.0), 4), "march_roofline_fp32": roof}
            del vs
            torch.cuda.empty_cache()
    c2 = c2_measure() if not (args.res or args.no_extras) else None
    mixed_steps = mixed_learned_steps() if not (args.res or args.no_extras) else None
    pcg = pcg_measure(RES) if not (args.res or args.no_extras) else None
    if pcg is not None:
        pcg["learned"] = learned_measure(RES)
        # the same solves at 512x256x256, where the level arrays no longer fit
        # in L2 and 16-bit storage halves their traffic
        pcg["at_512x256x256"] = pcg_measure(C4_RES, reps=3)
    c4 = c4_measure(steps=args.c4_steps) if not (args.res or args.no_extras) else None
    if world > 1:
        dist.barrier()
    if rank == 0:
        hbm, src = peaks()
        # HBM-bound roofline: the plain MGPCG solve to 1e-6 (one CUDA graph:
        # set-up, CG loop, solution copy); else the step's second projection
        if pcg:
            roof_kernel = "mgpcg_solve to 1e-6 relative residual (CG loop graph)"
            mg_bytes, solve_ms, it2 = pcg["algorithmic_bytes"], pcg["ms"], pcg["iters"]
        else:
            roof_kernel = "mgpcg_solve (CG loop graph, second projection of the step)"
            solve_ms = stages.get("mgpcg_solve_2", 0.0)
            it2 = max(iters[1], 0) + 1
            mg_bytes = MG_SETUP_BYTES + it2 * MG_ITER_BYTES
        achieved = mg_bytes / (solve_ms * 1e-3) / 1e9 if solve_ms > 0 else None
        # the headline workload unless --res / --variant ask for another one
        run_res = tuple(args.res) if args.res else RES
        grid = "x".join(map(str, run_res))
        metric = METRIC if (run_res == RES and args.variant == "edge") else \
            f"{args.variant.upper()} steps/s at {grid}"
        line = {
            "metric": metric, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms_max / args.steps, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded four-vortex rings, init_four_vorts geometry)",
            "config": {"workload": f"four-vortex collision {grid}, {args.variant.upper()}, CFL 0.5, reinit 12, "
                                   f"{mg_levels}-level MGPCG, BFECC clamp", "res": list(run_res),
                       "variant": args.variant,
                       "parallelism": f"replicas x{world}", "l2": "step working set ~1.7 GB > L2 (no flush needed)"},
            "roofline": {"kernel": roof_kernel, "bound": "hbm",
                         "achieved": achieved, "peak": hbm, "unit": "GB/s",
                         "frac": (achieved / hbm) if achieved else None,
                         "traffic": PCG_TRAFFIC if pcg else None,
                         "algorithmic_bytes": mg_bytes, "iterations": it2, "peak_source": src},
            "stages_ms": {k: round(v, 4) for k, v in stages.items()},
            "roofline_fp32": march_roofline(stages, args.variant, fp32_peak, math.prod(run_res)),
            "pcg": pcg,
            "variants": variants or None,
            "c2_solid_particles": c2,
            "c4_mixed": c4,
            "precision_steps": mixed_steps,
            "mgpcg_iters": list(iters),
            "clocks": clk.summary(),
            "gpu_launches": launches,
        }
        if e2e:
            line["e2e"] = e2e
        if cpu:
            line["cpu_baseline"] = cpu
        print(json.dumps(line), flush=True)
    if world > 1:
        dist.destroy_process_group()
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=24)
    ap.add_argument("--warmup", type=int, default=4)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--variant", default="edge", choices=["edge", "ed4", "ed8", "ge", "efm"])
    ap.add_argument("--e2e-steps", type=int, default=-1,
                    help="steps of the end-to-end (host buffers) measurement; default: --steps")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--ref-max-steps", type=int, default=2)
    ap.add_argument("--unpacked", action="store_true", help="separate-field map layout in the device driver "
                    "(default: float4 planes)")
    ap.add_argument("--pcg-only", action="store_true", help="only the PCG-to-1e-6 measurement (profiling)")
    ap.add_argument("--learned-only", action="store_true", help="only the learned-preconditioner measurement")
    ap.add_argument("--c2-only", action="store_true", help="only the solid + particle configuration")
    ap.add_argument("--c4-only", action="store_true", help="only the 512x256x256 mixed-precision configuration")
    ap.add_argument("--c4-steps", type=int, default=100)
    ap.add_argument("--c0-full", action="store_true",
                    help="configuration 0 in full (100 steps) on the device and on the host cores (oracle)")
    ap.add_argument("--no-variants", action="store_true", help="skip the ED4/ED8/GE/EFM step timings")
    ap.add_argument("--no-extras", action="store_true",
                    help="only the EDGE steps (no ED4/ED8, PCG or FP32-peak measurements; profiling)")
    ap.add_argument("--res", type=int, nargs=3, default=None,
                    help="grid override for profiling a smaller case (not a bench line)")
    args = ap.parse_args()
    rank = int(os.environ.get("RANK", 0))
    world = int(os.environ.get("WORLD_SIZE", 1))
    local_rank = int(os.environ.get("LOCAL_RANK", 0))
    if args.impl == "reference":
        return run_reference(args, rank, world)
    if args.pcg_only:
        return run_pcg_only(args)
    if args.learned_only:
        return run_learned_only(args)
    if args.c2_only:
        import torch
        torch.cuda.set_device(0)
        print(json.dumps({"c2_solid_particles": c2_measure()}), flush=True)
        return 0
    if args.c4_only:
        return run_c4_only(args)
    if args.c0_full:
        import torch
        torch.cuda.set_device(0)
        print(json.dumps({"c0_full": c0_measure()}), flush=True)
        return 0
    return run_ours(args, rank, world, local_rank)


if __name__ == "__main__":
    sys.exit(main())
