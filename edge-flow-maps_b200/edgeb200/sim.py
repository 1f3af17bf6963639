"""The EDGE / ED4 / ED8 / GE / EFM substep on one B200 (run_edge.py:588-712,
run_ed4.py:402-484, run_ed8.py:365-451, run_ge.py:363-448,
run_efm.py:319-406), on device-resident state.

Differences from the reference's orchestration that do not change results:
  * the flow-map state is ping-ponged between two buffer sets instead of being
    marched into temporaries and copied back (hermite.py:1515-1521);
  * right after a reinitialisation the EDGE march composes with the identity
    map analytically instead of reading a reset map;
  * the Hermite evaluations of psi and grad psi at the face centres, which
    map_u_psi, map_smoke_psi and clamp_smoke_psi each recompute
    (run_edge.py:377-505), are evaluated once per step into face buffers, and
    the pullbacks read them (the value accumulation of the gradient
    interpolant is the value interpolant, hermite.py:299-456);
  * the BFECC add/scale passes (run_edge.py:675-688) are fused into the
    pullback kernels, and copies become buffer swaps.
"""
import math

import torch

from . import _native as N
from . import ops
from .fields import face_shapes, zeros_cells, zeros_faces
from .projection import Projection

# GE (run_ge.py) keeps the ED8 map (psi, T, dT, d2T, full Hermite) and differs
# from ED8 only in the march; EFM (run_efm.py) keeps no cell map: its backward
# map is re-integrated on the faces every step through the cached velocities
VARIANTS = {"edge": N.HERMITE_GARM, "ed4": N.HERMITE_FD, "ed8": N.HERMITE_FULL, "ge": N.HERMITE_FULL, "efm": None}


class EdgeSim:
    def __init__(self, res, dx, variant="edge", cfl=0.5, reinit_every=12, ed_eps=None, base_level=3,
                 bfecc_clamp=True, visualize_dt=0.1, abs_tol=1e-12, rel_tol=1e-12, device="cuda", solid=None,
                 emitters=None, packed=True, precision=0, learned=None):
        """precision: 0 runs the reference's float32 arithmetic; 1 (BF16) and
        2 (FP16) store the projection's V-cycle levels in 16 bits (float32
        residuals and arithmetic, float64 dot products, as in
        Projection(precision=...)) and accumulate the EDGE march's composed
        Jacobian in float64.  learned: U-Net parameters (edgeb200.train_unet
        load_params) of the learned coarse-level solver; both projections of
        every step then run MGPCG with the network as the V-cycle's coarse
        group (edgeb200.unet.LearnedCoarsePCG, plain MGPCG as fallback)."""
        if variant not in VARIANTS:
            raise ValueError(f"variant must be one of {sorted(VARIANTS)}")
        if precision not in (0, 1, 2):
            raise ValueError("precision must be 0 (float32), 1 (BF16 V-cycle) or 2 (FP16 V-cycle)")
        self.precision = int(precision)
        N.load()
        self.res = tuple(int(n) for n in res)
        self.dx = float(dx)
        self.variant = variant
        self.hv = VARIANTS[variant]
        self.cfl = float(cfl)
        self.reinit_every = int(reinit_every)
        self.ed_eps = float(ed_eps) if ed_eps is not None else 0.025 * self.dx
        self.bfecc_clamp = bool(bfecc_clamp)
        self.visualize_dt = float(visualize_dt)
        self.abs_tol, self.rel_tol = abs_tol, rel_tol
        r = self.res
        # velocity (faces) and dye (cells)
        self.u = zeros_faces(r)
        self.tmp_u = zeros_faces(r)
        self.init_u = zeros_faces(r)
        self.err_u = zeros_faces(r)
        self.smoke = zeros_cells(r, 4)
        self.init_smoke = zeros_cells(r, 4)
        self.err_smoke = zeros_cells(r, 4)
        # backward map state, two sets (ping-pong); `packed` keeps them as
        # float4 planes (edge_map_pack layout) instead of the reference layout
        self.packed = bool(packed)
        if variant == "efm":
            # velocity cache of the current reinitialisation interval
            # (run_efm.py:104-109) and its step sizes in float32 (dts field)
            self.u_cache = [zeros_faces(r) for _ in range(self.reinit_every)]
            self.dts = [0.0] * self.reinit_every
            self.packed = False
            self.maps = None
        elif self.packed:
            planes = ops.PLANES[self.hv]
            self.pmaps = [torch.zeros((planes,) + r + (4,), dtype=torch.float32, device=device) for _ in range(2)]
            self._unpacked = None
        else:
            self.maps = [self._map_set() for _ in range(2)]
        self.cur = 0
        # forward map on the faces
        self.phi = zeros_faces(r, 3)
        self.F = zeros_faces(r, 3)
        # per-step face evaluation of the backward map
        self.fpsi = zeros_faces(r, 3)
        self.fcol = zeros_faces(r, 3)
        self.max_speed_dev = torch.zeros(1, dtype=torch.float32, device=device)
        self.max_speed_host = torch.zeros(1, dtype=torch.float32).pin_memory()
        # solid obstacles (MGPCG_Solid_3 path, run_edge.py:166-173) and dye
        # emitters re-injected through the forward map every step
        # (run_edge.py:643-648)
        self.solid = solid is not None
        if self.solid:
            mask, bvel = solid
            self.proj = Projection(r, base_level=base_level, mask=mask, bvel=bvel, precision=self.precision)
            self.abs_tol, self.rel_tol, self.max_iters = 1e-12, 0.0, 100  # mgpcg_solid.py:413-416
        else:
            self.proj = Projection(r, base_level=base_level, precision=self.precision)
            self.max_iters = 400  # mgpcg.py:434-438
        self.learned = None
        if learned is not None:
            from .unet import LearnedCoarsePCG
            self.learned = LearnedCoarsePCG(self.proj, learned)
        self.emitters = emitters
        self.side_stream = torch.cuda.Stream(device=device)
        self.particles = None
        self.i = -1
        self.sub_t = 0.0
        self.frame_idx = 0
        self.last_dt = 0.0
        self.last_iters = (None, None)
        self._io = None  # step_host: events and copy stream of the host round trip

    def _map_set(self):
        r = self.res
        m = {"psi": zeros_cells(r, 3), "T": [zeros_cells(r, 3) for _ in range(3)]}
        if self.variant in ("edge", "ed8", "ge"):
            m["dT"] = [zeros_cells(r, 3) for _ in range(3)]
        if self.variant in ("ed8", "ge"):
            m["d2T"] = [zeros_cells(r) for _ in range(3)]
        return m

    @property
    def map(self):
        """The current backward map in the reference layout (unpacked on
        demand when the driver keeps packed planes); None for EFM."""
        if self.variant == "efm":
            return None
        if not self.packed:
            return self.maps[self.cur]
        m = self._map_set()
        ops.map_unpack(self.hv, self.pmaps[self.cur], m["psi"], m["T"], m.get("dT"), m.get("d2T"))
        return m

    # -- state I/O --------------------------------------------------------------
    def set_velocity(self, u_x, u_y, u_z):
        for d, s in zip(self.u, (u_x, u_y, u_z)):
            d.copy_(s)

    def set_smoke(self, smoke):
        self.smoke.copy_(smoke)

    def state_dict(self):
        """Everything a later step reads: velocity, dye, the interval's
        initial fields, both maps (backward map state or EFM velocity cache,
        forward map), the particles and the frame bookkeeping.  Loading it
        into a simulation built with the same arguments continues bit for
        bit, also in the middle of a reinitialisation interval (the
        reference's checkpoints hold u and dye only and restart the maps,
        run_edge.py:559-566)."""
        d = {"u": list(self.u), "smoke": self.smoke, "init_u": list(self.init_u), "init_smoke": self.init_smoke,
             "phi": list(self.phi), "F": list(self.F),
             "scalars": dict(i=self.i, sub_t=self.sub_t, frame_idx=self.frame_idx, last_dt=self.last_dt,
                             cur=self.cur, variant=self.variant, packed=self.packed, res=self.res)}
        if self.variant == "efm":
            d["u_cache"] = [list(c) for c in self.u_cache]
            d["scalars"]["dts"] = list(self.dts)
        elif self.packed:
            d["pmap"] = self.pmaps[self.cur]
        else:
            d["map"] = self.maps[self.cur]
        if self.particles is not None:
            d["particles"] = {k: v for k, v in self.particles.items() if torch.is_tensor(v) or isinstance(v, list)}
        return {k: _detach_copy(v) for k, v in d.items()}

    def load_state_dict(self, d):
        s = d["scalars"]
        if s["variant"] != self.variant or tuple(s["res"]) != self.res or s["packed"] != self.packed:
            raise ValueError("state was saved by a simulation with another variant, grid or map layout")
        _copy_into(self.u, d["u"])
        _copy_into(self.init_u, d["init_u"])
        _copy_into(self.phi, d["phi"])
        _copy_into(self.F, d["F"])
        self.smoke.copy_(d["smoke"])
        self.init_smoke.copy_(d["init_smoke"])
        self.i, self.sub_t, self.frame_idx, self.last_dt = s["i"], s["sub_t"], s["frame_idx"], s["last_dt"]
        self.cur = s["cur"]
        if self.variant == "efm":
            for dst, src in zip(self.u_cache, d["u_cache"]):
                _copy_into(dst, src)
            self.dts = list(s["dts"])
        elif self.packed:
            self.pmaps[self.cur].copy_(d["pmap"])
        else:
            m = self.maps[self.cur]
            for k, v in d["map"].items():
                _copy_into(m[k], v) if isinstance(v, list) else m[k].copy_(v)
        if "particles" in d:
            if self.particles is None:
                raise ValueError("state holds particles: call add_particles first")
            for k, v in d["particles"].items():
                _copy_into(self.particles[k], v) if isinstance(v, list) else self.particles[k].copy_(v)

    def add_particles(self, pos, vel, rad, domain, St, gravity, density_ratio, epiral_radius_ratio, Re,
                      laden_radius):
        """Two-way coupled laden particles (the `lp` branch of the driver,
        run_edge.py:627-641, 662-667, 704-708; sim/lp.py).  pos, vel: (N, 3);
        rad: (N,); domain: (Lx, Ly, Lz)."""
        n = pos.shape[0]
        self.particles = dict(pos=pos, vel=vel, rad=rad, acc=torch.zeros_like(vel), vdiff=torch.zeros_like(vel),
                              num=n, L=tuple(float(v) for v in domain), St=St, gravity=gravity,
                              density_ratio=density_ratio, erad=epiral_radius_ratio, Re=Re, lrad=laden_radius,
                              drag=zeros_faces(self.res), vis=zeros_faces(self.res),
                              max_dev=torch.zeros(1, dtype=torch.float32, device=pos.device))

    # -- dt (run_edge.py:595-614) -------------------------------------------------
    def next_dt(self):
        ops.max_speed(self.u, self.max_speed_dev)
        if self.particles is not None:
            P = self.particles
            ops.lp_max_speed(P["vel"], P["num"], P["max_dev"])
            # dt = min(CFL dx / max|u|, CFL dx / max|v_particle|)
            torch.maximum(self.max_speed_dev, P["max_dev"], out=self.max_speed_dev)
        self.max_speed_host.copy_(self.max_speed_dev, non_blocking=True)
        torch.cuda.current_stream().synchronize()
        ms = float(self.max_speed_host[0])
        curr = self.cfl * self.dx / ms
        if self.sub_t + curr >= self.visualize_dt:
            curr = self.visualize_dt - self.sub_t
            self.sub_t = 0.0
            self.frame_idx += 1
        elif self.sub_t + curr * 2 >= self.visualize_dt:
            curr = (self.visualize_dt - self.sub_t) / 2
            self.sub_t += curr
        else:
            self.sub_t += curr
        return curr

    # -- the substep ---------------------------------------------------------------
    def step(self, dt=None, timers=None):
        tm = timers if timers is not None else _NoTimer()
        tm.start("substep")
        tm.start("pre-advect")
        self.i += 1
        j = self.i % self.reinit_every
        curr_dt = self.next_dt() if dt is None else float(dt)
        self.last_dt = curr_dt
        dx = self.dx
        reinit = j == 0
        io = self._io
        if io is not None and (reinit or self.emitters is not None):
            torch.cuda.current_stream().wait_event(io["smoke_in"])
        if reinit:
            # run_edge.py:616-625
            ops.reset_faces(self.res, dx, self.phi, self.F)
            for a, b in zip(self.init_u, self.u):
                ops.copy(b, a)
            ops.copy(self.smoke, self.init_smoke)
        if self.emitters is not None:
            centers, colors, radius = self.emitters
            self.smoke.zero_()
            ops.emit_smoke(dx, centers, colors, radius, self.smoke)
            ops.pullback_dye(self.smoke, dx, self.phi, self.err_smoke)
            ops.axpy(self.init_smoke, self.err_smoke, 1.0, self.init_smoke)
            ops.clamp_max(self.init_smoke, 1.0)
        if self.particles is not None:
            self._particles_forces(curr_dt)
        # midpoint velocity (run_edge.py:650-654)
        ops.advect_u_sl(self.u, dx, 0.5 * curr_dt, self.tmp_u)
        self.u, self.tmp_u = self.tmp_u, self.u
        tm.stop("pre-advect")
        proj = self.learned if self.learned is not None else self.proj
        proj.poisson(*self.u, abs_tol=self.abs_tol, rel_tol=self.rel_tol, max_iters=self.max_iters)
        tm.start("advect")
        # The backward-map march and the forward-map march both read only the
        # projected u: the forward map runs on a side stream next to the march
        # (the march's register footprint leaves most warp slots free), and
        # later the dye chain runs there next to the velocity chain.
        main = torch.cuda.current_stream()
        side = self.side_stream
        ev = torch.cuda.Event()
        ev.record(main)
        with torch.cuda.stream(side):
            side.wait_event(ev)
            ops.advance_map(self.u, dx, curr_dt, self.phi, self.F)          # run_edge.py:660
            ev_fwd = torch.cuda.Event()
            ev_fwd.record(side)
        self._march(curr_dt, reinit, j)
        main.wait_event(ev_fwd)
        if self.particles is not None:
            # the forcing integrated into the map's origin velocity through the
            # forward map (run_edge.py:662-667)
            P = self.particles
            ops.pullback_u(P["vis"], dx, self.phi, self.F, self.tmp_u)
            for a, t in zip(self.init_u, self.tmp_u):
                ops.axpy(a, t, curr_dt, a)
        if self.variant == "efm":
            pass  # the backtrack wrote fpsi / fcol
        elif self.packed:
            ops.face_map_packed(self.hv, dx, self.pmaps[self.cur], self.res, self.fpsi, self.fcol)
        else:
            m = self.maps[self.cur]
            ops.face_map(self.hv, dx, m["psi"], m["T"], m.get("dT"), m.get("d2T"), self.fpsi, self.fcol)
        ev_map = torch.cuda.Event()
        ev_map.record(main)
        with torch.cuda.stream(side):
            # dye: smoke = smoke_init(psi); err = 0.5*(smoke(phi) - smoke_init);
            # smoke - err(psi), clamped                     run_edge.py:670, 677-689
            side.wait_event(ev_map)
            if io is not None:
                side.wait_event(io["smoke_in"])  # the dye chain overwrites the dye the copy brings in
            ops.pullback_dye(self.init_smoke, dx, self.fpsi, self.smoke)
            ops.pullback_dye(self.smoke, dx, self.phi, self.err_smoke, init=self.init_smoke, scale=0.5)
            ops.pullback_dye(self.err_smoke, dx, self.fpsi, self.smoke, sub=self.smoke, clampsrc=self.init_smoke)
            ev_dye = torch.cuda.Event()
            ev_dye.record(side)
        if io is not None:
            # the step's dye is final: copy it out while the velocity chain runs
            io["copy"].wait_event(ev_dye)
            with torch.cuda.stream(io["copy"]):
                io["host_smoke"].copy_(self.smoke, non_blocking=True)
                io["smoke_out"] = io["copy"].record_event()
        # u = (grad psi)^T u_init(psi)                                 run_edge.py:669
        ops.pullback_u(self.init_u, dx, self.fpsi, self.fcol, self.u)
        # err = 0.5*(F^T u(phi) - u_init)                             run_edge.py:671-676
        ops.pullback_u(self.u, dx, self.phi, self.F, self.err_u, init=self.init_u, scale=0.5)
        # u - (grad psi)^T err(psi)                                    run_edge.py:683-686
        ops.pullback_u(self.err_u, dx, self.fpsi, self.fcol, self.tmp_u, sub=self.u)
        main.wait_event(ev_dye)
        if self.bfecc_clamp:
            ops.clamp_u(self.tmp_u, self.u, self.tmp_u)                  # run_edge.py:690-696
        self.u, self.tmp_u = self.tmp_u, self.u
        tm.stop("advect")
        if self.particles is not None:
            # Poisson_with_buffer: vis receives -grad p (run_edge.py:704-708)
            P = self.particles
            for v in P["vis"]:
                v.zero_()
            proj.poisson(*self.u, f=P["vis"], abs_tol=self.abs_tol, rel_tol=self.rel_tol,
                         max_iters=self.max_iters)
        else:
            proj.poisson(*self.u, abs_tol=self.abs_tol, rel_tol=self.rel_tol, max_iters=self.max_iters)
        tm.stop("substep")
        return curr_dt

    def step_host(self, host_u, host_smoke, dt=None, chunks=4):
        """One step whose state comes from and goes back to pinned host
        buffers (the three face velocity arrays and the dye), as a caller
        that keeps the fields on the host drives the simulation.  Returns dt;
        the host buffers hold the step's results once the current stream and
        the two copy streams have completed (torch.cuda.synchronize(); the
        last copies of a step run on `self.copy_stream`).

        The copies run on two copy streams beside the computation, host to
        device on `self.copy_in_stream`, device to host on `self.copy_stream`:
        the velocity in before the step starts; the dye in while the step's
        first half runs (a step reads the incoming dye only at a
        reinitialisation or with emitters, and otherwise the dye chain
        overwrites it, so only those wait for it); the dye out as soon as the
        dye chain ends, during the velocity chain and the projection; the
        velocity out at the end.  Each velocity array moves in `chunks`
        pieces, and a piece of the next step's copy in waits only for the
        same piece of this step's copy out, so the two directions of the
        round trip overlap instead of following each other."""
        if not hasattr(self, "copy_stream"):
            dev = self.u[0].device
            self.copy_stream = torch.cuda.Stream(device=dev)
            self.copy_in_stream = torch.cuda.Stream(device=dev)
            self._host_out = None  # events of the previous step_host's copies out
        main = torch.cuda.current_stream()
        ci, co = self.copy_in_stream, self.copy_stream
        pieces = []
        for d, h in zip(self.u, host_u):
            fd, fh = d.view(-1), h.view(-1)
            n = fd.numel()
            step_n = -(-n // max(1, int(chunks)))
            for a0 in range(0, n, step_n):
                pieces.append((fd[a0:a0 + step_n], fh[a0:a0 + step_n]))
        prev = self._host_out
        if prev is not None and len(prev["u"]) != len(pieces):
            prev = {"u": [prev["u"][-1]] * len(pieces), "smoke": prev["smoke"]}
        ci.wait_event(main.record_event())  # the previous step's kernels are done with the buffers
        with torch.cuda.stream(ci):
            for q, (d, h) in enumerate(pieces):
                if prev is not None:
                    ci.wait_event(prev["u"][q])  # this piece of the host buffer has been read back
                d.copy_(h, non_blocking=True)
            u_in = ci.record_event()
            if prev is not None:
                ci.wait_event(prev["smoke"])
            self.smoke.copy_(host_smoke, non_blocking=True)
            smoke_in = ci.record_event()
        main.wait_event(u_in)
        io = {"copy": co, "smoke_in": smoke_in, "host_smoke": host_smoke}
        self._io = io
        try:
            dt = self.step(dt=dt)
        finally:
            self._io = None
        co.wait_event(main.record_event())
        with torch.cuda.stream(co):
            if "smoke_out" not in io:
                host_smoke.copy_(self.smoke, non_blocking=True)
                io["smoke_out"] = co.record_event()
            outs = []
            for d, h in pieces:
                h.copy_(d, non_blocking=True)
                outs.append(co.record_event())
        self._host_out = {"u": outs, "smoke": io["smoke_out"]}
        return dt

    def _particles_forces(self, dt):
        """run_edge.py:627-641: G2P, particle update, P2G drag, viscous force."""
        P = self.particles
        dx, u = self.dx, self.u
        ops.lp_acc(u, dx, P["vel"], P["pos"], P["acc"], P["num"], dt, P["St"], P["gravity"])
        ops.lp_velocity(P["acc"], P["vel"], P["pos"], dt, dx, P["num"], P["L"])
        ops.lp_vel_diff(u, dx, P["vel"], P["vdiff"], P["pos"], P["num"], P["St"], P["density_ratio"], P["erad"])
        ops.lp_p2g(self.res, dx, P["drag"], P["vdiff"], P["pos"], P["rad"], P["num"], P["lrad"], P["L"])
        ops.lp_position(P["vel"], P["pos"], dt, P["num"], P["L"])
        ops.lp_viscous(u, dx, P["Re"], P["vis"])
        for v, d in zip(P["vis"], P["drag"]):
            ops.axpy(v, d, 1.0, v)

    def _march(self, dt, reinit, j=0):
        dx, eps = self.dx, self.ed_eps
        if self.variant == "efm":
            # run_efm.py:360-365: cache u, then backtrack_psi_grid(j) onto the faces
            for a, b in zip(self.u_cache[j], self.u):
                ops.copy(b, a)
            self.dts[j] = float(torch.tensor(dt, dtype=torch.float32))
            ops.efm_backtrack(self.u_cache[:j + 1], self.dts[:j + 1], dx, self.fpsi, self.fcol)
            return
        if self.packed:
            src, dst = self.pmaps[self.cur], self.pmaps[self.cur ^ 1]
            if reinit and self.variant != "edge":
                m = self._map_set()
                ops.reset_cells(dx, m["psi"], m["T"], m.get("dT"), m.get("d2T"))
                ops.map_pack(self.hv, m["psi"], m["T"], m.get("dT"), m.get("d2T"), src)
            if self.variant == "ge":
                ops.march_ge_packed(self.u, dx, dt, src, dst, self.res)
            else:
                ops.march_packed(self.hv, self.u, dx, dt, eps, src, dst, self.res,
                                 identity=reinit and self.variant == "edge", f64_compose=self.precision > 0)
            self.cur ^= 1
            return
        src, dst = self.maps[self.cur], self.maps[self.cur ^ 1]
        if self.variant == "edge":
            ops.march_edge(self.u, dx, dt, eps, src["psi"], src["T"], src["dT"], dst["psi"], dst["T"], dst["dT"],
                           identity=reinit)
        else:
            if reinit:
                ops.reset_cells(dx, src["psi"], src["T"], src.get("dT"), src.get("d2T"))
            if self.variant == "ed4":
                ops.march_ed4(self.u, dx, dt, eps, src["psi"], src["T"], dst["psi"], dst["T"])
            elif self.variant == "ge":
                ops.march_ge(self.u, dx, dt, src["psi"], src["T"], src["dT"], src["d2T"], dst["psi"], dst["T"],
                             dst["dT"], dst["d2T"])
            else:
                ops.march_ed8(self.u, dx, dt, eps, src["psi"], src["T"], src["dT"], src["d2T"], dst["psi"],
                              dst["T"], dst["dT"], dst["d2T"])
        self.cur ^= 1


def _detach_copy(v):
    if torch.is_tensor(v):
        return v.detach().clone()
    if isinstance(v, list):
        return [_detach_copy(x) for x in v]
    if isinstance(v, dict):
        return {k: _detach_copy(x) for k, x in v.items()}
    return v


def _copy_into(dst, src):
    for a, b in zip(dst, src):
        a.copy_(b)


class _NoTimer:
    def start(self, k):
        pass

    def stop(self, k, skip=0):
        pass


# -- initial conditions of the benchmark cases ---------------------------------------
def four_vortex_init(res, dx, num_samples=500, device="cuda"):
    """init_four_vorts (init_conditions.py:38-67) with the long axis along x:
    the reference's (x, y, z) ring geometry is mapped to (z, y, x), so the rings
    travel along x on an (nx, ny, nz) = (2N, N, N) grid.  Returns face
    velocities (after split_central_vector) and the 4-channel dye."""
    u_c = zeros_cells(res, 3, device)
    smoke = zeros_cells(res, 4, device)
    tmp = zeros_cells(res, 4, device)
    x_off = y_off = 0.16
    size = 0.15
    c45 = math.cos(math.pi / 4)
    perm = lambda v: (v[2], v[1], v[0])  # noqa: E731  reference (x,y,z) -> ours (z,y,x)
    Lz = res[0] * dx  # long axis
    mid = Lz / 2.0
    rings = [
        (2.e-2, (0.5 - x_off, 0.5 - y_off, mid), (-c45, c45, 0.), (1, 0, 0)),
        (-2.e-2, (0.5 + x_off, 0.5 - y_off, mid), (c45, c45, 0.), (0, 1, 0)),
        (2.e-2, (0.5 - x_off, 0.5 + y_off, mid), (c45, c45, 0.), (0, 0, 1)),
        (-2.e-2, (0.5 + x_off, 0.5 + y_off, mid), (-c45, c45, 0.), (0, 0, 0)),
    ]
    for q, (w, c, ex, color) in enumerate(rings):
        n = math.sqrt(sum(v * v for v in ex))
        ex = tuple(v / n for v in ex)
        target = smoke if q == 0 else tmp
        if q > 0:
            tmp.zero_()
        ops.add_vortex_ring(dx, w, size, 0.024, perm(c), perm(ex), perm((0., 0., 1.)), u_c, target, color,
                            num_samples)
        if q > 0:
            ops.axpy(smoke, tmp, 1.0, smoke)
    u = zeros_faces(res, None, device)
    ops.split_central_vector(u_c, u)
    return u, smoke


def leapfrog_init(res, dx, radii=(0.21, 0.28), sigma=0.03, circulation=1.0, x_start=0.3, num_samples=2000,
                  device="cuda"):
    """Two coaxial rings along x (add_vortex_ring_and_smoke, init_conditions.py:11-36;
    init_vorts_leapfrog geometry, init_conditions.py:70-86, with the radii,
    core and centre of the 64x32x32 leapfrogging benchmark)."""
    u_c = zeros_cells(res, 3, device)
    smoke = zeros_cells(res, 4, device)
    tmp = zeros_cells(res, 4, device)
    gap = 0.625 * radii[0]
    for q, (rad, col) in enumerate(zip(radii, ((1., 0., 0.), (0., 0., 1.)))):
        target = smoke if q == 0 else tmp
        ops.add_vortex_ring(dx, circulation, rad, sigma, (x_start + q * gap, 0.5, 0.5), (0., 0., -1.), (0., 1., 0.),
                            u_c, target, col, num_samples)
    ops.axpy(smoke, tmp, 1.0, smoke)
    u = zeros_faces(res, None, device)
    ops.split_central_vector(u_c, u)
    return u, smoke


def random_potential_init(res, dx, kmax=8, slope=-17.0 / 6.0, seed=0, u_max=1.0, device="cuda"):
    """Divergence-free-in-the-continuum initial velocity u = curl A of a seeded
    random vector potential: every Fourier mode of the grid's periodic box
    with integer index vector m, 1 <= |m| <= kmax (and below each axis's
    Nyquist index), gets an independent
    complex normal amplitude per component scaled by |m|^slope (numpy
    default_rng(seed), modes in lexicographic order of (m0, m1, m2) with
    m2 >= 0); A is evaluated at the cell centres by an inverse real FFT,
    u_c = curl(A) by the reference's clamped central differences
    (taichi_utils.py:69-92), split to the faces (taichi_utils.py:103-116) and
    scaled so that max |u| = u_max.  No reference counterpart (the
    512x256x256 mixed-precision workload)."""
    import numpy as np
    nx, ny, nz = res
    rng = np.random.default_rng(seed)
    r = np.arange(-kmax, kmax + 1)
    m0, m1, m2 = np.meshgrid(r, r, np.arange(0, kmax + 1), indexing="ij")
    k2 = m0 ** 2 + m1 ** 2 + m2 ** 2
    # modes below each axis's Nyquist index only (no two modes share a bin)
    sel = (k2 >= 1) & (k2 <= kmax * kmax) & (2 * np.abs(m0) < nx) & (2 * np.abs(m1) < ny) & (2 * m2 < nz)
    m0, m1, m2, k2 = m0[sel], m1[sel], m2[sel], k2[sel]
    amp = np.power(k2.astype(np.float64), slope / 2.0)
    coef = (rng.standard_normal((3, m0.size)) + 1j * rng.standard_normal((3, m0.size))) * amp
    spec = torch.zeros((3, nx, ny, nz // 2 + 1), dtype=torch.complex128, device=device)
    idx = (torch.from_numpy(m0 % nx).to(device), torch.from_numpy(m1 % ny).to(device),
           torch.from_numpy(m2).to(device))
    for c in range(3):
        spec[c][idx] = torch.from_numpy(coef[c]).to(device)
    A = torch.fft.irfftn(spec, s=(nx, ny, nz), dim=(1, 2, 3), norm="forward")
    A = A.permute(1, 2, 3, 0).contiguous().float()
    u_c = zeros_cells(res, 3, device)
    ops.curl(A, u_c, dx)
    del A, spec
    u_c.mul_(float(u_max) / float(u_c.norm(dim=-1).max()))
    u = zeros_faces(res, None, device)
    ops.split_central_vector(u_c, u)
    return u


def wedge_mask(res, dx, apex=(0.1, 0.5, 0.2), chord=1.0, half_angle_deg=15.0, aoa_deg=0.0, thickness_cells=4,
               shell_vel=(0.6 * math.cos(math.radians(20)), 0.0, 0.6 * math.sin(math.radians(20))), device="cuda"):
    """Solid mask and solid velocities of the delta-wing case
    (set_boundary_mask_delta, init_conditions.py:139-167 and
    set_boundary_mask_delta_kernel, 128-136): a triangular plate with its apex
    at `apex`, extending `chord` downstream along x (tilted by `aoa_deg` about
    the y axis), half angle `half_angle_deg`, `thickness_cells` cells thick,
    plus a solid outer shell of cells carrying `shell_vel` (the inflow).  The
    reference voxelises the triangle with trimesh (not installed); here a cell
    is solid when its centre is within the plate's thickness and inside the
    triangle widened by half a cell."""
    import numpy as np
    nx, ny, nz = res
    idx = np.indices(res).astype(np.float64)
    X = (idx + 0.5) * dx
    rel = [X[0] - apex[0], X[1] - apex[1], X[2] - apex[2]]
    a = math.radians(aoa_deg)
    # plate coordinates: s along the chord, n normal to the plate
    s_ = rel[0] * math.cos(a) + rel[2] * math.sin(a)
    n_ = -rel[0] * math.sin(a) + rel[2] * math.cos(a)
    t = math.tan(math.radians(half_angle_deg))
    inside = (s_ >= -0.5 * dx) & (s_ <= chord * math.cos(math.radians(half_angle_deg)) + 0.5 * dx) & \
             (np.abs(rel[1]) <= s_ * t + 0.5 * dx) & (n_ >= 0.0) & (n_ < thickness_cells * dx)
    mask = inside.astype(np.int32)
    bvel = np.zeros(tuple(res) + (3,), np.float32)
    shell = np.zeros(res, bool)
    shell[0, :, :] = shell[-1, :, :] = True
    shell[:, 0, :] = shell[:, -1, :] = True
    shell[:, :, 0] = shell[:, :, -1] = True
    mask[shell] = 1
    bvel[shell] = np.asarray(shell_vel, np.float32)
    return (torch.from_numpy(mask).to(device), torch.from_numpy(bvel).to(device))


def delta_emitters(offset=(0.1, 0.5, 0.25), half_angle_deg=15.0, radius=0.015):
    """The eight dye emitters of emit_smoke_delta (init_conditions.py:177-232)."""
    a = math.radians(half_angle_deg)
    centers, colors = [], []
    for d, col in ((0.25, (1, 0, 0, 0)), (0.45, (0, 1, 0, 0)), (0.65, (0, 0, 1, 0)), (0.85, (0, 0, 0, 1))):
        x, y = math.cos(a) * d, math.sin(a) * d
        for sy in (1, -1):
            centers.append((x + offset[0], sy * y + offset[1], offset[2]))
            colors.append(col)
    return centers, colors, radius


def uniform_flow(res, vel, device="cuda"):
    """init_delta (init_conditions.py:170-175) followed by split_central_vector:
    a uniform velocity on every face."""
    u = zeros_faces(res, None, device)
    for c in range(3):
        u[c].fill_(float(vel[c]))
    return u


# the two ink-drop cases of sim/lp_init.py: (sphere radius, centre x, centre z,
# cell velocity inside the sphere, particle velocity)
_INK = {
    0: (3.0, 64.0, 64.0, (0.0, 1.0, 0.0), (0.0, 1.0, 0.0)),                        # lp_init.py:6-35
    1: (8.0, 128.0 * 0.3, 128.0 * 0.3, (0.2, 0.5, 0.3), (0.0, 0.0, 0.0)),          # lp_init.py:69-104
}


def ink_particles(case, num, domain_range_y=256.0):
    """ink_drop_particle_case0/1 (lp_init.py:6-20, 69-86): `num` positions
    drawn by rejection from the cube around the sphere with Python's random
    module seeded 0, in the reference's order (so the same particles)."""
    import random

    import numpy as np
    r, cx, cz = _INK[case][:3]
    cy = 0.05 * domain_range_y
    out = np.zeros((num, 3), np.float64)
    rng = random.Random(0)
    n = 0
    while n < num:
        x = rng.random() * r * 2 + cx - r
        y = rng.random() * r * 2 + cy
        z = rng.random() * r * 2 + cz - r
        if (x - cx) ** 2 + (y - cy - r) ** 2 + (z - cz) ** 2 < r ** 2:
            out[n] = (x, y, z)
            n += 1
    return out


def ink_init(case, res, dx, num, laden_radius, domain_range_y=256.0, device="cuda"):
    """ink_init_case0/1 (lp_init.py:48-66, 107-125) followed by
    split_central_vector: face velocities (the sphere of cells moving with the
    case's velocity), particle positions and velocities, and the per-particle
    reference radius (compute_laden_radius for all)."""
    import numpy as np
    r, cx, cz, ucell, upart = _INK[case]
    cy = 0.05 * domain_range_y
    X = (np.indices(res).astype(np.float32) + np.float32(0.5)) * np.float32(dx)
    inside = (X[0] - cx) ** 2 + (X[1] - cy - r) ** 2 + (X[2] - cz) ** 2 < r ** 2
    uc = np.zeros(tuple(res) + (3,), np.float32)
    uc[inside] = np.asarray(ucell, np.float32)
    u = zeros_faces(res, None, device)
    ops.split_central_vector(torch.from_numpy(uc).to(device), u)
    pos = torch.from_numpy(ink_particles(case, num, domain_range_y).astype(np.float32)).to(device)
    vel = torch.tensor(upart, dtype=torch.float32, device=device).expand(num, 3).contiguous()
    rad = torch.full((num,), float(laden_radius), dtype=torch.float32, device=device)
    return u, pos, vel, rad
