"""Learned preconditioner: a 3-D U-Net whose convolutions run on the B200
tensor cores (tcgen05, BF16 operands, FP32 accumulation in TMEM), trained on
the GPU by the library's own forward and backward kernels, and used inside
flexible CG with the plain MGPCG V-cycle as fallback.  There is no reference
counterpart (the reference only has MGPCG).

Architecture (16/32/64 channels, 3x3x3 convolutions, 2x2x2 mean pooling,
nearest upsampling, skip connections as second inputs of the decoder
convolutions; input scaled by 1/rms so the map is scale-equivariant):

    e0 = relu(c3(relu(c3(r s; W0a)); W0b))               16 ch, full grid
    e1 = relu(c3(relu(c3(pool(e0); W1a)); W1b))          32 ch, 1/2 grid
    e2 = relu(c3(relu(c3(pool(e1); W2a)); W2b))          64 ch, 1/4 grid
    f1 = relu(c3(relu(c3(up(e2); W3a) + c3(e1; W3s)); W3b))
    f0 = relu(c3(relu(c3(up(f1); W4a) + c3(e0; W4s)); W4b))
    z  = c3(f0; W5) / s
"""
import ctypes

import torch

from . import _native as N
from .fields import ptr, ptr_any, stream

BF16 = (torch.bfloat16,)
I32 = (torch.int32,)
F64 = (torch.float64,)

CH = (16, 32, 64)
# (name, out channels, in channels); skip convs ("s") share the bias of "a"
LAYERS = [
    ("W0a", CH[0], 1), ("W0b", CH[0], CH[0]),
    ("W1a", CH[1], CH[0]), ("W1b", CH[1], CH[1]),
    ("W2a", CH[2], CH[1]), ("W2b", CH[2], CH[2]),
    ("W3a", CH[1], CH[2]), ("W3s", CH[1], CH[1]), ("W3b", CH[1], CH[1]),
    ("W4a", CH[0], CH[1]), ("W4s", CH[0], CH[0]), ("W4b", CH[0], CH[0]),
    ("W5", 1, CH[0]),
]
BIASES = ["W0a", "W0b", "W1a", "W1b", "W2a", "W2b", "W3a", "W3b", "W4a", "W4b", "W5"]
SHAPES = {n: (co, ci) for n, co, ci in LAYERS}
TC_LAYERS = [n for n, co, ci in LAYERS if ci >= 16 and co >= 16]


def tc_selftest(mode, A, B):
    """D = A B^T through one tcgen05 GEMM (mode 0: A 128xK, B NxK; mode 1:
    A Kx64, B KxN, i.e. D = A^T B).  Returns (D, timed_out)."""
    if mode == 0:
        M, K = A.shape
        n = B.shape[0]
    else:
        K, M = A.shape
        n = B.shape[1]
    D = torch.empty(M, n, device="cuda", dtype=torch.float32)
    err = torch.zeros(1, device="cuda", dtype=torch.int32)
    N.call("edge_tc_selftest", int(mode), int(n), int(K), ptr_any(A.contiguous(), BF16, "A"),
           ptr_any(B.contiguous(), BF16, "B"), ptr(D), ptr_any(err, I32, "err"), stream())
    torch.cuda.synchronize()
    return D, bool(err.item())


def init_params(seed=0, device="cuda"):
    """He-style initial weights [co][ci][27] (float32) and zero biases."""
    g = torch.Generator().manual_seed(seed)
    p = {}
    for name, co, ci in LAYERS:
        std = (2.0 / (27 * ci)) ** 0.5
        p[name] = (torch.randn(co, ci, 27, generator=g) * std).to(device)
    for name in BIASES:
        p["b" + name[1:]] = torch.zeros(SHAPES[name][0], device=device)
    return p


class Act:
    """One activation tensor of the network (padded chunked bf16)."""

    def __init__(self, res, channels):
        lc = ctypes.c_longlong()
        N.call("edge_unet_geometry", *res, ctypes.byref(lc))
        self.res = tuple(res)
        self.channels = channels
        self.lc = lc.value
        self.t = torch.zeros(channels // 8 * lc.value * 8, dtype=torch.bfloat16, device="cuda")

    @property
    def p(self):
        return ptr_any(self.t, BF16)


# forward activations: name -> (level, channels)
FWD = {"h0": (0, 16), "e0": (0, 16), "d1": (1, 16), "h1": (1, 32), "e1": (1, 32), "d2": (2, 32), "h2": (2, 64),
       "e2": (2, 64), "u1": (1, 64), "h3": (1, 32), "f1": (1, 32), "u0": (0, 32), "h4": (0, 16), "f0": (0, 16)}
# gradient buffers: name -> (level, channels)
BWD = {"g16a": (0, 16), "g16b": (0, 16), "g_u0": (0, 32), "g_e0": (0, 16),
       "g32a": (1, 32), "g32b": (1, 32), "g_u1": (1, 64), "g_e1": (1, 32), "g_d1": (1, 16),
       "g64a": (2, 64), "g64b": (2, 64), "g_d2": (2, 32)}


class UNet:
    """The 3-level U-Net on a grid whose sides are multiples of 4.
    forward(r, z) evaluates it; train_step(r, x, lr) does one Adam step on
    the mean-removed squared error of the scaled prediction against x."""

    def __init__(self, res, params=None, seed=0):
        if any(n % 4 for n in res):
            raise ValueError("grid sides must be multiples of 4")
        self.res = tuple(int(n) for n in res)
        r0 = self.res
        self.lv = (r0, tuple(n // 2 for n in r0), tuple(n // 4 for n in r0))
        self.params = params if params is not None else init_params(seed)
        self.a = {k: Act(self.lv[l], c) for k, (l, c) in FWD.items()}
        self.g = None
        self.scale = torch.zeros(1, device="cuda")
        self.scale_work = torch.zeros(1026, dtype=torch.float64, device="cuda")
        self.err = torch.zeros(1, dtype=torch.int32, device="cuda")
        self.z = torch.zeros(r0, device="cuda")
        self.packed = {}
        self.packed_t = {}
        self.grads = {k: torch.zeros_like(v) for k, v in self.params.items()}
        self.m = {k: torch.zeros_like(v) for k, v in self.params.items()}
        self.v = {k: torch.zeros_like(v) for k, v in self.params.items()}
        self.step_count = 0
        self.pack()

    # ---- parameters ----------------------------------------------------------
    def pack(self):
        """Refresh the bf16 copies of the weights (after an optimiser step)."""
        for name, co, ci in LAYERS:
            w = self.params[name].contiguous()
            if name in TC_LAYERS:
                for tr, dst in ((0, self.packed), (1, self.packed_t)):
                    out = dst.get(name)
                    if out is None:
                        out = dst[name] = torch.empty(co * ci * 27, dtype=torch.bfloat16, device="cuda")
                    N.call("edge_unet_pack_weights", ptr(w), co, ci, tr, ptr_any(out, BF16), stream())
            else:
                self.packed[name] = w.to(torch.bfloat16).float().reshape(-1).contiguous()

    def _conv(self, res, x0, w0, x1, w1, cout, bias, flags, y, table=None):
        table = self.packed if table is None else table
        N.call("edge_unet_conv", *res, x0.p, ptr_any(table[w0], BF16), x0.channels,
               x1.p if x1 else None, ptr_any(table[w1], BF16) if x1 else None, x1.channels if x1 else 0,
               cout, ptr(bias), int(flags), y.p, ptr_any(self.err, I32), stream())

    # ---- forward -------------------------------------------------------------
    def forward(self, r, z=None):
        """z = U-Net(r) for float32 r of the grid's shape (into z or self.z)."""
        z = self.z if z is None else z
        a, p = self.a, self.params
        r0, r1, r2 = self.lv
        N.call("edge_unet_input_scale", ptr(r), ctypes.c_longlong(r.numel()), ptr_any(self.scale_work, F64),
               ptr(self.scale), stream())
        N.call("edge_unet_conv_first", *r0, ptr(r), ptr(self.scale), ptr(self.packed["W0a"]), ptr(p["b0a"]),
               a["h0"].p, stream())
        self._conv(r0, a["h0"], "W0b", None, None, 16, p["b0b"], 1, a["e0"])
        N.call("edge_unet_pool", *r0, 16, a["e0"].p, a["d1"].p, stream())
        self._conv(r1, a["d1"], "W1a", None, None, 32, p["b1a"], 1, a["h1"])
        self._conv(r1, a["h1"], "W1b", None, None, 32, p["b1b"], 1, a["e1"])
        N.call("edge_unet_pool", *r1, 32, a["e1"].p, a["d2"].p, stream())
        self._conv(r2, a["d2"], "W2a", None, None, 64, p["b2a"], 1, a["h2"])
        self._conv(r2, a["h2"], "W2b", None, None, 64, p["b2b"], 1, a["e2"])
        N.call("edge_unet_upsample", *r1, 64, a["e2"].p, a["u1"].p, stream())
        self._conv(r1, a["u1"], "W3a", a["e1"], "W3s", 32, p["b3a"], 1, a["h3"])
        self._conv(r1, a["h3"], "W3b", None, None, 32, p["b3b"], 1, a["f1"])
        N.call("edge_unet_upsample", *r0, 32, a["f1"].p, a["u0"].p, stream())
        self._conv(r0, a["u0"], "W4a", a["e0"], "W4s", 16, p["b4a"], 1, a["h4"])
        self._conv(r0, a["h4"], "W4b", None, None, 16, p["b4b"], 1, a["f0"])
        N.call("edge_unet_conv_last", *r0, a["f0"].p, ptr(self.packed["W5"]), ptr(p["b5"]), ptr(self.scale),
               ptr(z), stream())
        return z

    # ---- backward ------------------------------------------------------------
    def _ensure_bwd(self):
        if self.g is not None:
            return
        self.g = {k: Act(self.lv[l], c) for k, (l, c) in BWD.items()}
        n0 = self.res[0] * self.res[1] * self.res[2]
        self.dzn = torch.zeros(self.res, device="cuda")
        self.stats = torch.zeros(2, dtype=torch.float64, device="cuda")
        self.nsplit = 64
        self.partial = torch.zeros(self.nsplit * 27 * 64 * 64, device="cuda")
        self.nblk = max(1, min(256, n0 // 4096))

    def _wgrad(self, res, d, cout, x, name):
        N.call("edge_unet_wgrad", *res, d.p, cout, x.p, x.channels, ptr(self.partial), self.nsplit,
               ptr(self.grads[name]), ptr_any(self.err, I32), stream())

    def _bias(self, res, d, name):
        N.call("edge_unet_chan_sum", *res, d.channels, d.p, ptr(self.partial), self.nblk,
               ptr(self.grads["b" + name[1:]]), stream())

    def _relu_bwd(self, res, dy, y, out):
        N.call("edge_unet_relu_bwd", *res, dy.channels, dy.p, y.p, out.p, stream())

    def _dgrad(self, res, d, name, out, accumulate=False):
        co, ci = SHAPES[name]
        self._conv(res, d, name, None, None, ci, None, 2 if accumulate else 0, out, table=self.packed_t)

    def backward(self, dzn):
        """Parameter gradients (into self.grads) for dL/dz_n = dzn, z_n the
        network output before the 1/s rescale (the forward pass must have
        run on the same input)."""
        self._ensure_bwd()
        a, g = self.a, self.g
        r0, r1, r2 = self.lv
        # last layer
        N.call("edge_unet_last_bwd", *r0, ptr(dzn), ptr(self.packed["W5"]), a["f0"].p, g["g16a"].p,
               ptr(self.partial), self.nblk, ptr(self.grads["W5"]), stream())
        self.grads["b5"].copy_(dzn.sum().reshape(1))
        # W4b
        self._relu_bwd(r0, g["g16a"], a["f0"], g["g16b"])
        self._wgrad(r0, g["g16b"], 16, a["h4"], "W4b")
        self._bias(r0, g["g16b"], "W4b")
        self._dgrad(r0, g["g16b"], "W4b", g["g16a"])
        # W4a (+ W4s skip)
        self._relu_bwd(r0, g["g16a"], a["h4"], g["g16b"])
        self._wgrad(r0, g["g16b"], 16, a["u0"], "W4a")
        self._wgrad(r0, g["g16b"], 16, a["e0"], "W4s")
        self._bias(r0, g["g16b"], "W4a")
        self._dgrad(r0, g["g16b"], "W4a", g["g_u0"])
        self._dgrad(r0, g["g16b"], "W4s", g["g_e0"])
        N.call("edge_unet_up_bwd", *r0, 32, g["g_u0"].p, g["g32a"].p, stream())
        # W3b
        self._relu_bwd(r1, g["g32a"], a["f1"], g["g32b"])
        self._wgrad(r1, g["g32b"], 32, a["h3"], "W3b")
        self._bias(r1, g["g32b"], "W3b")
        self._dgrad(r1, g["g32b"], "W3b", g["g32a"])
        # W3a (+ W3s skip)
        self._relu_bwd(r1, g["g32a"], a["h3"], g["g32b"])
        self._wgrad(r1, g["g32b"], 32, a["u1"], "W3a")
        self._wgrad(r1, g["g32b"], 32, a["e1"], "W3s")
        self._bias(r1, g["g32b"], "W3a")
        self._dgrad(r1, g["g32b"], "W3a", g["g_u1"])
        self._dgrad(r1, g["g32b"], "W3s", g["g_e1"])
        N.call("edge_unet_up_bwd", *r1, 64, g["g_u1"].p, g["g64a"].p, stream())
        # W2b, W2a
        self._relu_bwd(r2, g["g64a"], a["e2"], g["g64b"])
        self._wgrad(r2, g["g64b"], 64, a["h2"], "W2b")
        self._bias(r2, g["g64b"], "W2b")
        self._dgrad(r2, g["g64b"], "W2b", g["g64a"])
        self._relu_bwd(r2, g["g64a"], a["h2"], g["g64b"])
        self._wgrad(r2, g["g64b"], 64, a["d2"], "W2a")
        self._bias(r2, g["g64b"], "W2a")
        self._dgrad(r2, g["g64b"], "W2a", g["g_d2"])
        N.call("edge_unet_pool_bwd", *r1, 32, g["g_d2"].p, g["g_e1"].p, 1, stream())
        # W1b, W1a
        self._relu_bwd(r1, g["g_e1"], a["e1"], g["g32b"])
        self._wgrad(r1, g["g32b"], 32, a["h1"], "W1b")
        self._bias(r1, g["g32b"], "W1b")
        self._dgrad(r1, g["g32b"], "W1b", g["g32a"])
        self._relu_bwd(r1, g["g32a"], a["h1"], g["g32b"])
        self._wgrad(r1, g["g32b"], 32, a["d1"], "W1a")
        self._bias(r1, g["g32b"], "W1a")
        self._dgrad(r1, g["g32b"], "W1a", g["g_d1"])
        N.call("edge_unet_pool_bwd", *r0, 16, g["g_d1"].p, g["g_e0"].p, 1, stream())
        # W0b, W0a
        self._relu_bwd(r0, g["g_e0"], a["e0"], g["g16b"])
        self._wgrad(r0, g["g16b"], 16, a["h0"], "W0b")
        self._bias(r0, g["g16b"], "W0b")
        self._dgrad(r0, g["g16b"], "W0b", g["g16a"])
        self._relu_bwd(r0, g["g16a"], a["h0"], g["g16b"])
        self._bias(r0, g["g16b"], "W0a")
        self._rfirst_bwd(g["g16b"])
        return self.grads

    def _rfirst_bwd(self, d):
        N.call("edge_unet_first_bwd", *self.res, d.p, ptr(self._r), ptr(self.scale), ptr(self.partial), self.nblk,
               ptr(self.grads["W0a"]), stream())

    # ---- training ------------------------------------------------------------
    def loss_and_grad(self, r, x):
        """Forward on r, loss against the solution x (both float32, grid
        shaped) and gradients; returns the loss as a device scalar."""
        self._ensure_bwd()
        self._r = r
        self.forward(r, self.z)
        N.call("edge_unet_loss", ptr(self.z), ptr(x), ptr(self.scale), ctypes.c_longlong(x.numel()),
               ptr_any(self.stats, F64), ptr(self.dzn), stream())
        self.backward(self.dzn)
        return self.stats[1]

    def adam_step(self, lr=1e-3, b1=0.9, b2=0.999, eps=1e-8):
        self.step_count += 1
        for k, p in self.params.items():
            N.call("edge_unet_adam", ctypes.c_longlong(p.numel()), ptr(p), ptr(self.grads[k]), ptr(self.m[k]),
                   ptr(self.v[k]), ctypes.c_float(lr), ctypes.c_float(b1), ctypes.c_float(b2), ctypes.c_float(eps),
                   self.step_count, stream())
        self.pack()

    def train_step(self, r, x, lr=1e-3):
        loss = self.loss_and_grad(r, x)
        self.adam_step(lr)
        return loss

    def timed_out(self):
        return bool(self.err.item())


def act_to_dense(act):
    """(C, X, Y, Z) float32 copy of an activation tensor (tests, debugging)."""
    X, Y, Z = act.res
    G = (Y + 2) * (Z + 2) + (Z + 2) + 2
    v = act.t.view(act.channels // 8, act.lc, 8)[:, G:G + (X + 2) * (Y + 2) * (Z + 2), :]
    v = v.reshape(act.channels // 8, X + 2, Y + 2, Z + 2, 8)[:, 1:-1, 1:-1, 1:-1, :]
    return v.permute(0, 4, 1, 2, 3).reshape(act.channels, X, Y, Z).float()


def dense_to_act(x, act):
    """Write a (C, X, Y, Z) tensor into an activation tensor (bf16-rounded)."""
    X, Y, Z = act.res
    G = (Y + 2) * (Z + 2) + (Z + 2) + 2
    v = act.t.view(act.channels // 8, act.lc, 8)[:, G:G + (X + 2) * (Y + 2) * (Z + 2), :]
    v = v.view(act.channels // 8, X + 2, Y + 2, Z + 2, 8)
    v[:, 1:-1, 1:-1, 1:-1, :] = x.reshape(act.channels // 8, 8, X, Y, Z).permute(0, 2, 3, 4, 1).to(torch.bfloat16)


# ---- flexible CG with the learned preconditioner ------------------------------
class LearnedPCG:
    """Flexible preconditioned CG (Polak-Ribiere beta, so a nonlinear
    preconditioner is admissible) for the all-Neumann pressure Poisson
    problem A x = b of a Projection, preconditioned by

        mode "warm":    z = N(r) + V(r - A N(r))  (the MGPCG V-cycle warm-started
                        from the network's guess, i.e. one V-cycle from z0 = N(r))
        mode "net":     z = N(r)
        mode "vcycle":  z = V(r)  (plain MGPCG, the fallback)

    The learned modes fall back to the plain V-cycle for the rest of the
    solve when an iteration reduces |r| by less than `stall` (the residual
    stalls).  Dot products and norms are float64; vectors float32.  The
    network and V-cycle are the library's kernels; the vector updates are
    torch tensor operations."""

    def __init__(self, proj, net, stall=0.7):
        self.P = proj
        self.net = net
        self.stall = stall
        res = proj.res
        self.z0 = torch.zeros(res, device="cuda")
        self.t = torch.zeros(res, device="cuda")
        self.v = torch.zeros(res, device="cuda")

    def precond(self, r, z, mode):
        if mode == "vcycle":
            self.P.vcycle(r, z)
        elif mode == "net":
            self.net.forward(r, z)
        else:
            self.net.forward(r, self.z0)
            self.P.apply_A(self.z0, self.t)
            torch.sub(r, self.t, out=self.t)
            self.P.vcycle(self.t, self.v)
            torch.add(self.z0, self.v, out=z)
        z -= z.mean()

    def solve(self, b, x, rel_tol=1e-6, max_iters=200, mode="warm", record=None):
        """x (zeroed here) solves A x = b - mean(b) to ||r|| <= rel_tol ||b||.
        Returns (iterations, final relative residual, fell_back).  With a
        list `record`, (r_k, x_k) of every iterate is appended to it (training
        pairs: the correction of r_k is x_final - x_k)."""
        r = b - b.mean()
        x.zero_()
        bn = float(torch.linalg.vector_norm(r.double()))
        if bn == 0.0:
            return 0, 0.0, False
        z = torch.empty_like(r)
        Ap = torch.empty_like(r)
        fell_back = False
        self.precond(r, z, mode)
        p = z.clone()
        rz = float(torch.dot(r.double().view(-1), z.double().view(-1)))
        rn = bn
        it = 0
        while it < max_iters:
            if record is not None:
                record.append((r.clone(), x.clone()))
            self.P.apply_A(p, Ap)
            pAp = float(torch.dot(p.double().view(-1), Ap.double().view(-1)))
            if pAp <= 0.0:
                break
            alpha = rz / pAp
            x.add_(p, alpha=alpha)
            r_old = r.clone()
            r.sub_(Ap, alpha=alpha)
            r -= r.mean()
            it += 1
            rn_new = float(torch.linalg.vector_norm(r.double()))
            if rn_new <= rel_tol * bn:
                rn = rn_new
                break
            if mode != "vcycle" and rn_new > self.stall * rn:
                mode, fell_back = "vcycle", True
            rn = rn_new
            self.precond(r, z, mode)
            beta = float(torch.dot(z.double().view(-1), (r - r_old).double().view(-1))) / rz
            rz = float(torch.dot(r.double().view(-1), z.double().view(-1)))
            p.mul_(beta).add_(z)
        return it, rn / bn, fell_back


def mgpcg_pairs(sim, steps, every=1):
    """(r, x) training pairs from a running EdgeSim: after each projection the
    solver's right-hand side r = -div u and its pressure solution x (A x = r)."""
    out = []
    for s in range(steps):
        sim.step()
        if s % every == 0:
            div = sim.proj.get("div")
            x = sim.proj.get("p")
            out.append(((-div).contiguous(), x.contiguous()))
    return out


# ---- learned coarse-grid solver inside MGPCG -----------------------------------
class LearnedCoarsePCG:
    """MGPCG whose coarse group is the U-Net.  The V-cycle's coarsest levels
    (lc..L-1, which the solver otherwise runs in one shared-memory block) solve
    the level-lc residual equation A_lc z = r_lc approximately; here the
    network, trained on exact solutions of that equation, supplies z_lc, and
    everything else (the finer levels' sweeps, restrictions and
    prolongations, the CG updates with their device-side scalars) is the
    plain solver's cooperative iteration kernel.  The network works at the
    coarse level's size (32x16x16 for the 128x64x64 and 256x128x128 grids),
    a few hundred times fewer voxels than the fine grid.

    Fallback: when an iteration reduces |r| by less than `stall`, the rest of
    the solve takes the built-in coarse group (plain MGPCG), the CG recursion
    restarted (p = z) from the current iterate.  One iteration
    (coarse step + CG iteration) is a CUDA graph replayed per iteration; the
    host reads the status (and r.r for the stall test) between iterations."""

    def __init__(self, proj, params, stall=0.5, graphs=True):
        self.P = proj
        self.level, self.dims = proj.coarse_shape()
        self.net = UNet(self.dims, params=params)
        self.r = torch.zeros(self.dims, device="cuda")
        self.z = torch.zeros(self.dims, device="cuda")
        self.stall = float(stall)
        self.graphs = {}
        self.use_graphs = bool(graphs)
        self.fell_back = False

    def _step(self, mode):
        if mode == "net":
            self.P.coarse_get_r(self.r)
            self.net.forward(self.r, self.z)
            self.P.coarse_set_z(self.z)
        elif mode == "exact":
            # the coarse-level equation solved to 1e-7 (the best any coarse
            # solver can do; for measurement, not speed)
            self.P.coarse_get_r(self.r)
            self.exact_solver().solve(self.r, self.z, abs_tol=0.0, rel_tol=1e-14, max_iters=400)
            self.P.coarse_set_z(self.z)
        else:
            self.P.coarse_default()
        self.P.solve_iter()

    def exact_solver(self):
        if getattr(self, "_exact", None) is None:
            import math
            from .projection import Projection
            lg = int(math.log2(min(self.dims)))
            self._exact = Projection(self.dims, base_level=max(1, lg - 2))
        return self._exact

    def _run(self, mode):
        if not self.use_graphs or mode == "exact":
            self._step(mode)
            return
        g = self.graphs.get(mode)
        if g is None:
            # capture after the buffers exist; a launch that cannot be captured
            # leaves the eager path in place
            try:
                g = torch.cuda.CUDAGraph()
                s = torch.cuda.Stream()
                s.wait_stream(torch.cuda.current_stream())
                with torch.cuda.stream(s):
                    g.capture_begin()
                    self._step(mode)
                    g.capture_end()
                torch.cuda.current_stream().wait_stream(s)
                self.graphs[mode] = g
            except RuntimeError:
                self.use_graphs = False
                self._step(mode)
                return
        g.replay()

    def poisson(self, u_x, u_y, u_z, f=None, abs_tol=1e-12, rel_tol=1e-12, max_iters=-1, mode="net"):
        """The projection (Projection.poisson's arguments and effect) with the
        learned coarse solver."""
        self.P.poisson_begin(u_x, u_y, u_z, abs_tol=abs_tol, rel_tol=rel_tol, max_iters=max_iters)
        fell = self._loop(mode)
        self.P.poisson_end(u_x, u_y, u_z, f)
        self.fell_back = fell

    def solve(self, b, x, abs_tol=1e-12, rel_tol=1e-12, max_iters=400, mode="net"):
        """x solves A x = b (the solver's tolerance semantics, mgpcg.py:224).
        Returns (iterations, r.r, status, fell_back)."""
        P = self.P
        P.solve_begin(b, abs_tol=abs_tol, rel_tol=rel_tol, max_iters=max_iters)
        fell_back = self._loop(mode)
        P.solve_end(b, x)
        it, rtr, st = P.result()
        return it, rtr, st, fell_back

    def _loop(self, mode):
        P = self.P
        fell_back = False
        prev = None
        while True:
            self._run(mode)
            it, rtr, running = P.progress()
            if not running:
                break
            if mode == "net" and prev is not None and rtr > self.stall * self.stall * prev:
                # the built-in coarse group from here on, the recursion
                # restarted from the current iterate (p = z)
                mode, fell_back = "vcycle", True
                P.restart()
            prev = rtr
        return fell_back
