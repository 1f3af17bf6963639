"""torch-level wrappers of the C ABI entry points (one per kernel family).

Every function takes torch CUDA tensors in the reference's layout, launches on
the current stream and returns nothing (outputs are written into the given
tensors) unless stated.  Shapes are checked here; the library re-checks sizes
and pointers.
"""
import ctypes

import torch

from . import _native as N
from .fields import NULL, cell_dims, dims_from_faces, ptr, stream

F = ctypes.c_float

# kernels each entry point launches (memcpy/memset nodes are not counted)
_KERNELS = {"edge_max_speed": 2, "edge_copy": 0, "edge_lp_max_speed": 2, "edge_march_ge": 3,
            "edge_march_ge_packed": 3, "edge_calc_fd_3_from_grad": 2, "edge_face_map_packed": 3}
_launched = [0]


def _call(name, *args):
    N.call(name, *args)
    _launched[0] += _KERNELS.get(name, 1)


def launch_count():
    """Kernels of libedgeb200.so launched so far by this process: the direct
    entry points plus what every live MGPCG solver counted on the device
    (synchronises)."""
    from .projection import live_solvers
    return _launched[0] + sum(p.kernel_count() for p in live_solvers())


def _p3(ts):
    return [ptr(t) for t in ts] if ts is not None else [NULL, NULL, NULL]


# ---- point samplers ---------------------------------------------------------
def points_mac(u, dx, pts):
    nx, ny, nz = dims_from_faces(*u)
    n = pts.shape[0]
    v = torch.empty((n, 3), device=pts.device)
    vg = torch.empty((n, 3), device=pts.device)
    g = torch.empty((n, 3, 3), device=pts.device)
    _call("edge_points_mac", nx, ny, nz, F(dx), *_p3(u), ptr(pts), n, ptr(v), ptr(vg), ptr(g), stream())
    return v, vg, g


def points_dye(smoke, dx, pts):
    nx, ny, nz = cell_dims(smoke)
    n = pts.shape[0]
    out = [torch.empty((n, 4), device=pts.device) for _ in range(3)]
    _call("edge_points_dye", nx, ny, nz, F(dx), ptr(smoke), ptr(pts), n, *[ptr(o) for o in out], stream())
    return out


def points_hermite(variant, psi, T, dT, d2T, dx, pts):
    nx, ny, nz = cell_dims(psi)
    n = pts.shape[0]
    val = torch.empty((n, 3), device=pts.device)
    gval = torch.empty((n, 3), device=pts.device)
    grad = torch.empty((n, 3, 3), device=pts.device)
    _call("edge_points_hermite", variant, nx, ny, nz, F(dx), ptr(psi), *_p3(T), *_p3(dT), *_p3(d2T), ptr(pts), n,
           ptr(val), ptr(gval), ptr(grad), stream())
    return val, gval, grad


# ---- map state ----------------------------------------------------------------
def reset_cells(dx, psi, T, dT=None, d2T=None):
    nx, ny, nz = cell_dims(psi)
    _call("edge_reset_cells", nx, ny, nz, F(dx), ptr(psi), *_p3(T), *_p3(dT), *_p3(d2T), stream())


def reset_faces(res, dx, phi, Fm):
    _call("edge_reset_faces", *res, F(dx), *_p3(phi), *_p3(Fm), stream())


def march_edge(u, dx, dt, eps, psi, T, dT, opsi, oT, odT, identity=False):
    nx, ny, nz = cell_dims(opsi)
    _call("edge_march_edge", nx, ny, nz, F(dx), F(dt), F(eps), *_p3(u), ptr(psi), *_p3(T), *_p3(dT), ptr(opsi),
           *_p3(oT), *_p3(odT), int(bool(identity)), stream())


def march_ed4(u, dx, dt, eps, psi, T, opsi, oT):
    nx, ny, nz = cell_dims(opsi)
    _call("edge_march_ed4", nx, ny, nz, F(dx), F(dt), F(eps), *_p3(u), ptr(psi), *_p3(T), ptr(opsi), *_p3(oT),
           stream())


def march_ed8(u, dx, dt, eps, psi, T, dT, d2T, opsi, oT, odT, od2T):
    nx, ny, nz = cell_dims(opsi)
    _call("edge_march_ed8", nx, ny, nz, F(dx), F(dt), F(eps), *_p3(u), ptr(psi), *_p3(T), *_p3(dT), *_p3(d2T),
           ptr(opsi), *_p3(oT), *_p3(odT), *_p3(od2T), stream())


def march_ge(u, dx, dt, psi, T, dT, d2T, opsi, oT, odT, od2T):
    nx, ny, nz = cell_dims(opsi)
    _call("edge_march_ge", nx, ny, nz, F(dx), F(dt), *_p3(u), ptr(psi), *_p3(T), *_p3(dT), *_p3(d2T), ptr(opsi),
          *_p3(oT), *_p3(odT), *_p3(od2T), stream())


def calc_fd_3_from_grad(dx, T, dT, d2T):
    nx, ny, nz = cell_dims(T[0])
    _call("edge_calc_fd_3_from_grad", nx, ny, nz, F(dx), *_p3(T), *_p3(dT), *_p3(d2T), stream())


PLANES = {0: 8, 1: 8, 2: 8}  # packed float4 planes per Hermite variant (edge_packed_planes)


def map_pack(variant, psi, T, dT, d2T, packed):
    nx, ny, nz = cell_dims(psi)
    _check_packed(variant, packed, (nx, ny, nz))
    _call("edge_map_pack", variant, nx, ny, nz, ptr(psi), *_p3(T), *_p3(dT), *_p3(d2T), ptr(packed), stream())
    _launched[0] += variant != 2  # the derived-plane pass of ED4 / EDGE maps


def _check_packed(variant, packed, res):
    want = (N.load().edge_packed_planes(variant),) + tuple(res) + (4,)
    if tuple(packed.shape) != want or packed.dtype != torch.float32 or not packed.is_contiguous():
        raise ValueError(f"packed map must be a contiguous float32 tensor of shape {want}")


def map_unpack(variant, packed, psi, T, dT, d2T):
    nx, ny, nz = cell_dims(psi)
    _call("edge_map_unpack", variant, nx, ny, nz, ptr(packed), ptr(psi), *_p3(T), *_p3(dT), *_p3(d2T), stream())


def march_packed(variant, u, dx, dt, eps, packed_in, packed_out, res, identity=False, f64_compose=False):
    """f64_compose: accumulate the composed Jacobian in float64 (EDGE)."""
    _check_packed(variant, packed_out, res)
    flags = (1 if identity else 0) | (2 if f64_compose else 0)
    _call("edge_march_packed", variant, *res, F(dx), F(dt), F(eps), *_p3(u), ptr(packed_in), ptr(packed_out),
          flags, stream())
    _launched[0] += variant != 2


def march_ge_packed(u, dx, dt, packed_in, packed_out, res):
    _call("edge_march_ge_packed", *res, F(dx), F(dt), *_p3(u), ptr(packed_in), ptr(packed_out), stream())


def face_map_packed(variant, dx, packed, res, fpsi, fcol):
    _call("edge_face_map_packed", variant, *res, F(dx), ptr(packed), *_p3(fpsi), *_p3(fcol), stream())


def face_map(variant, dx, psi, T, dT, d2T, fpsi, fcol):
    nx, ny, nz = cell_dims(psi)
    _call("edge_face_map", variant, nx, ny, nz, F(dx), ptr(psi), *_p3(T), *_p3(dT), *_p3(d2T), *_p3(fpsi),
           *_p3(fcol), stream())


def efm_backtrack(u_cache, dts, dx, psi, T):
    """Backward face map of the EFM driver through the cached velocities
    u_cache[0..j] (slot j = the current velocity) with step sizes dts[0..j]."""
    n = len(u_cache)
    nx, ny, nz = dims_from_faces(*u_cache[0])
    arrs = [(ctypes.c_void_p * n)(*[ptr(u[a]) for u in u_cache]) for a in range(3)]
    d = (ctypes.c_float * n)(*[float(x) for x in dts])
    _call("edge_efm_backtrack", nx, ny, nz, F(dx), n - 1, *[ctypes.addressof(a) for a in arrs], ctypes.addressof(d),
          *_p3(psi), *_p3(T), stream())


def advance_map(u, dx, dt, phi, Fm):
    nx, ny, nz = dims_from_faces(*u)
    _call("edge_advance_map", nx, ny, nz, F(dx), F(dt), *_p3(u), *_p3(phi), *_p3(Fm), stream())


# ---- transport ----------------------------------------------------------------
def advect_u_sl(u0, dx, dt, u1):
    nx, ny, nz = dims_from_faces(*u0)
    _call("edge_advect_u_sl", nx, ny, nz, F(dx), F(dt), *_p3(u0), *_p3(u1), stream())


def pullback_u(u0, dx, pos, col, out, init=None, scale=1.0, sub=None):
    nx, ny, nz = dims_from_faces(*u0)
    _call("edge_pullback_u", nx, ny, nz, F(dx), *_p3(u0), *_p3(pos), *_p3(col), *_p3(init), F(scale), *_p3(sub),
           *_p3(out), stream())


def map_u_psi(variant, u0, out, dx, psi, T, dT):
    nx, ny, nz = cell_dims(psi)
    _call("edge_map_u_psi", variant, nx, ny, nz, F(dx), *_p3(u0), *_p3(out), ptr(psi), *_p3(T), *_p3(dT), stream())


def pullback_dye(smoke0, dx, pos, out, init=None, scale=1.0, sub=None, clampsrc=None, inplace_clamp=False):
    nx, ny, nz = cell_dims(out)
    _call("edge_pullback_dye", nx, ny, nz, F(dx), ptr(smoke0), *_p3(pos), ptr(init), F(scale), ptr(sub),
           ptr(clampsrc), int(bool(inplace_clamp)), ptr(out), stream())


def smoke_psi(variant, mode, smoke0, out, dx, psi, T, dT):
    nx, ny, nz = cell_dims(psi)
    _call("edge_smoke_psi", variant, mode, nx, ny, nz, F(dx), ptr(smoke0), ptr(out), ptr(psi), *_p3(T), *_p3(dT),
           stream())


def clamp_u(u, u1, u2):
    nx, ny, nz = dims_from_faces(*u)
    _call("edge_clamp_u", nx, ny, nz, *_p3(u), *_p3(u1), *_p3(u2), stream())


def max_speed(u, out):
    nx, ny, nz = dims_from_faces(*u)
    _call("edge_max_speed", nx, ny, nz, *_p3(u), ptr(out), stream())


def axpy(f1, f2, a, dest):
    _call("edge_axpy", ctypes.c_longlong(dest.numel()), ptr(f1), ptr(f2), F(a), ptr(dest), stream())


def copy(src, dst):
    if src.numel() != dst.numel():
        raise ValueError("copy: size mismatch")
    _call("edge_copy", ctypes.c_longlong(dst.numel()), ptr(src), ptr(dst), stream())


# ---- initial conditions ----------------------------------------------------------
def add_vortex_ring(dx, w, rad, delta, c, ex, ey, u, smoke, color, num_samples):
    nx, ny, nz = cell_dims(u)
    f3 = lambda v: (ctypes.c_float * 3)(*[float(a) for a in v])  # noqa: E731
    _call("edge_add_vortex_ring", nx, ny, nz, F(dx), F(w), F(rad), F(delta), f3(c), f3(ex), f3(ey), ptr(u),
           ptr(smoke), f3(color), int(num_samples), stream())


def emit_smoke(dx, centers, colors, radius, smoke):
    nx, ny, nz = cell_dims(smoke)
    k = len(centers)
    c = (ctypes.c_float * (3 * k))(*[float(v) for p in centers for v in p])
    col = (ctypes.c_float * (4 * k))(*[float(v) for p in colors for v in p])
    _call("edge_emit_smoke", nx, ny, nz, F(dx), c, col, k, F(radius), ptr(smoke), stream())


def clamp_max(x, hi):
    _call("edge_clamp_max", ctypes.c_longlong(x.numel()), F(hi), ptr(x), stream())


def split_central_vector(vc, u):
    nx, ny, nz = cell_dims(vc)
    _call("edge_split_central_vector", nx, ny, nz, ptr(vc), *_p3(u), stream())


def get_central_vector(u, vc):
    nx, ny, nz = cell_dims(vc)
    _call("edge_get_central_vector", nx, ny, nz, *_p3(u), ptr(vc), stream())


def curl(vf, cf, dx):
    nx, ny, nz = cell_dims(vf)
    _call("edge_curl", nx, ny, nz, F(dx), ptr(vf), ptr(cf), stream())


# ---- particles ----------------------------------------------------------------
def lp_acc(u, dx, vel, pos, acc, num, dt, St, gravity):
    nx, ny, nz = dims_from_faces(*u)
    _call("edge_lp_acc", nx, ny, nz, F(dx), *_p3(u), ptr(vel), ptr(pos), ptr(acc), int(num), int(acc.shape[0]),
           F(dt), F(St), F(gravity), stream())


def lp_velocity(acc, vel, pos, dt, dx, num, L):
    _call("edge_lp_velocity", ptr(acc), ptr(vel), ptr(pos), F(dt), F(dx), int(num), *[F(v) for v in L], stream())


def lp_vel_diff(u, dx, vel, vdiff, pos, num, St, density_ratio, epiral_radius_ratio):
    nx, ny, nz = dims_from_faces(*u)
    _call("edge_lp_vel_diff", nx, ny, nz, F(dx), *_p3(u), ptr(vel), ptr(vdiff), ptr(pos), int(num), F(St),
           F(density_ratio), F(epiral_radius_ratio), stream())


def lp_p2g(res, dx, drag, vdiff, pos, rad, num, laden_radius, L):
    _call("edge_lp_p2g", *res, F(dx), *_p3(drag), ptr(vdiff), ptr(pos), ptr(rad), int(num), F(laden_radius),
           *[F(v) for v in L], stream())


def lp_max_speed(vel, num, out):
    _call("edge_lp_max_speed", ptr(vel), int(num), ptr(out), stream())


def lp_position(vel, pos, dt, num, L):
    _call("edge_lp_position", ptr(vel), ptr(pos), F(dt), int(num), *[F(v) for v in L], stream())


def lp_viscous(u, dx, Re, vis):
    nx, ny, nz = dims_from_faces(*u)
    _call("edge_lp_viscous", nx, ny, nz, F(dx), F(Re), *_p3(u), *_p3(vis), stream())


# ---- measurement ------------------------------------------------------------------
def fma_peak_tflops(iters=2048, reps=3):
    """FP32 FMA throughput of the current GPU in TFLOP/s (best of `reps`
    launches of 8 resident blocks per SM, timed with CUDA events)."""
    dev = torch.cuda.current_device()
    blocks = 8 * torch.cuda.get_device_properties(dev).multi_processor_count
    out = torch.zeros(1, device="cuda")
    flops = ctypes.c_double()
    _call("edge_fma_peak", blocks, iters, ptr(out), ctypes.byref(flops), stream())  # warm-up
    best = 0.0
    for _ in range(reps):
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record()
        _call("edge_fma_peak", blocks, iters, ptr(out), ctypes.byref(flops), stream())
        e1.record()
        torch.cuda.synchronize()
        best = max(best, flops.value / (e0.elapsed_time(e1) * 1e-3) / 1e12)
    return best
