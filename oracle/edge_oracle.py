"""ctypes front end of the C restatement oracle (``edge_oracle.c``).

TEST INFRASTRUCTURE ONLY — the checker for the CUDA library and the timed
CPU baseline.  Only ``tests/``, ``__graft_entry__.smoke()`` and the CPU legs of
``bench.py`` import this module; the product never does.

All arrays are numpy float32 in the reference's index order (z fastest, vector
components last, as Taichi's ``to_numpy()`` returns them).  Functions that
update fields in place in the reference do the same here.  Every function
names the reference lines it restates.
"""
import ctypes
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_SO = os.path.join(_HERE, "_build", "libedge_oracle.so")
_SO_FMA = os.path.join(_HERE, "_build", "libedge_oracle_fma.so")
_libs = {}
_variant = ["plain"]

F32 = np.float32


def build():
    """Compile the oracle with its Makefile (plain gcc + OpenMP)."""
    subprocess.run(["make", "-s", "-C", _HERE], check=True)


def lib():
    v = _variant[0]
    if v not in _libs:
        # spinning OpenMP barriers collapse when any core is busy (a torch or
        # driver thread); the multigrid's many short parallel loops need
        # blocking waits unless the caller chose otherwise
        os.environ.setdefault("OMP_WAIT_POLICY", "PASSIVE")
        so = _SO_FMA if v == "fma" else _SO
        if not os.path.exists(so) or os.path.getmtime(so) < os.path.getmtime(os.path.join(_HERE, "edge_oracle.c")):
            build()
        L = ctypes.CDLL(so)
        L.orc_calc_max_speed.restype = ctypes.c_float
        for name in ("orc_poisson", "orc_poisson_solid", "orc_vcycle"):
            getattr(L, name).restype = ctypes.c_int
        _libs[v] = L
    return _libs[v]


class fma_twin:
    """Context manager: oracle calls inside it run the fused-multiply-add
    build of the same source (libedge_oracle_fma.so), a second float32
    evaluation of the reference arithmetic that differs only in rounding."""

    def __enter__(self):
        self._prev = _variant[0]
        _variant[0] = "fma"
        return self

    def __exit__(self, *exc):
        _variant[0] = self._prev
        return False


def _p(a):
    if a is None:
        return None
    assert a.flags.c_contiguous, "oracle arrays must be C-contiguous"
    return a.ctypes.data_as(ctypes.c_void_p)


def _f(x):
    return ctypes.c_float(float(x))


def _i(x):
    return ctypes.c_int(int(x))


def _c32(a):
    return np.ascontiguousarray(a, dtype=F32)


# ----------------------------------------------------------------------------
# fields
# ----------------------------------------------------------------------------
def face_shapes(res):
    nx, ny, nz = res
    return [(nx + 1, ny, nz), (nx, ny + 1, nz), (nx, ny, nz + 1)]


def center_coords(res, dx):
    """taichi_utils.py:23-26 center_coords_func."""
    idx = np.indices(res).astype(F32)
    return np.ascontiguousarray(np.stack([(idx[c] + F32(0.5)) * F32(dx) for c in range(3)], -1))


def face_coords(res, dx, axis):
    """taichi_utils.py:29-44 x/y/z_coords_func."""
    shp = face_shapes(res)[axis]
    idx = np.indices(shp).astype(F32)
    return np.ascontiguousarray(np.stack(
        [(idx[c] + (F32(0.0) if c == axis else F32(0.5))) * F32(dx) for c in range(3)], -1))


# ----------------------------------------------------------------------------
# point samplers (golden tests)
# ----------------------------------------------------------------------------
def points_mac(u, dx, pts):
    ux, uy, uz = (_c32(a) for a in u)
    nx, ny, nz = uy.shape[0], ux.shape[1], ux.shape[2]
    pts = _c32(pts)
    n = pts.shape[0]
    v = np.zeros((n, 3), F32)
    vg = np.zeros((n, 3), F32)
    g = np.zeros((n, 3, 3), F32)
    lib().orc_points_mac(_i(nx), _i(ny), _i(nz), _f(dx), _p(ux), _p(uy), _p(uz), _p(pts), _i(n), _p(v), _p(vg), _p(g))
    return v, vg, g


def points_dye(smoke, dx, pts):
    smoke = _c32(smoke)
    pts = _c32(pts)
    n = pts.shape[0]
    lin, mn, mx = (np.zeros((n, 4), F32) for _ in range(3))
    lib().orc_points_dye(*(_i(s) for s in smoke.shape[:3]), _f(dx), _p(smoke), _p(pts), _i(n), _p(lin), _p(mn), _p(mx))
    return lin, mn, mx


HV_FD, HV_GARM, HV_FULL = 0, 1, 2


def points_hermite(variant, psi, T, dT, d2T, dx, pts):
    psi = _c32(psi)
    T = [_c32(t) for t in T]
    dT = [_c32(t) for t in dT] if dT is not None else [None] * 3
    d2T = [_c32(t) for t in d2T] if d2T is not None else [None] * 3
    pts = _c32(pts)
    n = pts.shape[0]
    val, gval = np.zeros((n, 3), F32), np.zeros((n, 3), F32)
    grad = np.zeros((n, 3, 3), F32)
    lib().orc_points_hermite(_i(variant), *(_i(s) for s in psi.shape[:3]), _f(dx), _p(psi), *(_p(t) for t in T),
                             *(_p(t) for t in dT), *(_p(t) for t in d2T), _p(pts), _i(n), _p(val), _p(gval), _p(grad))
    return val, gval, grad


# ----------------------------------------------------------------------------
# marches (return new arrays; inputs untouched)
# ----------------------------------------------------------------------------
def march_edge(u, psi, T, dT, dx, dt, eps):
    """hermite.py:1426-1521 advect_psi_garm_ed4_fusion_unroll."""
    u = [_c32(a) for a in u]
    res = psi.shape[:3]
    o = [np.empty(res + (3,), F32) for _ in range(7)]
    lib().orc_march_edge(*(_i(s) for s in res), _f(dx), _f(dt), _f(eps), *(_p(a) for a in u), _p(_c32(psi)),
                         *(_p(_c32(t)) for t in T), *(_p(_c32(t)) for t in dT), *(_p(a) for a in o))
    return o[0], o[1:4], o[4:7]


def march_ed4(u, psi, T, dx, dt, eps):
    """hermite.py:1375-1395 advect_ps_hermite_ed4_fd_unroll."""
    u = [_c32(a) for a in u]
    res = psi.shape[:3]
    o = [np.empty(res + (3,), F32) for _ in range(4)]
    lib().orc_march_ed4(*(_i(s) for s in res), _f(dx), _f(dt), _f(eps), *(_p(a) for a in u), _p(_c32(psi)),
                        *(_p(_c32(t)) for t in T), *(_p(a) for a in o))
    return o[0], o[1:4]


def march_ed8(u, psi, T, dT, d2T, dx, dt, eps):
    """hermite.py:1290-1338 advect_ps_hermite_ed8."""
    u = [_c32(a) for a in u]
    res = psi.shape[:3]
    o = [np.empty(res + (3,), F32) for _ in range(7)] + [np.empty(res, F32) for _ in range(3)]
    lib().orc_march_ed8(*(_i(s) for s in res), _f(dx), _f(dt), _f(eps), *(_p(a) for a in u), _p(_c32(psi)),
                        *(_p(_c32(t)) for t in T), *(_p(_c32(t)) for t in dT), *(_p(_c32(t)) for t in d2T),
                        *(_p(a) for a in o))
    return o[0], o[1:4], o[4:7], o[7:10]


def calc_fd_3_from_grad(T, dx):
    """hermite.py:1180-1256 -> (dT, d2T) from the gradient rows T."""
    res = T[0].shape[:3]
    dT = [np.empty(res + (3,), F32) for _ in range(3)]
    d2T = [np.empty(res, F32) for _ in range(3)]
    lib().orc_calc_fd_3_from_grad(*(_i(s) for s in res), _f(dx), *(_p(_c32(t)) for t in T), *(_p(a) for a in dT),
                                  *(_p(a) for a in d2T))
    return dT, d2T


def march_ge(u, psi, T, dT, d2T, dx, dt):
    """hermite.py:1398-1424 advect_ps_garm (GE)."""
    u = [_c32(a) for a in u]
    res = psi.shape[:3]
    o = [np.empty(res + (3,), F32) for _ in range(7)] + [np.empty(res, F32) for _ in range(3)]
    lib().orc_march_ge(*(_i(s) for s in res), _f(dx), _f(dt), *(_p(a) for a in u), _p(_c32(psi)),
                       *(_p(_c32(t)) for t in T), *(_p(_c32(t)) for t in dT), *(_p(_c32(t)) for t in d2T),
                       *(_p(a) for a in o))
    return o[0], o[1:4], o[4:7], o[7:10]


def split_psi_hermite(psi, T, dT, d2T, dx):
    """run_ed8.py:191-224 split_psi_hermite -> (psi_faces, T_faces)."""
    res = psi.shape[:3]
    pf = [np.empty(s + (3,), F32) for s in face_shapes(res)]
    tf = [np.empty(s + (3,), F32) for s in face_shapes(res)]
    lib().orc_split_psi_hermite(*(_i(s) for s in res), _f(dx), _p(_c32(psi)), *(_p(_c32(t)) for t in T),
                                *(_p(_c32(t)) for t in dT), *(_p(_c32(t)) for t in d2T),
                                *(_p(a) for a in pf), *(_p(a) for a in tf))
    return pf, tf


# ----------------------------------------------------------------------------
# face / cell step kernels
# ----------------------------------------------------------------------------
def _res_from_u(u):
    return (u[1].shape[0], u[0].shape[1], u[0].shape[2])


def advect_u_semi_lagrangian(u, dx, dt):
    """hermite.py:1578-1621 (dt as passed by the caller)."""
    u = [_c32(a) for a in u]
    res = _res_from_u(u)
    out = [np.empty_like(a) for a in u]
    lib().orc_advect_u_semi_lagrangian(*(_i(s) for s in res), _f(dx), _f(dt), *(_p(a) for a in u),
                                       *(_p(a) for a in out))
    return out


def advance_map(u, phi, F, axis, dx, dt):
    """run_edge.py:337-357 advance_map (in place on phi, F)."""
    u = [_c32(a) for a in u]
    res = _res_from_u(u)
    lib().orc_advance_map(*(_i(s) for s in res), _i(axis), _f(dx), _f(dt), *(_p(a) for a in u), _p(phi), _p(F))


def efm_backtrack(u_cache, dts, dx):
    """run_efm.py:179-186 backtrack_psi_grid(len(u_cache) - 1): the face map
    reset to the identity, then advance_map with -dts[s] through the cached
    velocities, newest first.  Returns (psi_faces, T_faces)."""
    res = _res_from_u(u_cache[0])
    psi = [face_coords(res, dx, a).astype(F32) for a in range(3)]
    T = [np.broadcast_to(np.eye(3, dtype=F32)[a], s + (3,)).copy() for a, s in enumerate(face_shapes(res))]
    for s in reversed(range(len(u_cache))):
        for a in range(3):
            advance_map(u_cache[s], psi[a], T[a], a, dx, -F32(dts[s]))
    return psi, T


def map_u(u0, F, phi, dx):
    """run_edge.py:361-373 map_u."""
    u0 = [_c32(a) for a in u0]
    res = _res_from_u(u0)
    out = [np.empty_like(a) for a in u0]
    lib().orc_map_u(*(_i(s) for s in res), _f(dx), *(_p(a) for a in u0), *(_p(a) for a in out),
                    *(_p(_c32(a)) for a in F), *(_p(_c32(a)) for a in phi))
    return out


def map_u_psi(variant, u0, psi, T, dT, dx):
    """run_edge.py:377-417 (HV_GARM) / run_ed4.py:219-260 (HV_FD)."""
    u0 = [_c32(a) for a in u0]
    res = psi.shape[:3]
    out = [np.empty_like(a) for a in u0]
    dT = dT if dT is not None else [None] * 3
    lib().orc_map_u_psi(_i(variant), *(_i(s) for s in res), _f(dx), *(_p(a) for a in u0), *(_p(a) for a in out),
                        _p(_c32(psi)), *(_p(_c32(t)) for t in T),
                        *(_p(_c32(t)) if t is not None else None for t in dT))
    return out


def map_smoke_psi(variant, smoke0, psi, T, dT, dx):
    """run_edge.py:444-466 / run_ed4.py:293-310."""
    res = psi.shape[:3]
    out = np.empty(res + (4,), F32)
    dT = dT if dT is not None else [None] * 3
    lib().orc_map_smoke_psi(_i(variant), *(_i(s) for s in res), _f(dx), _p(_c32(smoke0)), _p(out), _p(_c32(psi)),
                            *(_p(_c32(t)) for t in T), *(_p(_c32(t)) if t is not None else None for t in dT))
    return out


def clamp_smoke_psi(variant, smoke0, smoke1, psi, T, dT, dx):
    """run_edge.py:481-505 / run_ed4.py:313-336 (in place on smoke1)."""
    res = psi.shape[:3]
    dT = dT if dT is not None else [None] * 3
    lib().orc_clamp_smoke_psi(_i(variant), *(_i(s) for s in res), _f(dx), _p(_c32(smoke0)), _p(smoke1),
                              _p(_c32(psi)), *(_p(_c32(t)) for t in T),
                              *(_p(_c32(t)) if t is not None else None for t in dT))


def map_smoke(smoke0, phi, dx):
    """run_edge.py:421-427."""
    res = smoke0.shape[:3]
    out = np.empty(res + (4,), F32)
    lib().orc_map_smoke(*(_i(s) for s in res), _f(dx), _p(_c32(smoke0)), _p(out), *(_p(_c32(a)) for a in phi))
    return out


def clamp_smoke(smoke0, smoke1, phi, dx):
    """run_edge.py:470-477 (in place on smoke1)."""
    res = smoke0.shape[:3]
    lib().orc_clamp_smoke(*(_i(s) for s in res), _f(dx), _p(_c32(smoke0)), _p(smoke1), *(_p(_c32(a)) for a in phi))


def clamp_u(u, u1):
    """run_edge.py:509-519 clamp_u -> new array."""
    u = _c32(u)
    u1 = _c32(u1)
    out = np.empty_like(u)
    lib().orc_clamp_u(*(_i(s) for s in u.shape), _p(u), _p(u1), _p(out))
    return out


def calc_max_speed(u):
    """run_edge.py:296-303."""
    u = [_c32(a) for a in u]
    return float(lib().orc_calc_max_speed(*(_i(s) for s in _res_from_u(u)), *(_p(a) for a in u)))


# ----------------------------------------------------------------------------
# projection
# ----------------------------------------------------------------------------
def _bt(boundary_types):
    return np.ascontiguousarray(np.asarray(boundary_types, np.int32).reshape(6))


def poisson(u, base_level=3, boundary_types=((2, 2), (2, 2), (2, 2)), abs_tol=1e-12, rel_tol=1e-12,
            max_iters=400, force=None):
    """mgpcg.py:440-445 MGPCG_3.Poisson (in place on u; force buffers for
    Poisson_with_buffer, mgpcg.py:481-486).  Returns (iters, div, p, rTr)."""
    res = _res_from_u(u)
    div = np.empty(res, F32)
    p = np.empty(res, F32)
    rtr = ctypes.c_double(0)
    bt = _bt(boundary_types)
    f = force if force is not None else [None] * 3
    it = lib().orc_poisson(*(_i(s) for s in res), _i(base_level), _p(bt), ctypes.c_double(abs_tol),
                           ctypes.c_double(rel_tol), _i(max_iters), *(_p(a) for a in u), *(_p(a) for a in f),
                           _p(div), _p(p), ctypes.byref(rtr))
    return it, div, p, rtr.value


def vcycle(r, base_level, boundary_types=((2, 2), (2, 2), (2, 2))):
    """One application of mgpcg.py:177-195 plus Ap (mgpcg.py:112-117)."""
    r = _c32(r)
    z = np.empty_like(r)
    Ap = np.empty_like(r)
    L = lib().orc_vcycle(*(_i(s) for s in r.shape), _i(base_level), _p(_bt(boundary_types)), _p(r), _p(z), _p(Ap))
    return z, Ap, L


def poisson_solid(u, mask, bvel, base_level=3, boundary_types=((2, 2), (2, 2), (2, 2)), tol=1e-12, max_iters=100):
    """mgpcg_solid.py:418-427 MGPCG_Solid_3.Poisson (in place on u)."""
    res = _res_from_u(u)
    mask = np.ascontiguousarray(mask, np.int32)
    div = np.empty(res, F32)
    p = np.empty(res, F32)
    bm1 = np.zeros(tuple(s // 2 for s in res), np.int32)
    bm2 = np.zeros(tuple(s // 4 for s in res), np.int32)
    dsum = ctypes.c_double(0)
    it = lib().orc_poisson_solid(*(_i(s) for s in res), _i(base_level), _p(_bt(boundary_types)), _p(mask),
                                 _p(_c32(bvel)), ctypes.c_double(tol), _i(max_iters), *(_p(a) for a in u),
                                 _p(div), _p(p), _p(bm1), _p(bm2), ctypes.byref(dsum))
    return it, div, p, bm1, bm2, dsum.value


# ----------------------------------------------------------------------------
# particles
# ----------------------------------------------------------------------------
def lp_acc(u, dx, vel, pos, num, dt, St, gravity):
    """lp.py:6-29."""
    res = _res_from_u(u)
    acc = np.zeros_like(vel)
    lib().orc_lp_acc(*(_i(s) for s in res), _f(dx), *(_p(_c32(a)) for a in u), _p(_c32(vel)), _p(_c32(pos)),
                     _p(acc), _i(num), _i(vel.shape[0]), _f(dt), _f(St), _f(gravity))
    return acc


def lp_velocity(acc, vel, pos, dt, dx, num, L):
    """lp.py:32-70 (in place on vel)."""
    lib().orc_lp_velocity(_p(_c32(acc)), _p(vel), _p(_c32(pos)), _f(dt), _f(dx), _i(num), *(_f(v) for v in L))


def lp_vel_diff(u, dx, vel, pos, num, St, dens, erad):
    """lp.py:73-97."""
    res = _res_from_u(u)
    vd = np.zeros_like(vel)
    lib().orc_lp_vel_diff(*(_i(s) for s in res), _f(dx), *(_p(_c32(a)) for a in u), _p(_c32(vel)), _p(vd),
                          _p(_c32(pos)), _i(num), _f(St), _f(dens), _f(erad))
    return vd


def lp_p2g(res, dx, vdiff, pos, rad, num, lrad, L):
    """lp.py:100-156."""
    drag = [np.zeros(s, F32) for s in face_shapes(res)]
    lib().orc_lp_p2g(*(_i(s) for s in res), _f(dx), *(_p(d) for d in drag), _p(_c32(vdiff)), _p(_c32(pos)),
                     _p(_c32(rad)), _i(num), _f(lrad), *(_f(v) for v in L))
    return drag


def lp_position(vel, pos, dt, num, L):
    """lp.py:158-181 (in place on pos)."""
    lib().orc_lp_position(_p(_c32(vel)), _p(pos), _f(dt), _i(num), *(_f(v) for v in L))


def lp_viscous(u, dx, Re):
    """lp.py:183-219."""
    out = []
    for a in u:
        a = _c32(a)
        o = np.empty_like(a)
        lib().orc_lp_viscous(*(_i(s) for s in a.shape), _f(dx), _f(Re), _p(a), _p(o))
        out.append(o)
    return out


# ----------------------------------------------------------------------------
# initial conditions
# ----------------------------------------------------------------------------
def add_vortex_ring(res, dx, w, rad, delta, c, ex, ey, u, smoke, color, num_samples):
    """init_conditions.py:11-36 (accumulates into u and smoke in place)."""
    lib().orc_add_vortex_ring(*(_i(s) for s in res), _f(dx), _f(w), _f(rad), _f(delta), _p(_c32(c)), _p(_c32(ex)),
                              _p(_c32(ey)), _p(u), _p(smoke), _p(_c32(color)), _i(num_samples))


def split_central_vector(vc):
    """taichi_utils.py:103-116."""
    res = vc.shape[:3]
    out = [np.empty(s, F32) for s in face_shapes(res)]
    lib().orc_split_central_vector(*(_i(s) for s in res), _p(_c32(vc)), *(_p(a) for a in out))
    return out


def get_central_vector(u):
    """taichi_utils.py:95-100: the face average per cell (float32)."""
    ux, uy, uz = (np.asarray(a, F32) for a in u)
    vc = np.empty((ux.shape[0] - 1,) + ux.shape[1:] + (3,), F32)
    vc[..., 0] = F32(0.5) * (ux[1:] + ux[:-1])
    vc[..., 1] = F32(0.5) * (uy[:, 1:] + uy[:, :-1])
    vc[..., 2] = F32(0.5) * (uz[:, :, 1:] + uz[:, :, :-1])
    return vc


def curl(vf, dx):
    """taichi_utils.py:69-92: central differences with the neighbour index
    clamped to the grid (sample, taichi_utils.py:61-66), float32."""
    vf = np.asarray(vf, F32)
    inv = F32(1.0) / (F32(2.0) * F32(dx))
    p = np.pad(vf, ((1, 1), (1, 1), (1, 1), (0, 0)), mode="edge")
    n0, n1, n2 = vf.shape[:3]

    def d(c, axis):
        sl_hi = [slice(1, 1 + n0), slice(1, 1 + n1), slice(1, 1 + n2), c]
        sl_lo = list(sl_hi)
        sl_hi[axis] = slice(2, 2 + vf.shape[axis])
        sl_lo[axis] = slice(0, vf.shape[axis])
        return inv * (p[tuple(sl_hi)] - p[tuple(sl_lo)])
    cf = np.empty_like(vf)
    cf[..., 0] = d(2, 1) - d(1, 2)
    cf[..., 1] = d(0, 2) - d(2, 0)
    cf[..., 2] = d(1, 0) - d(0, 1)
    return cf


# ----------------------------------------------------------------------------
# the EDGE substep (run_edge.py:588-712), non-particle, non-solid path
# ----------------------------------------------------------------------------
class EdgeState:
    """Simulation state of the EDGE driver (run_edge.py:164-254 fields)."""

    def __init__(self, res, dx, u, smoke):
        self.res = tuple(res)
        self.dx = F32(dx)
        self.u = [np.array(a, F32) for a in u]
        self.smoke = np.array(smoke, F32)
        self.i = -1
        z3 = lambda: np.zeros(self.res + (3,), F32)  # noqa: E731
        self.psi, self.T, self.dT = z3(), [z3() for _ in range(3)], [z3() for _ in range(3)]
        self.phi = [np.zeros(s + (3,), F32) for s in face_shapes(self.res)]
        self.F = [np.zeros(s + (3,), F32) for s in face_shapes(self.res)]
        self.init_u = [np.zeros_like(a) for a in self.u]
        self.init_smoke = np.zeros_like(self.smoke)


def emit_smoke(res, dx, centers, colors, radius, smoke):
    """init_conditions.py:177-232 emit_smoke_delta (later emitters win)."""
    X = center_coords(res, dx).astype(np.float32)
    for c, col in zip(centers, colors):
        d = X - np.asarray(c, np.float32)
        hit = np.sqrt((d * d).sum(-1)) < F32(radius)
        smoke[hit] = np.asarray(col, np.float32)


def edge_substep(st, cfl=0.5, reinit_every=12, ed_eps=None, base_level=3, bfecc_clamp=True, dt=None,
                 abs_tol=1e-12, rel_tol=1e-12, variant="edge", solid=None, emitters=None, particles=None,
                 max_iters=400, project=None):
    """One iteration of run_edge.py:588-712 (variant "edge"), run_ed4.py:
    402-484 ("ed4"), run_ed8.py:365-451 ("ed8"), run_ge.py:363-448 ("ge",
    the ED8 substep with the GE march) or run_efm.py:319-406 ("efm", the ED8
    substep with the face map backtracked through the cached velocities);
    no frame bookkeeping: dt = CFL*dx/max_speed unless given.  Returns
    (dt, iters).

    max_iters bounds the plain projection's CG loop (mgpcg.py:440-445 fixes
    it at 400).  `project`, when given, replaces both projections of the
    substep: it is called as project(u, force) with the face velocity list
    (and the Poisson_with_buffer force list or None), must update u in place
    and return an iteration count; the parity tests use it to hand both
    implementations the same projected velocity."""
    if variant != "edge":
        return _ed_substep(st, cfl, reinit_every, ed_eps, base_level, bfecc_clamp, dt, abs_tol, rel_tol, variant,
                           max_iters, project)
    dx = float(st.dx)
    eps = F32(ed_eps if ed_eps is not None else 0.025 * dx)
    st.i += 1
    j = st.i % reinit_every
    if dt is None:
        ms = calc_max_speed(st.u)
        if particles is not None:  # run_edge.py:598-600
            P = particles
            v = P["vel"][:P["num"]].astype(np.float32)
            ms = max(ms, max(1e-3, float(np.sqrt((v * v).sum(-1)).max()) if len(v) else 1e-3))
        dt = cfl * dx / ms  # run_edge.py:595-614 (Python double)
    dt32 = F32(dt)

    hook = project

    def _project(u, force=None):
        if hook is not None:
            return hook(u, force)
        if solid is not None:
            return poisson_solid(u, solid[0], solid[1], base_level)[0]
        return poisson(u, base_level, abs_tol=abs_tol, rel_tol=rel_tol, max_iters=max_iters, force=force)[0]
    if j == 0:
        # run_edge.py:616-625
        for a in range(3):
            st.phi[a][...] = face_coords(st.res, dx, a)
            st.F[a][...] = np.eye(3, dtype=F32)[a]
        st.psi[...] = center_coords(st.res, dx)
        for c in range(3):
            st.T[c][...] = np.eye(3, dtype=F32)[c]
            st.dT[c][...] = 0
        st.init_u = [a.copy() for a in st.u]
        st.init_smoke = st.smoke.copy()
    vis = None
    if particles is not None:
        # run_edge.py:627-641
        P = particles
        L = P["L"]
        acc = lp_acc(st.u, dx, P["vel"], P["pos"], P["num"], dt32, P["St"], P["gravity"])
        lp_velocity(acc, P["vel"], P["pos"], dt32, dx, P["num"], L)
        vd = lp_vel_diff(st.u, dx, P["vel"], P["pos"], P["num"], P["St"], P["density_ratio"], P["erad"])
        drag = lp_p2g(st.res, dx, vd, P["pos"], P["rad"], P["num"], P["lrad"], L)
        lp_position(P["vel"], P["pos"], dt32, P["num"], L)
        vis = lp_viscous(st.u, dx, P["Re"])
        vis = [v + F32(1.0) * d for v, d in zip(vis, drag)]
    if emitters is not None:
        # run_edge.py:643-648
        centers, colors, radius = emitters
        st.smoke = np.zeros_like(st.smoke)
        emit_smoke(st.res, dx, centers, colors, radius, st.smoke)
        err = map_smoke(st.smoke, st.phi, dx)
        st.init_smoke = np.minimum(st.init_smoke + F32(1.0) * err, F32(1.0))
    st.u = advect_u_semi_lagrangian(st.u, dx, F32(0.5 * dt))
    it1 = _project(st.u)
    st.psi, st.T, st.dT = march_edge(st.u, st.psi, st.T, st.dT, dx, dt32, eps)
    for a in range(3):
        advance_map(st.u, st.phi[a], st.F[a], a, dx, dt32)
    if vis is not None:
        # run_edge.py:662-667
        tmp = map_u(vis, st.F, st.phi, dx)
        st.init_u = [a + dt32 * t for a, t in zip(st.init_u, tmp)]
    u_new = map_u_psi(HV_GARM, st.init_u, st.psi, st.T, st.dT, dx)
    smoke_new = map_smoke_psi(HV_GARM, st.init_smoke, st.psi, st.T, st.dT, dx)
    err_u = map_u(u_new, st.F, st.phi, dx)
    err_smoke = map_smoke(smoke_new, st.phi, dx)
    err_u = [(e + F32(-1.0) * a) for e, a in zip(err_u, st.init_u)]          # add_fields(err, init, err, -1)
    err_smoke = err_smoke + F32(-1.0) * st.init_smoke
    err_u = [F32(0.5) * e for e in err_u]                                    # scale_field(err, 0.5)
    err_smoke = F32(0.5) * err_smoke
    tmp_u = map_u_psi(HV_GARM, err_u, st.psi, st.T, st.dT, dx)
    tmp_smoke = map_smoke_psi(HV_GARM, err_smoke, st.psi, st.T, st.dT, dx)
    err_u = [a + F32(-1.0) * t for a, t in zip(u_new, tmp_u)]                # add_fields(u, tmp, err, -1)
    smoke_new = smoke_new + F32(-1.0) * tmp_smoke
    clamp_smoke_psi(HV_GARM, st.init_smoke, smoke_new, st.psi, st.T, st.dT, dx)
    if bfecc_clamp:
        st.u = [clamp_u(e, a) for e, a in zip(err_u, u_new)]
    else:
        st.u = err_u
    st.smoke = smoke_new
    if vis is not None:
        particles["vis"] = [np.zeros_like(a) for a in st.u]
        it2 = _project(st.u, force=particles["vis"])
    else:
        it2 = _project(st.u)
    return dt, (it1, it2)


def _ed_substep(st, cfl, reinit_every, ed_eps, base_level, bfecc_clamp, dt, abs_tol, rel_tol, variant, max_iters,
                project):
    def _project(u):
        if project is not None:
            return project(u, None)
        return poisson(u, base_level, abs_tol=abs_tol, rel_tol=rel_tol, max_iters=max_iters)[0]

    dx = float(st.dx)
    eps = F32(ed_eps if ed_eps is not None else 0.025 * dx)
    st.i += 1
    j = st.i % reinit_every
    if dt is None:
        dt = cfl * dx / calc_max_speed(st.u)
    dt32 = F32(dt)
    if not hasattr(st, "d2T"):
        st.d2T = [np.zeros(st.res, F32) for _ in range(3)]
    if j == 0:
        for a in range(3):
            st.phi[a][...] = face_coords(st.res, dx, a)
            st.F[a][...] = np.eye(3, dtype=F32)[a]
        st.psi[...] = center_coords(st.res, dx)
        for c in range(3):
            st.T[c][...] = np.eye(3, dtype=F32)[c]
            st.dT[c][...] = 0
            st.d2T[c][...] = 0
        st.init_u = [a.copy() for a in st.u]
        st.init_smoke = st.smoke.copy()
    st.u = advect_u_semi_lagrangian(st.u, dx, F32(0.5 * dt))
    it1 = _project(st.u)
    if variant == "efm":
        # run_efm.py:360-365: cache the projected velocity, backtrack the faces
        if not hasattr(st, "u_cache"):
            st.u_cache, st.dts = {}, {}
        st.u_cache[j] = [a.copy() for a in st.u]
        st.dts[j] = dt32
        pf, tf = efm_backtrack([st.u_cache[s] for s in range(j + 1)], [st.dts[s] for s in range(j + 1)], dx)
    elif variant == "ed4":
        st.psi, st.T = march_ed4(st.u, st.psi, st.T, dx, dt32, eps)
    elif variant == "ge":
        st.psi, st.T, st.dT, st.d2T = march_ge(st.u, st.psi, st.T, st.dT, st.d2T, dx, dt32)
    else:
        st.psi, st.T, st.dT, st.d2T = march_ed8(st.u, st.psi, st.T, st.dT, st.d2T, dx, dt32, eps)
    for a in range(3):
        advance_map(st.u, st.phi[a], st.F[a], a, dx, dt32)
    if variant == "ed4":
        # run_ed4.py:438-460
        u_new = map_u_psi(HV_FD, st.init_u, st.psi, st.T, None, dx)
        smoke_new = map_smoke_psi(HV_FD, st.init_smoke, st.psi, st.T, None, dx)
    else:
        # run_ed8.py:226-230, 410-433: psi and T on the faces, then map_u / map_smoke
        if variant != "efm":
            pf, tf = split_psi_hermite(st.psi, st.T, st.dT, st.d2T, dx)
        u_new = map_u(st.init_u, tf, pf, dx)
        smoke_new = map_smoke(st.init_smoke, pf, dx)
    err_u = map_u(u_new, st.F, st.phi, dx)
    err_smoke = map_smoke(smoke_new, st.phi, dx)
    err_u = [F32(0.5) * (e + F32(-1.0) * a) for e, a in zip(err_u, st.init_u)]
    err_smoke = F32(0.5) * (err_smoke + F32(-1.0) * st.init_smoke)
    if variant == "ed4":
        tmp_u = map_u_psi(HV_FD, err_u, st.psi, st.T, None, dx)
        tmp_smoke = map_smoke_psi(HV_FD, err_smoke, st.psi, st.T, None, dx)
    else:
        tmp_u = map_u(err_u, tf, pf, dx)
        tmp_smoke = map_smoke(err_smoke, pf, dx)
    err_u = [a + F32(-1.0) * t for a, t in zip(u_new, tmp_u)]
    smoke_new = smoke_new + F32(-1.0) * tmp_smoke
    if variant == "ed4":
        clamp_smoke_psi(HV_FD, st.init_smoke, smoke_new, st.psi, st.T, None, dx)
    else:
        clamp_smoke(st.init_smoke, smoke_new, pf, dx)
    st.u = [clamp_u(e, a) for e, a in zip(err_u, u_new)] if bfecc_clamp else err_u
    st.smoke = smoke_new
    it2 = _project(st.u)
    return dt, (it1, it2)
