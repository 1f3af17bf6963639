"""MGPCG pressure projection handle (sim/mgpcg.py, sim/mgpcg_solid.py) over
the C ABI.  One ``Projection`` owns the device level pyramid and the captured
solve graphs; ``poisson`` runs the whole projection on the current stream
with no host synchronisation.
"""
import ctypes
import weakref

import torch

from . import _native as N
from .fields import ptr, require, stream


_LIVE = weakref.WeakSet()


def live_solvers():
    return [p for p in list(_LIVE) if getattr(p, "_h", None)]


def boundary_array(boundary_types):
    """boundary_types (3x2, 2 = wall) as the int[6] the C ABI takes."""
    if hasattr(boundary_types, "tolist"):
        boundary_types = boundary_types.tolist()
    flat = [int(v) for row in boundary_types for v in row]
    if len(flat) != 6:
        raise ValueError("boundary_types must be 3x2")
    return (ctypes.c_int * 6)(*flat)


class Projection:
    def __init__(self, N_res, base_level=3, boundary_types=((2, 2), (2, 2), (2, 2)), mask=None, bvel=None,
                 precision=0):
        N.load()
        self.res = tuple(int(n) for n in N_res)
        self.base_level = int(base_level)
        self._bt = boundary_array(boundary_types)
        self.mask = mask
        self.bvel = bvel
        if mask is not None:
            require(mask, "boundary_mask")
            if mask.dtype != torch.int32 or tuple(mask.shape) != self.res:
                raise ValueError("boundary_mask must be int32 of the cell shape")
            require(bvel, "boundary_vel")
        h = ctypes.c_void_p()
        N.call("edge_mgpcg_create", ctypes.byref(h), *self.res, self.base_level, self._bt, ptr(mask), ptr(bvel),
               int(precision))
        self._h = h
        self.levels = N.load().edge_mgpcg_levels(h)
        _LIVE.add(self)

    def close(self):
        if getattr(self, "_h", None):
            N.load().edge_mgpcg_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def poisson(self, u_x, u_y, u_z, f=None, abs_tol=1e-12, rel_tol=1e-12, max_iters=-1):
        fx, fy, fz = (None, None, None) if f is None else f
        N.call("edge_mgpcg_poisson", self._h, ptr(u_x, "u_x"), ptr(u_y, "u_y"), ptr(u_z, "u_z"), ptr(fx), ptr(fy),
               ptr(fz), ctypes.c_double(abs_tol), ctypes.c_double(rel_tol), int(max_iters), stream())

    def solve(self, b, x, abs_tol=1e-12, rel_tol=1e-12, max_iters=-1):
        N.call("edge_mgpcg_solve", self._h, ptr(b, "b"), ptr(x, "x"), ctypes.c_double(abs_tol),
               ctypes.c_double(rel_tol), int(max_iters), stream())

    def result(self):
        """(iterations as the reference prints them, final r.r, status code);
        synchronises the stream."""
        it = ctypes.c_int()
        rtr = ctypes.c_double()
        st = ctypes.c_int()
        N.call("edge_mgpcg_result", self._h, ctypes.byref(it), ctypes.byref(rtr), ctypes.byref(st), stream())
        return it.value, rtr.value, st.value

    def restart(self):
        """The next CG update of a stepwise solve restarts the recursion."""
        N.call("edge_mgpcg_restart", self._h, stream())

    def progress(self):
        """(iterations, r.r, whether the CG loop is still running);
        synchronises the stream."""
        it = ctypes.c_int()
        rtr = ctypes.c_double()
        run = ctypes.c_int()
        N.call("edge_mgpcg_progress", self._h, ctypes.byref(it), ctypes.byref(rtr), ctypes.byref(run), stream())
        return it.value, rtr.value, bool(run.value)

    def kernel_count(self):
        """Kernels this solver has run (counted on the device; synchronises)."""
        c = ctypes.c_longlong()
        N.call("edge_mgpcg_kernel_count", self._h, ctypes.byref(c), stream())
        return c.value

    # -- stepwise solve with a replaceable coarse solver --------------------------
    def coarse_shape(self):
        """(level, (n0, n1, n2)) of the level whose residual equation the
        coarse group solves; raises on the per-level kernel path."""
        lvl = ctypes.c_int()
        dims = (ctypes.c_int * 3)()
        N.call("edge_mgpcg_coarse_shape", self._h, ctypes.byref(lvl), dims)
        return lvl.value, tuple(int(v) for v in dims)

    def solve_begin(self, b, abs_tol=1e-12, rel_tol=1e-12, max_iters=-1):
        N.call("edge_mgpcg_solve_begin", self._h, ptr(b, "b"), ctypes.c_double(abs_tol), ctypes.c_double(rel_tol),
               int(max_iters), stream())

    def poisson_begin(self, u_x, u_y, u_z, abs_tol=1e-12, rel_tol=1e-12, max_iters=-1):
        N.call("edge_mgpcg_poisson_begin", self._h, ptr(u_x, "u_x"), ptr(u_y, "u_y"), ptr(u_z, "u_z"),
               ctypes.c_double(abs_tol), ctypes.c_double(rel_tol), int(max_iters), stream())

    def poisson_end(self, u_x, u_y, u_z, f=None):
        fx, fy, fz = (None, None, None) if f is None else f
        N.call("edge_mgpcg_poisson_end", self._h, ptr(u_x, "u_x"), ptr(u_y, "u_y"), ptr(u_z, "u_z"), ptr(fx),
               ptr(fy), ptr(fz), stream())

    def coarse_get_r(self, dense):
        N.call("edge_mgpcg_coarse_get_r", self._h, ptr(dense), stream())

    def coarse_set_z(self, dense):
        N.call("edge_mgpcg_coarse_set_z", self._h, ptr(dense), stream())

    def coarse_default(self):
        N.call("edge_mgpcg_coarse_default", self._h, stream())

    def solve_iter(self):
        N.call("edge_mgpcg_solve_iter", self._h, stream())

    def solve_end(self, b, x):
        N.call("edge_mgpcg_solve_end", self._h, ptr(b, "b"), ptr(x, "x"), stream())

    def vcycle(self, r, z):
        N.call("edge_mgpcg_vcycle", self._h, ptr(r), ptr(z), stream())

    def apply_A(self, p, Ap):
        N.call("edge_mgpcg_apply_A", self._h, ptr(p), ptr(Ap), stream())

    def get(self, which):
        out = torch.empty(self.res, dtype=torch.float32, device="cuda")
        N.call("edge_mgpcg_get", self._h, {"div": 0, "p": 1}[which], ptr(out), stream())
        return out
