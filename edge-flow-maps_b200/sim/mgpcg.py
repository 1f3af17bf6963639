"""Drop-in for the reference's sim/mgpcg.py: MGPCG_3 with the same
constructor and Poisson / Poisson_with_buffer methods (mgpcg.py:364-491),
backed by the device-resident solver of libedgeb200.so.

Behaviour kept from the reference:
  * level count int(log2(min N)) - base_level + 1 (mgpcg.py:34), 2 pre/post
    and 20 bottom red-black sweeps, restriction x1/(dim-1);
  * convergence when r.r < max(abs_tol, rel_tol * z0.r0) (mgpcg.py:228, 254);
  * Poisson ignores its max_iters argument and uses 400
    (solve_pressure_MGPCG, mgpcg.py:434-438);
  * recentering of r over all cells when every wall is Neumann.
The reference prints a convergence line after every solve (a host
synchronisation); here it is printed only with verbose=True or
EDGE_MGPCG_LOG=1, and ``last_result()`` returns (iterations, |r|, status).
"""
import math
import os

import torch

from edgeb200.fields import dims_from_faces
from edgeb200.projection import Projection

_LOG = os.environ.get("EDGE_MGPCG_LOG", "0") == "1"


class MGPCG:
    """Shared constructor state of mgpcg.py:23-57."""

    def __init__(self, boundary_types, N, dim=3, base_level=3, real=float):
        if dim != 3:
            raise NotImplementedError("only the 3-D solver is on the EDGE path")
        self.N = list(int(n) for n in N)
        self.dim = dim
        self.base_level = base_level
        self.n_mg_levels = int(math.log2(min(self.N))) - base_level + 1
        self.pre_and_post_smoothing = 2
        self.bottom_smoothing = 20
        self.boundary_types = boundary_types
        self.num_entries = math.prod(self.N)
        self.use_multigrid = True

    def get_memory_usage(self):
        """Bytes of the level pyramid and CG vectors (mgpcg.py:285-287)."""
        n = self.num_entries
        lv = sum(math.prod(v // (2 ** l) for v in self.N) for l in range(self.n_mg_levels))
        return 4 * (2 * lv + 5 * n)


class MGPCG_3(MGPCG):
    def __init__(self, boundary_types, N, base_level=3, abs_tol=1e-12, rel_tol=1e-12, real=float):
        super().__init__(boundary_types, N, dim=3, base_level=base_level, real=real)
        self.abs_tol = abs_tol
        self.rel_tol = rel_tol
        self._proj = Projection(self.N, base_level=base_level, boundary_types=_bt(boundary_types))
        self._verbose_result = None

    def Poisson(self, u_x, u_y, u_z, max_iters=400, verbose=False):
        """mgpcg.py:440-445 (max_iters is fixed at 400 as in solve_pressure_MGPCG)."""
        dims_from_faces(u_x, u_y, u_z)
        self._proj.poisson(u_x, u_y, u_z, None, self.abs_tol, self.rel_tol, 400)
        self._report(verbose)

    def Poisson_with_buffer(self, u_x, u_y, u_z, f_x, f_y, f_z, max_iters=400, verbose=False):
        """mgpcg.py:481-486: also writes the pressure-gradient force -grad p."""
        dims_from_faces(u_x, u_y, u_z)
        self._proj.poisson(u_x, u_y, u_z, (f_x, f_y, f_z), self.abs_tol, self.rel_tol, 400)
        self._report(verbose)

    def _report(self, verbose):
        if verbose or _LOG:
            it, rtr, st = self._proj.result()
            err = math.sqrt(max(rtr, 0.0))
            if st == 0:
                print("[MGPCG] Converged at iter: ", it, " with final error: ", err)
            else:
                print("[MGPCG] Return without converging at iter: ", it, " with final error: ", err)

    def last_result(self):
        """(iterations as the reference prints them, sqrt(r.r), status)."""
        it, rtr, st = self._proj.result()
        return it, math.sqrt(max(rtr, 0.0)), st

    @property
    def u_div(self):
        return self._proj.get("div")

    @property
    def p(self):
        return self._proj.get("p")

    def get_memory_usage(self):
        return super().get_memory_usage() + 4 * self.num_entries


def _bt(boundary_types):
    if isinstance(boundary_types, torch.Tensor):
        boundary_types = boundary_types.tolist()
    return boundary_types
