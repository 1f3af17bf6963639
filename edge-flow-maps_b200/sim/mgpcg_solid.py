"""Drop-in for the reference's sim/mgpcg_solid.py: MGPCG_Solid_3
(mgpcg_solid.py:313-432) on libedgeb200.so.

Kept from the reference: solid-cell velocities imposed on their six faces
(mgpcg_solid.py:344-356), the fluid-only divergence whose mean is removed only
when its sum is positive (mgpcg_solid.py:359-383, 422-424), per-level masks
where a coarse cell is solid iff its 8 children are (downsampled before every
solve, mgpcg_solid.py:87-97, 238-239), recentering over all cells including
solids (mgpcg_solid.py:197-202), absolute tol 1e-12 and 100 iterations
(mgpcg_solid.py:413-416).  The reference prints the divergence sums every
call; here with verbose=True or EDGE_MGPCG_LOG=1.
"""
import math
import os

import torch

from edgeb200.fields import dims_from_faces, require
from edgeb200.projection import Projection

from .mgpcg import MGPCG, _bt

_LOG = os.environ.get("EDGE_MGPCG_LOG", "0") == "1"


class MGPCG_Solid_3(MGPCG):
    def __init__(self, boundary_types, boundary_mask, boundary_vel, N, base_level=3, real=float):
        super().__init__(boundary_types, N, dim=3, base_level=base_level, real=real)
        require(boundary_mask, "boundary_mask")
        require(boundary_vel, "boundary_vel")
        if boundary_mask.dtype != torch.int32:
            raise ValueError("boundary_mask must be an int32 tensor (ti.i32 field)")
        self.boundary_mask = boundary_mask
        self.boundary_vel = boundary_vel
        self._proj = Projection(self.N, base_level=base_level, boundary_types=_bt(boundary_types),
                                mask=boundary_mask, bvel=boundary_vel)

    def Poisson(self, u_x, u_y, u_z, verbose=False):
        """mgpcg_solid.py:418-427."""
        dims_from_faces(u_x, u_y, u_z)
        self._proj.poisson(u_x, u_y, u_z, None, 1e-12, 0.0, 100)
        if verbose or _LOG:
            it, rtr, st = self._proj.result()
            print("[MGPCG] Converged at iter: " if st == 0 else "[MGPCG] Return without converging at iter: ", it,
                  " with final error: ", math.sqrt(max(rtr, 0.0)))

    def last_result(self):
        it, rtr, st = self._proj.result()
        return it, math.sqrt(max(rtr, 0.0)), st

    @property
    def u_div(self):
        return self._proj.get("div")

    @property
    def p(self):
        return self._proj.get("p")

    def get_memory_usage(self):
        lv = sum(math.prod(v // (2 ** l) for v in self.N) for l in range(1, self.n_mg_levels))
        return super().get_memory_usage() + 4 * self.num_entries + 4 * lv
