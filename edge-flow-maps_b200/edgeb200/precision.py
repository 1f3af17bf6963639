"""Mixed-precision solves and the FP64 reference solve of the precision
study (no reference counterpart).

The mixed-precision solvers (Projection(..., precision=1 or 2)) store the
V-cycle's level arrays in bfloat16 or float16 while the CG vectors, the
residual and the arithmetic stay float32 and the dot products float64.
`RefinedSolver` wraps such a solver in iterative refinement: the residual of
a float64 iterate is formed in float64 on the device, each inner solve
reduces it by `inner_rel`, and the float64 iterate takes the correction, so
the TRUE relative residual reaches the target, not only the recursion's.
Errors are measured against an FP64 solve of the same system: flexible CG in
float64 (vectors, operator, dot products) whose preconditioner is the
float32 V-cycle; preconditioner rounding only slows convergence, the
float64 recursion sets the accuracy.
"""
import math

import torch

from . import _native as N
from .fields import ptr, ptr_any, stream

F64 = (torch.float64,)


class RefinedSolver:
    """Iterative refinement around a (mixed-precision) Projection on the
    all-Neumann or open-boundary Poisson system of its grid.  solve(b)
    returns the float64 solution x with ||b - A x|| <= rel_tol ||b|| and
    records the outer steps, inner iterations and the true residual."""

    def __init__(self, proj, inner_rel=1e-3, max_outer=12):
        self.P = proj
        self.inner_rel = float(inner_rel)
        self.max_outer = int(max_outer)
        res = proj.res
        self.r32 = torch.empty(res, device="cuda")
        self.d32 = torch.empty(res, device="cuda")
        self.sums = torch.zeros(2, dtype=torch.float64, device="cuda")
        self.host = torch.zeros(2, dtype=torch.float64).pin_memory()
        self.stats = {}

    def _residual(self, b64, x64):
        N.call("edge_mgpcg_refine_residual", self.P._h, ptr_any(b64, F64), ptr_any(x64, F64), ptr(self.r32),
               ptr_any(self.sums, F64), stream())
        self.host.copy_(self.sums, non_blocking=True)
        torch.cuda.current_stream().synchronize()
        return float(self.host[0]), float(self.host[1])

    def solve(self, b, x64=None, rel_tol=1e-6):
        b64 = b if b.dtype == torch.float64 else b.double()
        b64 = b64.contiguous()
        x64 = torch.zeros_like(b64) if x64 is None else x64
        inner_its = []
        rr, bb = self._residual(b64, x64)
        outer = 0
        while math.sqrt(rr) > rel_tol * math.sqrt(bb) and outer < self.max_outer:
            # the inner solve's tolerance is relative to its preconditioned
            # initial residual (mgpcg.py:224), the same number every step,
            # so one captured solve graph serves every outer step
            self.P.solve(self.r32, self.d32, abs_tol=0.0, rel_tol=self.inner_rel ** 2)
            N.call("edge_mgpcg_refine_update", self.P._h, ptr_any(x64, F64), ptr(self.d32), stream())
            it, _, st = self.P.result()
            inner_its.append(it)
            rr, bb = self._residual(b64, x64)
            outer += 1
        self.stats = {"outer": outer, "inner_iters": inner_its, "true_rel_residual": math.sqrt(rr / max(bb, 1e-300))}
        return x64


def apply_A64(P, p, Ap):
    N.call("edge_mgpcg_apply_A_f64", P._h, ptr_any(p, F64), ptr_any(Ap, F64), stream())


def fp64_solve(P, b, rel_tol=1e-12, max_iters=300):
    """x (float64) with ||b - mean(b) - A x|| <= rel_tol ||b - mean(b)||, the
    all-Neumann solution with zero mean."""
    b64 = b.double().contiguous()
    b64 = b64 - b64.mean()
    x = torch.zeros_like(b64)
    r = b64.clone()
    Ap = torch.empty_like(b64)
    z32 = torch.empty(b.shape, dtype=torch.float32, device=b.device)

    def precond(res):
        P.vcycle(res.float().contiguous(), z32)
        z = z32.double()
        return z - z.mean()

    bn = float(torch.linalg.vector_norm(b64))
    z = precond(r)
    p = z.clone()
    rz = float(torch.dot(r.view(-1), z.view(-1)))
    for _ in range(max_iters):
        apply_A64(P, p, Ap)
        alpha = rz / float(torch.dot(p.view(-1), Ap.view(-1)))
        x.add_(p, alpha=alpha)
        r_old = r.clone()
        r.sub_(Ap, alpha=alpha)
        r -= r.mean()
        if float(torch.linalg.vector_norm(r)) <= rel_tol * bn:
            break
        z = precond(r)
        beta = float(torch.dot(z.view(-1), (r - r_old).view(-1))) / rz
        rz = float(torch.dot(r.view(-1), z.view(-1)))
        p.mul_(beta).add_(z)
    return x - x.mean()


def rel_error(x, ref):
    """|| (x - mean x) - ref || / || ref || for a zero-mean reference."""
    d = x.double() - x.double().mean() - ref
    return float(torch.linalg.vector_norm(d) / torch.linalg.vector_norm(ref))
