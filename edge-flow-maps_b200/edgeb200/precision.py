"""FP64 reference solves for the precision study (no reference counterpart).

The mixed-precision solver (Projection(..., precision=1)) stores the
V-cycle's level arrays in bfloat16 while the CG vectors, the residual and
the arithmetic stay float32 and the dot products float64.  Its error, and
that of the float32 solver, is measured against an FP64 solve of the same
system: flexible CG in float64 (vectors, operator, dot products) whose
preconditioner is the float32 V-cycle; preconditioner rounding only slows
convergence, the float64 recursion sets the accuracy.
"""
import torch

from . import _native as N
from .fields import ptr_any, stream

F64 = (torch.float64,)


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
