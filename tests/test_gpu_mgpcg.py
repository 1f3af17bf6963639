"""MGPCG projection (sim/mgpcg.py, sim/mgpcg_solid.py) on the device against
the golden vectors and the oracle.

The reference's dot products are float32 atomics (order-nondeterministic);
the device solver and the oracle sum in float64, so CG iterates differ by
rounding: iteration counts may differ by one and converged fields are
compared with 1e-4 relative L2; the divergence left after projection must be
at the solver tolerance.
"""
import numpy as np
import pytest
import torch

from conftest import load_golden, rel_l2
from oracle import edge_oracle as O

pytestmark = pytest.mark.gpu


def T_(a, dtype=np.float32):
    return torch.from_numpy(np.ascontiguousarray(a, dtype=dtype)).cuda()


def N_(t):
    torch.cuda.synchronize()
    return t.detach().cpu().numpy()


def div_of(u):
    ux, uy, uz = u
    return (ux[1:] - ux[:-1]) + (uy[:, 1:] - uy[:, :-1]) + (uz[:, :, 1:] - uz[:, :, :-1])


def test_poisson_golden():
    from sim.mgpcg import MGPCG_3
    d = load_golden("mgpcg_plain")
    res = tuple(int(v) for v in d["res"])
    s = MGPCG_3([[2, 2], [2, 2], [2, 2]], list(res), base_level=1)
    assert s.n_mg_levels == int(d["meta_levels"])
    u = [T_(d["u_in_" + a]) for a in "xyz"]
    s.Poisson(*u)
    it, err, st = s.last_result()
    assert st == 0
    assert abs(it - int(d["meta_iters"])) <= 1
    for i, a in enumerate("xyz"):
        assert rel_l2(N_(u[i]), d["u_out_" + a]) < 1e-4
    assert rel_l2(N_(s.u_div), d["div"]) < 1e-6


def test_vcycle_and_operator_golden():
    from edgeb200.projection import Projection
    d = load_golden("mgpcg_plain")
    res = tuple(int(v) for v in d["res"])
    P = Projection(res, base_level=1)
    r = T_(d["vc_rhs"])
    z = torch.empty_like(r)
    P.vcycle(r, z)
    assert rel_l2(N_(z), d["vc_z"]) < 1e-5
    Ap = torch.empty_like(r)
    P.apply_A(r, Ap)
    assert rel_l2(N_(Ap), d["ap_out"]) < 1e-6


def test_solid_golden():
    from sim.mgpcg_solid import MGPCG_Solid_3
    d = load_golden("mgpcg_solid")
    res = tuple(int(v) for v in d["res"])
    mask = T_(d["mask"], np.int32)
    bvel = T_(d["bvel"])
    s = MGPCG_Solid_3([[2, 2], [2, 2], [2, 2]], mask, bvel, list(res), base_level=1)
    u = [T_(d["u_in_" + a]) for a in "xyz"]
    s.Poisson(*u)
    it, err, st = s.last_result()
    assert st == 0
    assert abs(it - int(d["meta_iters"])) <= 1
    for i, a in enumerate("xyz"):
        assert rel_l2(N_(u[i]), d["u_out_" + a]) < 1e-4
    assert rel_l2(N_(s.u_div), d["div"]) < 1e-5


# (128, 64, 64) runs two levels outside the shared-memory coarse group (the
# restriction then also applies the coarse level's first half sweep);
# (48, 24, 24) ends on a 6x3x3 level (an odd row length); the open x
# boundaries take the path without recentering.
@pytest.mark.parametrize("res,base_level,bt", [((64, 32, 32), 2, None), ((64, 32, 32), 3, None),
                                               ((32, 32, 16), 1, None), ((128, 64, 64), 2, None),
                                               ((48, 24, 24), 1, None), ((64, 32, 32), 2, ((1, 1), (2, 2), (2, 2)))])
def test_poisson_vs_oracle(res, base_level, bt):
    from edgeb200.projection import Projection
    bt = bt or ((2, 2), (2, 2), (2, 2))
    rng = np.random.default_rng(sum(res) + base_level)
    u = [rng.normal(size=s).astype(np.float32) for s in O.face_shapes(res)]
    uo = [a.copy() for a in u]
    it_o, div_o, p_o, rtr_o = O.poisson(uo, base_level=base_level, boundary_types=bt)
    P = Projection(res, base_level=base_level, boundary_types=bt)
    ug = [T_(a) for a in u]
    P.poisson(*ug)
    it, rtr, st = P.result()
    assert st == 0 and it_o >= 0
    assert abs(it - it_o) <= 1
    for i in range(3):
        assert rel_l2(N_(ug[i]), uo[i]) < 1e-4
    # the divergence left by the projection is the CG residual (stopped
    # below the solver's tolerance on the recursion) plus one float32
    # rounding of each stored face value
    got = [N_(t).astype(np.float64) for t in ug]
    d = np.sqrt((div_of(got) ** 2).sum())
    a = [np.abs(t) for t in got]
    floor = 2.0 ** -24 * np.sqrt(((a[0][1:] + a[0][:-1] + a[1][:, 1:] + a[1][:, :-1] + a[2][:, :, 1:]
                                   + a[2][:, :, :-1]) ** 2).sum())
    assert d <= np.sqrt(rtr) + 4 * floor, (d, rtr, floor)


@pytest.mark.parametrize("res,base_level", [((128, 64, 64), 2), ((48, 24, 24), 1)])
def test_vcycle_vs_oracle(res, base_level):
    """One preconditioner application against the oracle's V-cycle."""
    from edgeb200.projection import Projection
    rng = np.random.default_rng(11)
    r = rng.normal(size=res).astype(np.float32)
    z_o, ap_o, L = O.vcycle(r, base_level)
    P = Projection(res, base_level=base_level)
    assert P.levels == L
    z = torch.empty(res, device="cuda")
    P.vcycle(T_(r), z)
    assert rel_l2(N_(z), z_o) < 1e-5


def test_solid_vs_oracle():
    """Solid solver with two levels outside the shared-memory coarse group: a
    wedge-shaped obstacle moving with a constant velocity."""
    from edgeb200.projection import Projection
    res = (128, 64, 64)
    rng = np.random.default_rng(11)
    i, j, k = np.meshgrid(*(np.arange(n) for n in res), indexing="ij")
    mask = ((np.abs(j - 32) < (i - 20) * 0.6) & (i > 20) & (i < 60)).astype(np.int32)
    bvel = np.zeros(res + (3,), np.float32)
    bvel[..., 0] = 0.25
    u = [rng.normal(size=s).astype(np.float32) for s in O.face_shapes(res)]
    uo = [a.copy() for a in u]
    # r.r < 1e-6: the reference's 1e-12 on this grid is below float32
    # resolution of the initial residual, where iteration counts depend on
    # rounding
    it_o, div_o, p_o, bm1, bm2, dsum = O.poisson_solid(uo, mask, bvel, base_level=2, tol=1e-6)
    P = Projection(res, base_level=2, mask=T_(mask, np.int32), bvel=T_(bvel))
    ug = [T_(a) for a in u]
    P.poisson(*ug, abs_tol=1e-6, rel_tol=0.0, max_iters=100)
    it, rtr, st = P.result()
    assert it_o > 0 and st == 0
    assert abs(it - it_o) <= 1
    for a in range(3):
        assert rel_l2(N_(ug[a]), uo[a]) < 1e-4


def test_graph_reuse_and_repeat():
    """Repeated solves reuse the captured graph and give identical results."""
    from edgeb200.projection import Projection
    rng = np.random.default_rng(1)
    res = (32, 16, 16)
    P = Projection(res, base_level=2)
    u0 = [rng.normal(size=s).astype(np.float32) for s in O.face_shapes(res)]
    outs = []
    for _ in range(3):
        u = [T_(a) for a in u0]
        P.poisson(*u)
        outs.append([N_(t) for t in u])
        assert P.result()[2] == 0
    for o in outs[1:]:
        for a, b in zip(o, outs[0]):
            np.testing.assert_array_equal(a, b)


def test_max_iters_and_nan_status():
    """Non-convergence and non-finite residuals end the device loop with a
    status (no hang)."""
    from edgeb200 import EDGE_ENAN, EDGE_ENOCONV
    from edgeb200.projection import Projection
    rng = np.random.default_rng(2)
    res = (32, 16, 16)
    P = Projection(res, base_level=2)
    u = [T_(rng.normal(size=s)) for s in O.face_shapes(res)]
    P.poisson(*u, abs_tol=0.0, rel_tol=0.0, max_iters=3)
    it, rtr, st = P.result()
    assert st == EDGE_ENOCONV and it == 3
    u = [T_(rng.normal(size=s)) for s in O.face_shapes(res)]
    u[0][5, 5, 5] = float("nan")
    P.poisson(*u)
    it, rtr, st = P.result()
    assert st == EDGE_ENAN


def test_solve_rhs():
    """edge_mgpcg_solve: A x = b - mean(b) for the all-Neumann operator."""
    from edgeb200.projection import Projection
    rng = np.random.default_rng(4)
    res = (32, 32, 16)
    P = Projection(res, base_level=2)
    b = rng.normal(size=res).astype(np.float32)
    b -= b.mean()
    x = torch.zeros(res, device="cuda")
    P.solve(T_(b), x)
    assert P.result()[2] == 0
    Ax = torch.empty_like(x)
    P.apply_A(x, Ax)
    assert rel_l2(N_(Ax), b) < 1e-5


def test_poisson_with_buffer():
    from sim.mgpcg import MGPCG_3
    rng = np.random.default_rng(6)
    res = (32, 16, 16)
    s = MGPCG_3([[2, 2], [2, 2], [2, 2]], list(res), base_level=2)
    u0 = [rng.normal(size=sh).astype(np.float32) for sh in O.face_shapes(res)]
    u = [T_(a) for a in u0]
    f = [torch.zeros_like(t) for t in u]
    s.Poisson_with_buffer(*u, *f)
    uo = [a.copy() for a in u0]
    fo = [np.zeros_like(a) for a in u0]
    O.poisson(uo, base_level=2, force=fo)
    for i in range(3):
        assert rel_l2(N_(f[i]), fo[i]) < 1e-4
        assert rel_l2(N_(u[i]), uo[i]) < 1e-4


@pytest.mark.parametrize("precision,vtol", [(1, 3e-2), (2, 4e-3)])
@pytest.mark.parametrize("amp", [1.0, 1e-7])
def test_mixed_precision_vs_fp64(precision, vtol, amp):
    """BF16 (precision=1) or FP16 (precision=2, scaled by a power of two)
    V-cycle storage: one V-cycle within the storage format's rounding of the
    float32 one, and solves to 1e-6 whose error against an FP64 solve is of
    the float32 solver's size.  The tiny amplitude would underflow FP16
    without the scaling."""
    from edgeb200.precision import fp64_solve, rel_error
    from edgeb200.projection import Projection
    res = (128, 64, 64)
    g = torch.Generator().manual_seed(21)
    b = torch.randn(res, generator=g) * amp
    b = (b - b.mean()).cuda()
    P32 = Projection(res, base_level=1)
    P16 = Projection(res, base_level=1, precision=precision)
    z32, z16 = torch.empty_like(b), torch.empty_like(b)
    P32.vcycle(b, z32)
    P16.vcycle(b, z16)
    assert rel_l2(N_(z16), N_(z32)) < vtol
    if amp != 1.0:
        # the solve's tolerance semantics (an absolute eps of 1e-12 in the
        # step sizes, mgpcg.py:238, 272) are not scale-free: solve at O(1)
        return
    ref = fp64_solve(P32, b)
    bb = float((b.double() ** 2).sum())
    errs, its = [], []
    for P in (P32, P16):
        x = torch.zeros(res, device="cuda")
        P.solve(b, x, abs_tol=1e-12 * bb, rel_tol=0.0)
        it, rtr, st = P.result()
        assert st == 0
        its.append(it)
        errs.append(rel_error(x, ref))
    assert its[1] <= its[0] + 2
    assert errs[0] < 1e-3 and errs[1] < 3 * errs[0] + 1e-6, errs


_EAGER_SCRIPT = r"""
import sys
import numpy as np, torch
sys.path[:0] = [sys.argv[2], sys.argv[3]]
from edgeb200.projection import Projection
res = (128, 64, 64)
rng = np.random.default_rng(3)
u = [torch.from_numpy(rng.normal(size=s).astype(np.float32)).cuda()
     for s in ((129, 64, 64), (128, 65, 64), (128, 64, 65))]
P = Projection(res, base_level=2)
P.poisson(*u)
it, rtr, st = P.result()
np.savez(sys.argv[1], ux=u[0].cpu().numpy(), uy=u[1].cpu().numpy(), uz=u[2].cpu().numpy(),
         res=np.array([it, st]), rtr=np.array(rtr))
"""


def test_host_driven_loop_matches_graph(tmp_path):
    """The host-driven CG loop (EDGE_MGPCG_EAGER=1: one status read per
    iteration) gives the graph-captured solve's result bit for bit.  The
    switch is read once per process, so each runs in a child process."""
    import os
    import subprocess
    import sys
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    pkg = os.path.join(root, "edge-flow-maps_b200")
    outs = {}
    for eager in ("0", "1"):
        path = str(tmp_path / f"e{eager}.npz")
        env = dict(os.environ, EDGE_MGPCG_EAGER=eager)
        subprocess.run([sys.executable, "-c", _EAGER_SCRIPT, path, pkg, root], env=env, check=True, timeout=600)
        outs[eager] = np.load(path)
    ref = outs["0"]
    assert int(ref["res"][1]) == 0
    for k, d in outs.items():
        for f in ("ux", "uy", "uz", "res", "rtr"):
            np.testing.assert_array_equal(d[f], ref[f], err_msg=f"{f} {k}")


@pytest.mark.parametrize("precision", [0, 1, 2])
def test_refined_solve_reaches_true_tolerance(precision):
    """Iterative refinement (float64 residual and iterate on the device,
    float32/BF16/FP16 inner V-cycle-PCG solves) brings the TRUE relative
    residual below 1e-6, where the float32 recursion alone stops above it,
    and the result matches the FP64 solve."""
    from edgeb200.precision import RefinedSolver, fp64_solve, rel_error
    from edgeb200.projection import Projection
    res = (128, 64, 64)
    g = torch.Generator().manual_seed(5)
    b = torch.randn(res, generator=g, dtype=torch.float64)
    b = (b - b.mean()).cuda()
    P = Projection(res, base_level=2, precision=precision)
    R = RefinedSolver(P, inner_rel=1e-2)
    x = R.solve(b, rel_tol=1e-6)
    assert R.stats["true_rel_residual"] <= 1e-6, R.stats
    assert 1 <= R.stats["outer"] <= 8, R.stats
    # the float64 residual recomputed independently
    Ax = torch.empty_like(x)
    from edgeb200.precision import apply_A64
    apply_A64(P, x, Ax)
    true = float((b - Ax).norm() / b.norm())
    assert true <= 1.01e-6, true
    ref = fp64_solve(P, b.float())
    assert rel_error(x.float(), ref) < 1e-4


def test_solve_writes_each_callers_output():
    """Solves of the same right-hand side into two different output
    tensors each write their own output (the captured solve graph is keyed
    by the output pointer as well)."""
    from edgeb200.projection import Projection
    res = (64, 32, 32)
    g = torch.Generator().manual_seed(2)
    b = torch.randn(res, generator=g)
    b = (b - b.mean()).cuda()
    P = Projection(res, base_level=2)
    x1 = torch.zeros(res, device="cuda")
    x2 = torch.zeros(res, device="cuda")
    P.solve(b, x1, abs_tol=0.0, rel_tol=1e-12)
    P.solve(b, x2, abs_tol=0.0, rel_tol=1e-12)
    torch.cuda.synchronize()
    assert float(x2.abs().max()) > 0
    assert torch.equal(x1, x2)


_PAIR_SCRIPT = r"""
import sys
import numpy as np, torch
sys.path[:0] = [sys.argv[2], sys.argv[3]]
from edgeb200.projection import Projection
out = {}
cases = [((128, 64, 64), 2, 0, False), ((128, 64, 64), 2, 1, False), ((128, 64, 64), 2, 2, False),
         ((128, 64, 64), 2, 0, True), ((128, 64, 64), 2, 1, True), ((200, 72, 24), 1, 0, False),
         ((200, 72, 24), 1, 2, True)]
for n, (res, base, prec, solid) in enumerate(cases):
    rng = np.random.default_rng(20 + n)
    kw = {}
    if solid:
        i, j, k = np.meshgrid(*(np.arange(m) for m in res), indexing="ij")
        mask = ((np.abs(j - res[1] // 2) < (i - 20) * 0.6) & (i > 20) & (i < 60) & (k > 2)).astype(np.int32)
        bvel = np.zeros(res + (3,), np.float32)
        bvel[..., 0] = 0.25
        kw = dict(mask=torch.from_numpy(mask).cuda(), bvel=torch.from_numpy(bvel).cuda())
    shapes = [(res[0] + 1, res[1], res[2]), (res[0], res[1] + 1, res[2]), (res[0], res[1], res[2] + 1)]
    u = [torch.from_numpy(rng.normal(size=s).astype(np.float32)).cuda() for s in shapes]
    P = Projection(res, base_level=base, precision=prec, **kw)
    P.poisson(*u, abs_tol=1e-9, rel_tol=1e-9, max_iters=60)
    it, rtr, st = P.result()
    for a in range(3):
        out[f"u{a}_{n}"] = u[a].cpu().numpy()
    out[f"res_{n}"] = np.array([it, st])
    out[f"rtr_{n}"] = np.array(rtr)
    out[f"kernels_{n}"] = np.array(P.kernel_count())
    P.close()
np.savez(sys.argv[1], **out)
"""


def test_fused_half_sweep_pairs_match_unfused(tmp_path):
    """The V-cycle's half sweeps fused in pairs (k_hs_pair: a shared-memory
    tile with a two-row halo, the second sweep written to a third z plane)
    give the unfused sweeps' result bit for bit: FP32, BF16 and FP16 level
    storage, plain and solid solvers, and a ragged grid whose tiles overhang
    the level and whose second level has no four-slot layout.  The switch is
    read once per process, so each tile shape runs in a child process."""
    import os
    import subprocess
    import sys
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    pkg = os.path.join(root, "edge-flow-maps_b200")
    outs = {}
    for mode in ("0", "1", "2", "3"):
        path = str(tmp_path / f"p{mode}.npz")
        env = dict(os.environ, EDGE_MGPCG_PAIR=mode)
        subprocess.run([sys.executable, "-c", _PAIR_SCRIPT, path, pkg, root], env=env, check=True, timeout=900)
        outs[mode] = np.load(path)
    ref = outs["0"]
    for n in range(7):
        assert int(ref[f"res_{n}"][0]) > 2
    for mode, d in outs.items():
        for f in ref.files:
            if f.startswith("kernels"):
                continue
            np.testing.assert_array_equal(d[f], ref[f], err_msg=f"{f} mode {mode}")
        # fewer launches per V-cycle when the pairs run
        if mode != "0":
            assert int(d["kernels_0"]) < int(ref["kernels_0"]), (mode, int(d["kernels_0"]), int(ref["kernels_0"]))
