"""Learned preconditioner on the device: the tensor-core building blocks, the
network's forward pass and its parameter gradients against the CPU oracle
(oracle/unet_oracle.py), and a few training steps."""
import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


def _U():
    from oracle import unet_oracle as U
    return U


@pytest.mark.parametrize("mode", [0, 1])
@pytest.mark.parametrize("n,k", [(16, 16), (32, 64), (64, 128), (128, 32)])
def test_tc_selftest(mode, n, k):
    from edgeb200.unet import tc_selftest
    g = torch.Generator(device="cpu").manual_seed(n * 1000 + k + mode)
    m = 128 if mode == 0 else 64
    if mode == 0:
        A = torch.randn(m, k, generator=g).to(torch.bfloat16).cuda()
        B = torch.randn(n, k, generator=g).to(torch.bfloat16).cuda()
        ref = A.float() @ B.float().T
    else:
        A = torch.randn(k, m, generator=g).to(torch.bfloat16).cuda()
        B = torch.randn(k, n, generator=g).to(torch.bfloat16).cuda()
        ref = A.float().T @ B.float()
    D, timed_out = tc_selftest(mode, A, B)
    assert not timed_out
    # bf16 products are exact in fp32; only the summation order differs
    assert torch.allclose(D, ref, rtol=1e-5, atol=1e-4 * k ** 0.5)


def _packed(w, co, ci, transpose=0):
    from edgeb200 import _native as N
    from edgeb200 import unet as UN
    from edgeb200.fields import ptr, ptr_any, stream
    out = torch.empty(co * ci * 27, dtype=torch.bfloat16, device="cuda")
    N.call("edge_unet_pack_weights", ptr(w.contiguous()), co, ci, transpose, ptr_any(out, UN.BF16), stream())
    return out


def _rel(a, b):
    return np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-30)


@pytest.mark.parametrize("res,cin,cout,two,flags", [((8, 8, 8), 16, 16, False, 1), ((12, 8, 16), 32, 64, False, 1),
                                                     ((16, 12, 8), 64, 32, True, 1), ((8, 16, 8), 16, 16, True, 0),
                                                     ((8, 8, 12), 32, 16, False, 2)])
def test_conv_vs_oracle(res, cin, cout, two, flags):
    from edgeb200 import unet as UN
    U = _U()
    g = torch.Generator().manual_seed(sum(res) + cin + cout)
    x0 = torch.randn(cin, *res, generator=g)
    W0 = torch.randn(cout, cin, 27, generator=g) * (2.0 / (27 * cin)) ** 0.5
    b = torch.randn(cout, generator=g) * 0.1
    a0 = UN.Act(res, cin)
    UN.dense_to_act(x0.cuda(), a0)
    net = UN.UNet((4, 4, 4))  # its launch helper and error flag
    net.packed["T0"] = _packed(W0.cuda(), cout, cin)
    a1 = None
    if two:
        c1 = 32 if cout > 16 else 16
        x1 = torch.randn(c1, *res, generator=g)
        W1 = torch.randn(cout, c1, 27, generator=g) * (2.0 / (27 * c1)) ** 0.5
        a1 = UN.Act(res, c1)
        UN.dense_to_act(x1.cuda(), a1)
        net.packed["T1"] = _packed(W1.cuda(), cout, c1)
    y = UN.Act(res, cout)
    y0 = torch.randn(cout, *res, generator=g)
    if flags & 2:
        UN.dense_to_act(y0.cuda(), y)
    net._conv(res, a0, "T0", a1, "T1" if two else None, cout, b.cuda(), flags, y)
    torch.cuda.synchronize()
    assert not net.timed_out()
    got = UN.act_to_dense(y).cpu().numpy()
    ref = U.conv3(U.bf16(x0.numpy()), U.bf16(W0.numpy()), b.numpy().astype(np.float64))
    if two:
        ref = ref + U.conv3(U.bf16(x1.numpy()), U.bf16(W1.numpy()))
    if flags & 1:
        ref = np.maximum(ref, 0.0)
    if flags & 2:
        ref = ref + U.bf16(y0.numpy())
    ref = U.bf16(ref)
    assert _rel(got, ref) < 4e-3
    # everything outside the interior stays zero
    total = y.t.float().abs().sum().item()
    assert abs(total - np.abs(got).sum()) <= 1e-3 * max(1.0, total)


@pytest.mark.parametrize("res,cin,cout", [((8, 8, 8), 16, 16), ((8, 12, 8), 32, 64), ((12, 8, 8), 64, 32)])
def test_dgrad_and_wgrad_vs_oracle(res, cin, cout):
    """Data gradient (transposed tap-flipped packing) and weight gradient
    (M = 64 MN-major tensor-core kernel) of one convolution."""
    from edgeb200 import _native as N
    from edgeb200 import unet as UN
    from edgeb200.fields import ptr, ptr_any, stream
    U = _U()
    g = torch.Generator().manual_seed(3 * cin + cout)
    x = torch.randn(cin, *res, generator=g)
    d = torch.randn(cout, *res, generator=g)
    W = torch.randn(cout, cin, 27, generator=g) * 0.1
    ax, ad = UN.Act(res, cin), UN.Act(res, cout)
    UN.dense_to_act(x.cuda(), ax)
    UN.dense_to_act(d.cuda(), ad)
    net = UN.UNet((4, 4, 4))
    net.packed_t["T"] = _packed(W.cuda(), cout, cin, 1)
    dx = UN.Act(res, cin)
    net._conv(res, ad, "T", None, None, cin, None, 0, dx, table=net.packed_t)
    nsplit = 5
    partial = torch.zeros(nsplit * 27 * cout * cin, device="cuda")
    dw = torch.zeros(cout, cin, 27, device="cuda")
    N.call("edge_unet_wgrad", *res, ad.p, cout, ax.p, cin, ptr(partial), nsplit, ptr(dw), ptr_any(net.err, UN.I32),
           stream())
    torch.cuda.synchronize()
    assert not net.timed_out()
    ref_dx, ref_dw = U.conv3_bwd(U.bf16(x.numpy()), U.bf16(W.numpy()), U.bf16(d.numpy()))
    assert _rel(UN.act_to_dense(dx).cpu().numpy(), U.bf16(ref_dx)) < 4e-3
    assert _rel(dw.cpu().numpy(), ref_dw) < 1e-4


def _params_np(seed):
    U = _U()
    p = U.init_params(seed)
    rng = np.random.default_rng(seed + 100)
    for k in p:
        if k.startswith("b"):
            p[k] = (rng.standard_normal(p[k].shape) * 0.05).astype(np.float32)
    return p


@pytest.mark.parametrize("res", [(16, 16, 16), (32, 24, 16)])
def test_forward_vs_oracle(res):
    from edgeb200 import unet as UN
    U = _U()
    p = _params_np(5)
    r = np.random.default_rng(7).standard_normal(res).astype(np.float32)
    z_ref, _ = U.forward(p, r)
    net = UN.UNet(res, params={k: torch.from_numpy(v).cuda() for k, v in p.items()})
    z = torch.empty(res, device="cuda")
    net.forward(torch.from_numpy(r).cuda(), z)
    torch.cuda.synchronize()
    assert not net.timed_out()
    assert _rel(z.cpu().numpy(), z_ref) < 3e-2


def test_gradients_vs_oracle():
    """Every parameter gradient of the device backward pass against the
    oracle's (bf16 activations and gradients on the device: a few percent)."""
    from edgeb200 import unet as UN
    U = _U()
    res = (16, 16, 16)
    p = _params_np(9)
    rng = np.random.default_rng(11)
    r = rng.standard_normal(res).astype(np.float32)
    x = rng.standard_normal(res).astype(np.float32)
    _, c = U.forward(p, r)
    loss_ref, dzn = U.loss_grad(c["zn"], x.astype(np.float64) * c["s"])
    g_ref = U.backward(p, c, dzn)
    net = UN.UNet(res, params={k: torch.from_numpy(v).cuda() for k, v in p.items()})
    loss = net.loss_and_grad(torch.from_numpy(r).cuda(), torch.from_numpy(x).cuda())
    torch.cuda.synchronize()
    assert not net.timed_out()
    assert abs(loss.item() - loss_ref) <= 2e-2 * loss_ref
    bad = {}
    scale = max(np.linalg.norm(v) for v in g_ref.values())
    for k, gr in g_ref.items():
        got = net.grads[k].cpu().numpy().reshape(gr.shape)
        if np.linalg.norm(gr) < 1e-6 * scale:  # b5: dL/dz_n is mean-free, its sum is 0
            if np.linalg.norm(got) > 1e-4 * scale:
                bad[k] = np.linalg.norm(got)
        elif _rel(got, gr) >= 6e-2:
            bad[k] = _rel(got, gr)
    assert not bad, bad


def test_training_reduces_loss():
    """A few Adam steps on one (r, x) pair lower the loss."""
    from edgeb200 import unet as UN
    res = (16, 16, 16)
    g = torch.Generator().manual_seed(2)
    r = torch.randn(res, generator=g).cuda()
    x = torch.randn(res, generator=g).cuda()
    net = UN.UNet(res, seed=1)
    losses = [net.train_step(r, x, lr=3e-3).item() for _ in range(30)]
    assert not net.timed_out()
    assert losses[-1] < 0.8 * losses[0]


def test_learned_preconditioner_gain():
    """The shipped weights (trained on the GPU by edgeb200.train_unet from
    plain-MGPCG solves at 128x64x64) warm-start the V-cycle well enough that
    flexible CG needs fewer iterations to 1e-6 than with the plain V-cycle, on
    right-hand sides it was not trained on."""
    import os
    from edgeb200 import unet as UN
    from edgeb200.projection import Projection
    from edgeb200.train_unet import evaluate, load_params
    w = os.path.join(os.path.dirname(UN.__file__), "weights", "unet_pcg.npz")
    out = evaluate(load_params(w), sizes=((128, 64, 64),), seeds=(1, 2, 3))["128x64x64"]
    assert all(a < b for a, b in zip(out["warm"], out["vcycle"])), out


def test_forward_and_gradients_are_deterministic():
    """The forward pass, the loss and every parameter gradient are
    bit-identical run to run (fixed-order reductions, no float atomics)."""
    from edgeb200 import unet as UN
    res = (32, 24, 16)
    g = torch.Generator().manual_seed(4)
    r = torch.randn(res, generator=g).cuda()
    x = torch.randn(res, generator=g).cuda()
    outs = []
    for _ in range(2):
        net = UN.UNet(res, seed=3)
        z = torch.empty(res, device="cuda")
        net.forward(r, z)
        loss = net.loss_and_grad(r, x)
        torch.cuda.synchronize()
        assert not net.timed_out()
        outs.append((z.clone(), loss.clone(), {k: v.clone() for k, v in net.grads.items()}))
    assert torch.equal(outs[0][0], outs[1][0]) and torch.equal(outs[0][1], outs[1][1])
    for k in outs[0][2]:
        assert torch.equal(outs[0][2][k], outs[1][2][k]), k


@pytest.mark.parametrize("precision", [0, 2])
def test_stepwise_solve_matches_graph_solve(precision):
    """The stepwise solve with the built-in coarse group (the learned
    solver's frame: set-up, then per iteration a coarse step and the
    cooperative iteration kernel) gives the graph-captured solve's result
    and iteration count bit for bit; the level-lc residual round-trips
    through the cell-array I/O."""
    from edgeb200.projection import Projection
    from edgeb200.unet import LearnedCoarsePCG
    res = (128, 64, 64)
    g = torch.Generator().manual_seed(8)
    b = torch.randn(res, generator=g)
    b = (b - b.mean()).cuda()
    bb = float((b.double() ** 2).sum())
    P = Projection(res, base_level=2, precision=precision)
    x0 = torch.zeros(res, device="cuda")
    P.solve(b, x0, abs_tol=1e-12 * bb, rel_tol=0.0)
    ref = P.result()
    L = LearnedCoarsePCG(P, None)
    assert L.dims == (32, 16, 16)
    x1 = torch.zeros(res, device="cuda")
    it, rtr, st, fell = L.solve(b, x1, abs_tol=1e-12 * bb, rel_tol=0.0, mode="vcycle")
    assert (it, st) == (ref[0], ref[2]) and rtr == ref[1] and not fell
    assert torch.equal(x0, x1)
    # level-lc residual: cell array -> planes -> cell array is exact in float32
    P.solve_begin(b, abs_tol=1e-12 * bb, rel_tol=0.0)
    r = torch.empty(L.dims, device="cuda")
    P.coarse_get_r(r)
    P.coarse_set_z(r)
    P.coarse_default()
    torch.cuda.synchronize()
    assert float(r.abs().max()) > 0


def test_learned_coarse_solver_converges_with_fallback():
    """With untrained weights the network is a poor coarse solver: the solve
    still reaches the tolerance (the stall test hands it to the built-in
    coarse group when needed) and reports the status of the plain solver."""
    from edgeb200.projection import Projection
    from edgeb200.unet import LearnedCoarsePCG, init_params
    res = (128, 64, 64)
    g = torch.Generator().manual_seed(9)
    b = torch.randn(res, generator=g)
    b = (b - b.mean()).cuda()
    bb = float((b.double() ** 2).sum())
    P = Projection(res, base_level=2)
    L = LearnedCoarsePCG(P, init_params(3))
    x = torch.zeros(res, device="cuda")
    it, rtr, st, fell = L.solve(b, x, abs_tol=1e-12 * bb, rel_tol=0.0, mode="net")
    assert st == 0 and rtr < 1e-12 * bb
    Ax = torch.empty_like(x)
    P.apply_A(x, Ax)
    assert float((Ax - b).norm() / b.norm()) < 1e-5


def test_edge_steps_with_learned_coarse_solver():
    """EdgeSim(learned=...): both projections of every step run MGPCG with
    the network as the coarse group (untrained weights here, so the stall
    fallback is exercised); the steps converge and track the plain steps to
    the solver tolerance's reach."""
    from edgeb200.sim import EdgeSim, leapfrog_init
    from edgeb200.unet import init_params
    res, dx = (128, 64, 64), 1.0 / 64
    u, smoke = leapfrog_init(res, dx, radii=(0.21, 0.28), sigma=0.03, circulation=1.0)
    sims = [EdgeSim(res, dx, variant="edge", reinit_every=12, base_level=2, visualize_dt=1e9, learned=p)
            for p in (None, init_params(5))]
    for s in sims:
        s.set_velocity(*u)
        s.set_smoke(smoke)
    for i in range(3):
        for s in sims:
            s.step()
        assert sims[1].proj.result()[2] == 0
        for c in range(3):
            a, b = sims[1].u[c].double(), sims[0].u[c].double()
            assert float((a - b).norm() / b.norm()) < 2e-3, (i, c)
