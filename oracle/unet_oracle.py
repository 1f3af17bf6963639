"""CPU oracle of the learned preconditioner's network (test infrastructure
only: imported by tests/, never by the product path).

The network has no reference counterpart (the reference's solver is MGPCG
alone); this restates, in numpy, the architecture the device builds in
edgeb200/unet.py, so the device forward pass and its gradients can be checked:

    s  = 1 / rms(r)                       (scale invariance: the network sees r s)
    e0 = relu(c3(relu(c3(r s; W0a)); W0b))               16 channels, full grid
    e1 = relu(c3(relu(c3(pool(e0); W1a)); W1b))          32 channels, 1/2 grid
    e2 = relu(c3(relu(c3(pool(e1); W2a)); W2b))          64 channels, 1/4 grid
    f1 = relu(c3(relu(c3(up(e2); W3a) + c3(e1; W3s)); W3b))
    f0 = relu(c3(relu(c3(up(f1); W4a) + c3(e0; W4s)); W4b))
    z  = c3(f0; W5) / s

c3 = 3x3x3 cross-correlation with zero padding and bias, tap t = 9 (dx+1) +
3 (dy+1) + (dz+1) reading x[v + (dx, dy, dz)]; pool = 2x2x2 mean; up =
nearest 2x.  The device rounds weights and every stored activation to
bfloat16 (round to nearest even) and accumulates in float32; the oracle
applies the same bfloat16 rounding to weights and forward activations and
computes in float64.
"""
import numpy as np

CH = (16, 32, 64)
# (name, out channels, in channels)
LAYERS = [
    ("W0a", CH[0], 1), ("W0b", CH[0], CH[0]),
    ("W1a", CH[1], CH[0]), ("W1b", CH[1], CH[1]),
    ("W2a", CH[2], CH[1]), ("W2b", CH[2], CH[2]),
    ("W3a", CH[1], CH[2]), ("W3s", CH[1], CH[1]), ("W3b", CH[1], CH[1]),
    ("W4a", CH[0], CH[1]), ("W4s", CH[0], CH[0]), ("W4b", CH[0], CH[0]),
    ("W5", 1, CH[0]),
]
# biases: one per conv output, except the skip convs (their sum shares the
# bias of the 'a' conv)
BIASES = ["W0a", "W0b", "W1a", "W1b", "W2a", "W2b", "W3a", "W3b", "W4a", "W4b", "W5"]

ROUND = True  # bfloat16 rounding of weights and activations (off: exact float64 network)


def bf16(x):
    """Round to bfloat16 (nearest even), returned as float64."""
    if not ROUND:
        return np.asarray(x, np.float64)
    a = np.ascontiguousarray(x, dtype=np.float32)
    u = a.view(np.uint32).astype(np.uint64)
    r = ((u + 0x7FFF + ((u >> 16) & 1)) >> 16) << 16
    out = (r & 0xFFFFFFFF).astype(np.uint32).view(np.float32)
    out = np.where(np.isnan(a), a, out)
    return out.astype(np.float64)


def init_params(seed=0):
    """He-style initial weights (float32) and zero biases."""
    rng = np.random.default_rng(seed)
    p = {}
    for name, co, ci in LAYERS:
        std = np.sqrt(2.0 / (27 * ci))
        p[name] = (rng.standard_normal((co, ci, 27)) * std).astype(np.float32)
    for name in BIASES:
        co = dict((n, c) for n, c, _ in LAYERS)[name]
        p["b" + name[1:]] = np.zeros(co, np.float32)
    return p


def _shift(xp, t, shape):
    dx, dy, dz = t // 9 - 1, (t // 3) % 3 - 1, t % 3 - 1
    X, Y, Z = shape
    return xp[:, 1 + dx:1 + dx + X, 1 + dy:1 + dy + Y, 1 + dz:1 + dz + Z]


def conv3(x, W, b=None):
    """x (Ci, X, Y, Z), W (Co, Ci, 27) -> (Co, X, Y, Z), float64."""
    shape = x.shape[1:]
    xp = np.pad(x, ((0, 0), (1, 1), (1, 1), (1, 1)))
    out = np.zeros((W.shape[0],) + shape)
    for t in range(27):
        out += np.einsum("oc,cxyz->oxyz", W[:, :, t], _shift(xp, t, shape), optimize=True)
    if b is not None:
        out += b[:, None, None, None]
    return out


def conv3_bwd(x, W, dy):
    """Gradients of conv3 w.r.t. x and W for upstream dy."""
    shape = x.shape[1:]
    X, Y, Z = shape
    xp = np.pad(x, ((0, 0), (1, 1), (1, 1), (1, 1)))
    dxp = np.zeros_like(xp)
    dW = np.zeros(W.shape)
    for t in range(27):
        dx_, dy_, dz_ = t // 9 - 1, (t // 3) % 3 - 1, t % 3 - 1
        dxp[:, 1 + dx_:1 + dx_ + X, 1 + dy_:1 + dy_ + Y, 1 + dz_:1 + dz_ + Z] += np.einsum(
            "oc,oxyz->cxyz", W[:, :, t], dy, optimize=True)
        dW[:, :, t] = np.einsum("oxyz,cxyz->oc", dy, _shift(xp, t, shape), optimize=True)
    return dxp[:, 1:-1, 1:-1, 1:-1], dW


def pool(x):
    C, X, Y, Z = x.shape
    return x.reshape(C, X // 2, 2, Y // 2, 2, Z // 2, 2).mean(axis=(2, 4, 6))


def pool_bwd(dy):
    return np.repeat(np.repeat(np.repeat(dy, 2, 1), 2, 2), 2, 3) / 8.0


def up(x):
    return np.repeat(np.repeat(np.repeat(x, 2, 1), 2, 2), 2, 3)


def up_bwd(dy):
    C, X, Y, Z = dy.shape
    return dy.reshape(C, X // 2, 2, Y // 2, 2, Z // 2, 2).sum(axis=(2, 4, 6))


def scale_of(r):
    r = np.asarray(r, np.float64)
    return np.float32(1.0 / np.sqrt(np.mean(r * r)))


def forward(p, r):
    """z (float64, same shape as r) and the cache for backward."""
    W = {k: bf16(v) for k, v in p.items() if k.startswith("W")}
    b = {k: np.asarray(v, np.float64) for k, v in p.items() if k.startswith("b")}
    s = scale_of(r)
    c = {"s": s, "W": W}
    x = (np.asarray(r, np.float32) * s)[None].astype(np.float64)
    c["x"] = x

    def layer(name, inp, skip=None, relu=True):
        pre = conv3(inp, W[name], b.get("b" + name[1:]))
        if skip is not None:
            pre = pre + conv3(skip[0], W[skip[1]])
        return bf16(np.maximum(pre, 0.0)) if relu else pre

    c["h0"] = layer("W0a", x)
    c["e0"] = layer("W0b", c["h0"])
    c["d1"] = bf16(pool(c["e0"]))
    c["h1"] = layer("W1a", c["d1"])
    c["e1"] = layer("W1b", c["h1"])
    c["d2"] = bf16(pool(c["e1"]))
    c["h2"] = layer("W2a", c["d2"])
    c["e2"] = layer("W2b", c["h2"])
    c["u1"] = up(c["e2"])
    c["h3"] = layer("W3a", c["u1"], skip=(c["e1"], "W3s"))
    c["f1"] = layer("W3b", c["h3"])
    c["u0"] = up(c["f1"])
    c["h4"] = layer("W4a", c["u0"], skip=(c["e0"], "W4s"))
    c["f0"] = layer("W4b", c["h4"])
    zn = layer("W5", c["f0"], relu=False)[0]
    c["zn"] = zn
    return zn / s, c


def loss_grad(zn, target_n):
    """Mean-removed squared error of the scaled prediction and its gradient
    (the solution of the all-Neumann problem is defined up to a constant)."""
    d = zn - target_n
    d = d - d.mean()
    n = d.size
    return float((d * d).sum() / n), 2.0 * d / n


def backward(p, c, dzn):
    """Parameter gradients for upstream dL/dz_n (z_n = network output before
    the 1/s rescale)."""
    W = c["W"]
    g = {}

    def lin_bwd(name, inp, dout, relu_out=None):
        d = dout if relu_out is None else dout * (relu_out > 0)
        dx, g[name] = conv3_bwd(inp, W[name], d)
        if name in BIASES:
            g["b" + name[1:]] = d.sum(axis=(1, 2, 3))
        return dx

    d_f0 = lin_bwd("W5", c["f0"], dzn[None])
    d_h4r = d_f0 * (c["f0"] > 0)
    d_h4, g["W4b"] = conv3_bwd(c["h4"], W["W4b"], d_h4r)
    g["b4b"] = d_h4r.sum(axis=(1, 2, 3))
    d_h4a = d_h4 * (c["h4"] > 0)
    d_u0, g["W4a"] = conv3_bwd(c["u0"], W["W4a"], d_h4a)
    d_e0_skip, g["W4s"] = conv3_bwd(c["e0"], W["W4s"], d_h4a)
    g["b4a"] = d_h4a.sum(axis=(1, 2, 3))
    d_f1 = up_bwd(d_u0)
    d_h3 = lin_bwd("W3b", c["h3"], d_f1, c["f1"])
    d_h3a = d_h3 * (c["h3"] > 0)
    d_u1, g["W3a"] = conv3_bwd(c["u1"], W["W3a"], d_h3a)
    d_e1_skip, g["W3s"] = conv3_bwd(c["e1"], W["W3s"], d_h3a)
    g["b3a"] = d_h3a.sum(axis=(1, 2, 3))
    d_e2 = up_bwd(d_u1)
    d_h2 = lin_bwd("W2b", c["h2"], d_e2, c["e2"])
    d_d2 = lin_bwd("W2a", c["d2"], d_h2, c["h2"])
    d_e1 = pool_bwd(d_d2) + d_e1_skip
    d_h1 = lin_bwd("W1b", c["h1"], d_e1, c["e1"])
    d_d1 = lin_bwd("W1a", c["d1"], d_h1, c["h1"])
    d_e0 = pool_bwd(d_d1) + d_e0_skip
    d_h0 = lin_bwd("W0b", c["h0"], d_e0, c["e0"])
    lin_bwd("W0a", c["x"], d_h0, c["h0"])
    return g
