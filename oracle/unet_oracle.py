"""NumPy restatement of the learned preconditioner's U-Net -- TEST
INFRASTRUCTURE ONLY (the checker of the GPU forward / backward kernels in
cpu-free-model_b200/csrc/learned.cu; never part of the product).

The network has no reference counterpart (the reference has no learned or
tensor-core code).  Architecture, 4 levels L0..L3 at H/2^l x W/2^l with
32 / 64 / 128 / 256 channels:

    h0 = relu(cin(x))             2 -> 32    L0
    h1 = relu(e1(pool(h0)))      32 -> 64    L1
    h2 = relu(e2(pool(h1)))      64 -> 128   L2
    h3 = relu(e3(pool(h2)))     128 -> 256   L3
    g3 = relu(d3(h3))           256 -> 128   L3
    g2 = relu(d2(up(g3) + h2))  128 -> 64    L2
    g1 = relu(d1(up(g2) + h1))   64 -> 32    L1
    g0 = relu(d0(up(g1) + h0))   32 -> 32    L0
    out = cout(g0)               32 -> 1     L0

All convolutions 3x3, zero padding 1, with bias; pool = 2x2 mean, up =
nearest.  Parameters are one flat FP32 vector in LAYERS order, each layer
its weight [9][Cout][Cin] (tap = 3 dy + dx) then its bias [Cout].

Evaluated in float64; `bf16` rounds the tensors the GPU stores in BF16 (the
tensor-core convolution operands and every activation) so that the oracle
sees the values the GPU sees.
"""
import numpy as np

LAYERS = [("cin", 2, 32), ("e1", 32, 64), ("e2", 64, 128), ("e3", 128, 256),
          ("d3", 256, 128), ("d2", 128, 64), ("d1", 64, 32), ("d0", 32, 32), ("cout", 32, 1)]
TC_LAYERS = {"e1", "e2", "e3", "d3", "d2", "d1", "d0"}


def num_params():
    return sum(9 * co * ci + co for _, ci, co in LAYERS)


def unpack(theta):
    out, o = {}, 0
    for name, ci, co in LAYERS:
        w = theta[o:o + 9 * co * ci].reshape(9, co, ci)
        o += 9 * co * ci
        b = theta[o:o + co]
        o += co
        out[name] = (w, b)
    return out


def bf16(a):
    u = np.ascontiguousarray(a, np.float32).view(np.uint32).astype(np.uint64)
    u = ((u + 0x7FFF + ((u >> 16) & 1)) >> 16) << 16
    return u.astype(np.uint32).view(np.float32).astype(np.float64)


def conv(x, w, b):
    B, H, W, _ = x.shape
    xp = np.pad(x, ((0, 0), (1, 1), (1, 1), (0, 0)))
    out = np.zeros((B, H, W, w.shape[1]))
    for t in range(9):
        dy, dx = divmod(t, 3)
        out += xp[:, dy:dy + H, dx:dx + W, :] @ w[t].T
    return out + b


def conv_t(d, w):
    """Adjoint of conv with respect to its input."""
    B, H, W, _ = d.shape
    out = np.zeros((B, H + 2, W + 2, w.shape[2]))
    for t in range(9):
        dy, dx = divmod(t, 3)
        out[:, dy:dy + H, dx:dx + W, :] += d @ w[t]
    return out[:, 1:-1, 1:-1, :]


def conv_w(x, d):
    """Gradient of conv with respect to its weight [9][Cout][Cin]."""
    B, H, W, _ = x.shape
    xp = np.pad(x, ((0, 0), (1, 1), (1, 1), (0, 0)))
    return np.stack([np.einsum("byxo,byxi->oi", d, xp[:, t // 3:t // 3 + H, t % 3:t % 3 + W, :])
                     for t in range(9)])


def pool(x):
    return 0.25 * (x[:, 0::2, 0::2] + x[:, 0::2, 1::2] + x[:, 1::2, 0::2] + x[:, 1::2, 1::2])


def up(x):
    return x.repeat(2, axis=1).repeat(2, axis=2)


def down_sum(d):
    return d[:, 0::2, 0::2] + d[:, 0::2, 1::2] + d[:, 1::2, 0::2] + d[:, 1::2, 1::2]


def forward(theta, x, round_bf16=True):
    """x [B,H,W,2] -> (out [B,H,W], cache)."""
    P = unpack(theta)
    r = bf16 if round_bf16 else (lambda a: np.asarray(a, np.float64))
    W = {k: ((r(w) if k in TC_LAYERS else w.astype(np.float64)), b.astype(np.float64))
         for k, (w, b) in P.items()}
    c = {"x": x.astype(np.float64)}
    relu = lambda a: np.maximum(a, 0)
    c["h0"] = r(relu(conv(c["x"], *W["cin"])))
    c["p1"] = r(pool(c["h0"]))
    c["h1"] = r(relu(conv(c["p1"], *W["e1"])))
    c["p2"] = r(pool(c["h1"]))
    c["h2"] = r(relu(conv(c["p2"], *W["e2"])))
    c["p3"] = r(pool(c["h2"]))
    c["h3"] = r(relu(conv(c["p3"], *W["e3"])))
    c["g3"] = r(relu(conv(c["h3"], *W["d3"])))
    c["u2"] = r(up(c["g3"]) + c["h2"])
    c["g2"] = r(relu(conv(c["u2"], *W["d2"])))
    c["u1"] = r(up(c["g2"]) + c["h1"])
    c["g1"] = r(relu(conv(c["u1"], *W["d1"])))
    c["u0"] = r(up(c["g1"]) + c["h0"])
    c["g0"] = r(relu(conv(c["u0"], *W["d0"])))
    out = conv(c["g0"], *W["cout"])[..., 0]
    c["W"] = W
    return out, c


def backward(c, dout, round_bf16=False):
    """Gradient of sum(out * dout) with respect to the flat parameters.
    round_bf16: round every gradient tensor the GPU stores in BF16 (the
    convolution operands of the backward pass) at the same place."""
    W = c["W"]
    r = bf16 if round_bf16 else (lambda a: a)
    g = {}
    d = dout[..., None].astype(np.float64)
    g["cout"] = (conv_w(c["g0"], d), d.sum(axis=(0, 1, 2)))
    dz = r(conv_t(d, W["cout"][0]) * (c["g0"] > 0))
    g["d0"] = (conv_w(c["u0"], dz), dz.sum(axis=(0, 1, 2)))
    du0 = r(conv_t(dz, W["d0"][0]))
    dz = r(down_sum(du0) * (c["g1"] > 0))
    g["d1"] = (conv_w(c["u1"], dz), dz.sum(axis=(0, 1, 2)))
    du1 = r(conv_t(dz, W["d1"][0]))
    dz = r(down_sum(du1) * (c["g2"] > 0))
    g["d2"] = (conv_w(c["u2"], dz), dz.sum(axis=(0, 1, 2)))
    du2 = r(conv_t(dz, W["d2"][0]))
    dz = r(down_sum(du2) * (c["g3"] > 0))
    g["d3"] = (conv_w(c["h3"], dz), dz.sum(axis=(0, 1, 2)))
    dz = r(conv_t(dz, W["d3"][0]) * (c["h3"] > 0))
    g["e3"] = (conv_w(c["p3"], dz), dz.sum(axis=(0, 1, 2)))
    dz = r((du2 + 0.25 * up(r(conv_t(dz, W["e3"][0])))) * (c["h2"] > 0))
    g["e2"] = (conv_w(c["p2"], dz), dz.sum(axis=(0, 1, 2)))
    dz = r((du1 + 0.25 * up(r(conv_t(dz, W["e2"][0])))) * (c["h1"] > 0))
    g["e1"] = (conv_w(c["p1"], dz), dz.sum(axis=(0, 1, 2)))
    dz = r((du0 + 0.25 * up(r(conv_t(dz, W["e1"][0])))) * (c["h0"] > 0))
    g["cin"] = (conv_w(c["x"], dz), dz.sum(axis=(0, 1, 2)))
    return np.concatenate([np.concatenate([g[k][0].ravel(), g[k][1].ravel()]) for k, _, _ in LAYERS])
