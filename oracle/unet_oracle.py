"""CPU FP64 restatement of the learned preconditioner's 3D U-Net - test
infrastructure only (the comparison for the tensor-core kernels; never called by
the product path).

The network has no counterpart in the reference (which solves with plain
MGPCG only, Smoke_Solver/AlgebraicMultigrid.h:189-301), so this oracle is the
project's own definition of it: layer table, 3x3x3 zero-padded convolution,
ReLU, 2x2x2 average pooling, nearest upsampling, concatenated skips
(upsampled channels first), weighted MSE loss on the two output channels.
Its gradients are pinned by central finite differences (tests/test_unet_oracle.py).

Layouts follow the library: activations [Z][Y][X][C] (channels last);
weights W[cout][cin][27] with tap = 9*dz + 3*dy + dx for offsets dz,dy,dx in
{-1,0,1} (index d = offset + 1); parameters flattened per layer as W then b.

bf16() rounds to the nearest BF16 (ties to even) - the storage precision of
the GPU network's weights and activations; forward(..., round_acts=True)
rounds at the same points as the GPU kernels (each layer's stored output).
"""
import numpy as np

LAYERS = [  # name, cin, cout, relu
    ("E0A", 16, 16, 1), ("E0B", 16, 16, 1), ("E1A", 16, 32, 1), ("E1B", 32, 32, 1), ("E2A", 32, 64, 1),
    ("E2B", 64, 64, 1), ("B1", 64, 128, 1), ("B2", 128, 128, 1), ("D2A", 192, 64, 1), ("D2B", 64, 64, 1),
    ("D1A", 96, 32, 1), ("D1B", 32, 32, 1), ("D0A", 48, 16, 1), ("D0B", 16, 16, 1), ("OUT", 16, 16, 0),
]
OUT_VALID = 2


def num_params():
    return sum(co * (ci * 27 + 1) for _, ci, co, _ in LAYERS)


def unflatten(p):
    """Flat parameter vector -> {name: (W[cout][cin][27], b[cout])}."""
    out, off = {}, 0
    for name, ci, co, _ in LAYERS:
        w = p[off:off + co * ci * 27].reshape(co, ci, 27)
        off += co * ci * 27
        b = p[off:off + co]
        off += co
        out[name] = (w, b)
    return out


def flatten(d):
    return np.concatenate([np.concatenate([d[n][0].ravel(), d[n][1].ravel()]) for n, _, _, _ in LAYERS])


def bf16(x):
    x = np.ascontiguousarray(x, dtype=np.float32)
    u = x.view(np.uint32).astype(np.uint64)
    r = ((u + 0x7FFF + ((u >> 16) & 1)) & 0xFFFF0000).astype(np.uint32)
    return r.view(np.float32)


def _taps():
    for t in range(27):
        yield t, t // 9 - 1, (t // 3) % 3 - 1, t % 3 - 1


def _shift(a, dz, dy, dx):
    """a[z+dz, y+dy, x+dx] with zeros outside (a: [Z][Y][X][C])."""
    Z, Y, X = a.shape[:3]
    out = np.zeros_like(a)
    zs, ys, xs = slice(max(0, -dz), Z - max(0, dz)), slice(max(0, -dy), Y - max(0, dy)), slice(max(0, -dx),
                                                                                                 X - max(0, dx))
    zd, yd, xd = slice(max(0, dz), Z - max(0, -dz)), slice(max(0, dy), Y - max(0, -dy)), slice(max(0, dx),
                                                                                               X - max(0, -dx))
    out[zs, ys, xs] = a[zd, yd, xd]
    return out


def conv3(x, w, b=None):
    """y[v][co] = sum_{tap,ci} x[v+off(tap)][ci] w[co][ci][tap] (+ b)."""
    x = np.asarray(x, np.float64)
    w = np.asarray(w, np.float64)
    y = np.zeros(x.shape[:3] + (w.shape[0],))
    for t, dz, dy, dx in _taps():
        y += _shift(x, dz, dy, dx) @ w[:, :, t].T
    if b is not None:
        y += np.asarray(b, np.float64)
    return y


def conv3_backward_data(dy, w):
    """Gradient of conv3 with respect to its input."""
    dy = np.asarray(dy, np.float64)
    w = np.asarray(w, np.float64)
    dx = np.zeros(dy.shape[:3] + (w.shape[1],))
    for t, dz, ddy, ddx in _taps():
        dx += _shift(dy, -dz, -ddy, -ddx) @ w[:, :, t]
    return dx


def conv3_backward_weight(x, dy):
    """dW[co][ci][tap] = sum_v dy[v][co] x[v+off(tap)][ci]."""
    x = np.asarray(x, np.float64)
    dy = np.asarray(dy, np.float64)
    co, ci = dy.shape[3], x.shape[3]
    dw = np.zeros((co, ci, 27))
    d2 = dy.reshape(-1, co)
    for t, dz, ddy, ddx in _taps():
        dw[:, :, t] = d2.T @ _shift(x, dz, ddy, ddx).reshape(-1, ci)
    return dw


def pool(a):
    Z, Y, X, C = a.shape
    return a.reshape(Z // 2, 2, Y // 2, 2, X // 2, 2, C).mean(axis=(1, 3, 5))


def pool_backward(g):
    return np.repeat(np.repeat(np.repeat(g, 2, 0), 2, 1), 2, 2) / 8.0


def up(a):
    return np.repeat(np.repeat(np.repeat(a, 2, 0), 2, 1), 2, 2)


def up_backward(g):
    Z, Y, X, C = g.shape
    return g.reshape(Z // 2, 2, Y // 2, 2, X // 2, 2, C).sum(axis=(1, 3, 5))


def pack_input(in2):
    """[Z][Y][X][2] -> the network's 16-channel input (channels 2..15 zero)."""
    x = np.zeros(in2.shape[:3] + (16,))
    x[..., :2] = in2
    return x


def forward(params, in2, round_acts=False, weights_bf16=True):
    """Returns (out2 [Z][Y][X][2], cache for backward)."""
    P = unflatten(np.asarray(params, np.float64))
    rd = (lambda a: bf16(a).astype(np.float64)) if round_acts else (lambda a: a)
    W = {n: ((bf16(w).astype(np.float64) if weights_bf16 else w), b) for n, (w, b) in P.items()}
    c = {}

    def layer(name, x):
        w, b = W[name]
        relu = dict((n, r) for n, _, _, r in LAYERS)[name]
        z = conv3(x, w, b)
        a = np.maximum(z, 0.0) if relu else z
        return a

    c["in0"] = rd(pack_input(in2))
    c["a_e0a"] = rd(layer("E0A", c["in0"]))
    c["e0"] = rd(layer("E0B", c["a_e0a"]))
    c["p1"] = rd(pool(c["e0"]))
    c["a_e1a"] = rd(layer("E1A", c["p1"]))
    c["e1"] = rd(layer("E1B", c["a_e1a"]))
    c["p2"] = rd(pool(c["e1"]))
    c["a_e2a"] = rd(layer("E2A", c["p2"]))
    c["e2"] = rd(layer("E2B", c["a_e2a"]))
    c["p3"] = rd(pool(c["e2"]))
    c["a_b1"] = rd(layer("B1", c["p3"]))
    c["b3"] = rd(layer("B2", c["a_b1"]))
    c["cat2"] = np.concatenate([up(c["b3"]), c["e2"]], axis=3)
    c["a_d2a"] = rd(layer("D2A", c["cat2"]))
    c["d2"] = rd(layer("D2B", c["a_d2a"]))
    c["cat1"] = np.concatenate([up(c["d2"]), c["e1"]], axis=3)
    c["a_d1a"] = rd(layer("D1A", c["cat1"]))
    c["d1"] = rd(layer("D1B", c["a_d1a"]))
    c["cat0"] = np.concatenate([up(c["d1"]), c["e0"]], axis=3)
    c["a_d0a"] = rd(layer("D0A", c["cat0"]))
    c["d0"] = rd(layer("D0B", c["a_d0a"]))
    out = layer("OUT", c["d0"])
    c["W"] = W
    return out[..., :OUT_VALID], c


def loss_and_grad(params, in2, target2, weight, cw0=1.0, cw1=1.0, round_acts=False, weights_bf16=True):
    """Weighted MSE (mean over voxels) and its gradient with respect to the
    FP32 master parameters, in FP64 (weights used as BF16 in the forward,
    straight-through for the gradient, as on the GPU)."""
    out, c = forward(params, in2, round_acts=round_acts, weights_bf16=weights_bf16)
    W = c["W"]
    nv = out.shape[0] * out.shape[1] * out.shape[2]
    d = out - target2
    cw = np.array([cw0, cw1])
    loss = float(np.sum(weight[..., None] * cw * d * d) / nv)
    g_out = np.zeros(out.shape[:3] + (16,))
    g_out[..., :2] = 2.0 * weight[..., None] * cw * d / nv
    grads = {}

    def bwd(name, x, dz, need_dx=True):
        w, _ = W[name]
        grads[name] = (conv3_backward_weight(x, dz), dz.reshape(-1, dz.shape[3]).sum(axis=0))
        return conv3_backward_data(dz, w) if need_dx else None

    relu_mask = lambda a: (a > 0).astype(np.float64)  # noqa: E731
    g = bwd("OUT", c["d0"], g_out) * relu_mask(c["d0"])
    g = bwd("D0B", c["a_d0a"], g) * relu_mask(c["a_d0a"])
    g_cat0 = bwd("D0A", c["cat0"], g) * relu_mask(c["cat0"])
    g = up_backward(g_cat0[..., :32])
    g = bwd("D1B", c["a_d1a"], g) * relu_mask(c["a_d1a"])
    g_cat1 = bwd("D1A", c["cat1"], g) * relu_mask(c["cat1"])
    g = up_backward(g_cat1[..., :64])
    g = bwd("D2B", c["a_d2a"], g) * relu_mask(c["a_d2a"])
    g_cat2 = bwd("D2A", c["cat2"], g) * relu_mask(c["cat2"])
    g = up_backward(g_cat2[..., :128])
    g = bwd("B2", c["a_b1"], g) * relu_mask(c["a_b1"])
    g_p3 = bwd("B1", c["p3"], g)
    g_e2 = g_cat2[..., 128:] + pool_backward(g_p3) * relu_mask(c["e2"])
    g = bwd("E2B", c["a_e2a"], g_e2) * relu_mask(c["a_e2a"])
    g_p2 = bwd("E2A", c["p2"], g)
    g_e1 = g_cat1[..., 64:] + pool_backward(g_p2) * relu_mask(c["e1"])
    g = bwd("E1B", c["a_e1a"], g_e1) * relu_mask(c["a_e1a"])
    g_p1 = bwd("E1A", c["p1"], g)
    g_e0 = g_cat0[..., 32:] + pool_backward(g_p1) * relu_mask(c["e0"])
    g = bwd("E0B", c["a_e0a"], g_e0) * relu_mask(c["a_e0a"])
    bwd("E0A", c["in0"], g, need_dx=False)
    return loss, flatten(grads), out
