"""CPU: the U-Net oracle's gradients against central finite differences (the
network has no reference counterpart, so the FP64 oracle is pinned this way)."""
import numpy as np

from oracle import unet_oracle as uo


def test_conv_backward_matches_finite_differences():
    rng = np.random.default_rng(0)
    x = rng.standard_normal((3, 4, 5, 6))
    w = rng.standard_normal((7, 6, 27))
    dy = rng.standard_normal((3, 4, 5, 7))
    # <dy, conv(x)> is linear in x and in w: its gradients are exact adjoints
    f = lambda xx, ww: float(np.sum(dy * uo.conv3(xx, ww)))  # noqa: E731
    gx, gw = uo.conv3_backward_data(dy, w), uo.conv3_backward_weight(x, dy)
    for _ in range(10):
        i = tuple(rng.integers(0, s) for s in x.shape)
        e = np.zeros_like(x)
        e[i] = 1e-3
        assert abs((f(x + e, w) - f(x - e, w)) / 2e-3 - gx[i]) < 1e-8
        j = tuple(rng.integers(0, s) for s in w.shape)
        e = np.zeros_like(w)
        e[j] = 1e-3
        assert abs((f(x, w + e) - f(x, w - e)) / 2e-3 - gw[j]) < 1e-8


def test_conv_zero_padding_and_tap_order():
    x = np.zeros((3, 3, 3, 1))
    x[1, 1, 2, 0] = 1.0  # voxel (x=2, y=1, z=1)
    w = np.zeros((1, 1, 27))
    w[0, 0, 9 * 1 + 3 * 1 + 2] = 1.0  # tap offset (dz, dy, dx) = (0, 0, +1)
    y = uo.conv3(x, w)
    assert y[1, 1, 1, 0] == 1.0 and y.sum() == 1.0  # y[v] = x[v + (0,0,1)]


def test_network_gradient_matches_finite_differences():
    rng = np.random.default_rng(1)
    n = uo.num_params()
    p = np.zeros(n)
    off = 0
    for _, ci, co, _ in uo.LAYERS:
        p[off:off + co * ci * 27] = rng.standard_normal(co * ci * 27) * np.sqrt(2.0 / (ci * 27))
        off += co * ci * 27
        p[off:off + co] = 0.05 * rng.standard_normal(co)
        off += co
    S = 8
    in2 = rng.standard_normal((S, S, S, 2))
    t2 = rng.standard_normal((S, S, S, 2))
    wgt = rng.uniform(0.0, 1.0, (S, S, S))
    loss, g, _ = uo.loss_and_grad(p, in2, t2, wgt, 1.0, 0.5, weights_bf16=False)
    # parameters spread over every layer (weights and biases)
    idx, off = [], 0
    for _, ci, co, _ in uo.LAYERS:
        idx.append(off + int(rng.integers(0, min(co, 2) * ci * 27)))
        off += co * ci * 27
        idx.append(off + int(rng.integers(0, min(co, 2))))
        off += co
    for i in idx:
        e = np.zeros(n)
        e[i] = 1e-6
        lp = uo.loss_and_grad(p + e, in2, t2, wgt, 1.0, 0.5, weights_bf16=False)[0]
        lm = uo.loss_and_grad(p - e, in2, t2, wgt, 1.0, 0.5, weights_bf16=False)[0]
        fd = (lp - lm) / 2e-6
        assert abs(fd - g[i]) <= 1e-5 * max(1.0, abs(g[i])), (i, fd, g[i])


def test_bf16_rounding():
    x = np.array([1.0, 1.0 + 2 ** -8, 1.0 + 3 * 2 ** -8, -2.5, 65504.0], np.float32)
    r = uo.bf16(x)
    assert r[0] == 1.0 and r[1] == 1.0 and r[2] == 1.0 + 4 * 2 ** -8 and r[3] == -2.5
