"""GPU: the U-Net's tensor-core convolutions (forward, backward-data,
backward-weight) and the whole network's loss and gradients against the
CPU FP64 oracle (oracle/unet_oracle.py, itself pinned by finite
differences).

Tolerances: FP32 outputs of one convolution differ from FP64 only by the
order of FP32 accumulation (relative L2 <= 1e-5); BF16 outputs by one
rounding (<= 2^-8 relative per element).  The network's gradients carry
BF16 rounding of every stored activation and gradient, so they are compared
per layer in relative L2 (<= 5e-2) and as one vector by cosine (>= 0.999).
"""
import numpy as np
import pytest

from oracle import unet_oracle as uo

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def net():
    from vflip_b200.learned import UNet

    with UNet(seed=3) as n:
        yield n


def rel(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    return np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-30)


def bf16_tensor(shape, rng, scale=1.0):
    a = (rng.standard_normal(shape) * scale).astype(np.float32)
    t = torch.from_numpy(a).to("cuda").to(torch.bfloat16)
    return t, t.float().cpu().numpy().astype(np.float64)


CONV_CASES = [  # (X, Y, Z), cin, cout, ctot, coff
    ((8, 16, 3), 16, 16, 16, 0),
    ((20, 23, 5), 16, 32, 48, 32),
    ((13, 40, 4), 48, 16, 48, 0),
    ((20, 23, 5), 192, 64, 192, 0),
    ((9, 17, 3), 64, 128, 64, 0),
    ((16, 16, 4), 32, 192, 96, 64),
    ((10, 7, 2), 128, 256, 128, 0),
]


@pytest.mark.parametrize("dims,cin,cout,ctot,coff", CONV_CASES)
def test_conv_forward(net, dims, cin, cout, ctot, coff):
    rng = np.random.default_rng(cin * 7 + cout)
    X, Y, Z = dims
    x, xn = bf16_tensor((Z, Y, X, ctot), rng)
    w = (rng.standard_normal((cout, cin, 27)) / np.sqrt(cin * 27)).astype(np.float32)
    b = rng.standard_normal(cout).astype(np.float32)
    wt, bt = torch.from_numpy(w).cuda(), torch.from_numpy(b).cuda()
    got = net.conv3(x, wt, cin, cout, bias=bt, in_coff=coff).cpu().numpy()
    want = uo.conv3(xn[..., coff:coff + cin], uo.bf16(w), b)
    assert rel(got, want) < 1e-5
    # BF16 output with ReLU and a mask, written into a channel view
    m, mn = bf16_tensor((Z, Y, X, cout), rng)
    out = torch.zeros((Z, Y, X, cout + 16), dtype=torch.bfloat16, device="cuda")
    net.conv3(x, wt, cin, cout, bias=bt, relu=True, mask=m, in_coff=coff, out=out, out_coff=16)
    o = out.float().cpu().numpy()
    ref = np.maximum(want, 0) * (mn > 0)
    # one BF16 rounding, plus FP32-vs-FP64 slack where the ReLU cuts near zero
    assert np.all(np.abs(o[..., 16:] - ref) <= 2.0 ** -8 * np.abs(ref) + 1e-5 * np.abs(want).max())
    assert np.all(o[..., :16] == 0)


@pytest.mark.parametrize("dims,cin,cout,ctot,coff", CONV_CASES[:5])
def test_conv_backward_data(net, dims, cin, cout, ctot, coff):
    # gradient with respect to the input of a layer cin -> cout
    rng = np.random.default_rng(cin + 3 * cout)
    X, Y, Z = dims
    dy, dyn = bf16_tensor((Z, Y, X, cout), rng)
    w = (rng.standard_normal((cout, cin, 27)) / np.sqrt(cout * 27)).astype(np.float32)
    m, mn = bf16_tensor((Z, Y, X, cin), rng)
    got = net.conv3(dy, torch.from_numpy(w).cuda(), cin, cout, backward_data=True, mask=m).cpu().numpy()
    want = uo.conv3_backward_data(dyn, uo.bf16(w)) * (mn > 0)
    assert rel(got, want) < 1e-5


@pytest.mark.parametrize("dims,cin,cout,ctot,coff", CONV_CASES[:6])
def test_conv_backward_weight(net, dims, cin, cout, ctot, coff):
    rng = np.random.default_rng(5 * cin + cout)
    X, Y, Z = dims
    x, xn = bf16_tensor((Z, Y, X, ctot), rng)
    if cout > 128:
        cout = 128
    dy, dyn = bf16_tensor((Z, Y, X, cout + 16), rng)
    got = net.conv3_wgrad(x, dy, cin=cin, cout=cout, x_coff=coff, dy_coff=16).cpu().numpy()
    want = uo.conv3_backward_weight(xn[..., coff:coff + cin], dyn[..., 16:16 + cout])
    assert rel(got, want) < 1e-5


def _sample(S, rng):
    in2 = np.zeros((S, S, S, 2), np.float32)
    in2[..., 0] = rng.standard_normal((S, S, S))
    in2[..., 1] = (rng.uniform(size=(S, S, S)) > 0.2).astype(np.float32)
    t2 = rng.standard_normal((S, S, S, 2)).astype(np.float32)
    wgt = in2[..., 1].copy()
    return in2, t2, wgt


def test_network_forward_matches_oracle(net):
    rng = np.random.default_rng(11)
    S = 16
    in2, _, _ = _sample(S, rng)
    got = net.forward(torch.from_numpy(in2).cuda()).cpu().numpy()
    want, _ = uo.forward(net.get_params().astype(np.float64), in2.astype(np.float64), round_acts=True)
    assert rel(got, want) < 2e-2
    again = net.forward(torch.from_numpy(in2).cuda()).cpu().numpy()
    assert np.array_equal(got, again)  # deterministic


def test_network_forward_replay_follows_inputs_and_weights(net):
    """vflip_unet_forward replays a captured graph when the grid and the
    buffers repeat: new input values and new weights in the same buffers
    give the eager forward's bits (the training path's forward), and the
    oracle's answer for the new weights."""
    rng = np.random.default_rng(12)
    S = 16
    a, t2, wgt = _sample(S, rng)
    b, _, _ = _sample(S, rng)
    in2 = torch.from_numpy(a).cuda()
    out2 = torch.empty((S, S, S, 2), dtype=torch.float32, device="cuda")
    p0 = net.get_params()
    try:
        net.forward(in2, out2)
        in2.copy_(torch.from_numpy(b))
        got_b = net.forward(in2, out2).clone()
        net.set_params(p0 * 0.9)
        got_b2 = net.forward(in2, out2).clone()
        want, _ = uo.forward(net.get_params().astype(np.float64), b.astype(np.float64), round_acts=True)
        assert rel(got_b2.cpu().numpy(), want) < 2e-2
        assert not torch.equal(got_b, got_b2)
        # the training path runs the same forward eagerly: the same output
        net.gradients(in2, torch.from_numpy(t2).cuda(), torch.from_numpy(wgt).cuda())
        again = net.forward(in2, out2)
        assert torch.equal(again, got_b2)
    finally:
        net.set_params(p0)


def test_network_gradients_match_oracle(net):
    rng = np.random.default_rng(12)
    S = 16
    in2, t2, wgt = _sample(S, rng)
    T = lambda a: torch.from_numpy(a).cuda()  # noqa: E731
    loss, g = net.gradients(T(in2), T(t2), T(wgt), 1.0, 0.5)
    g = g.cpu().numpy().astype(np.float64)
    p = net.get_params().astype(np.float64)
    lw, gw, _ = uo.loss_and_grad(p, in2.astype(np.float64), t2.astype(np.float64), wgt.astype(np.float64), 1.0, 0.5,
                                 round_acts=True)
    assert abs(loss - lw) <= 1e-2 * abs(lw)
    off = 0
    for name, ci, co, _ in uo.LAYERS:
        n = co * ci * 27 + co
        assert rel(g[off:off + n], gw[off:off + n]) < 5e-2, name
        off += n
    cos = float(g @ gw / (np.linalg.norm(g) * np.linalg.norm(gw)))
    assert cos > 0.999


def test_training_reduces_loss():
    from vflip_b200.learned import UNet

    rng = np.random.default_rng(13)
    S = 16
    in2 = np.zeros((S, S, S, 2), np.float32)
    in2[..., 0] = rng.standard_normal((S, S, S))
    in2[..., 1] = 1.0
    # a smooth target the network can fit: a blurred copy of the input
    k = np.ones(3) / 3
    t = in2[..., 0]
    for ax in range(3):
        t = np.apply_along_axis(lambda r: np.convolve(r, k, mode="same"), ax, t)
    t2 = np.stack([t, 0.5 * t], axis=-1).astype(np.float32)
    wgt = np.ones((S, S, S), np.float32)
    T = lambda a: torch.from_numpy(np.ascontiguousarray(a)).cuda()  # noqa: E731
    with UNet(seed=5) as n:
        l0 = n.train_step(T(in2), T(t2), T(wgt), 1e-3)
        for _ in range(80):
            last = n.train_step(T(in2), T(t2), T(wgt), 1e-3)
        assert last < 0.3 * l0, (l0, last)


def test_network_rejects_bad_grid(net):
    from vflip_b200._lib import VflipError

    with pytest.raises(VflipError):
        net.forward(torch.zeros((12, 16, 16, 2), dtype=torch.float32, device="cuda"))
