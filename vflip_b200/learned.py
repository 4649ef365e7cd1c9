"""The learned preconditioner's 3D U-Net over the C ABI (vflip_unet_*).

``UNet`` owns one network (FP32 master parameters, Adam state, BF16 packed
weights, activation buffers) on a device and runs on torch's current stream.
Inputs and outputs are torch CUDA tensors, channels last:
``in2``/``out2``/``target2`` are [Z, Y, X, 2] float32 and ``weight`` is
[Z, Y, X] float32.  The network has no reference counterpart; its CPU FP64
definition is oracle/unet_oracle.py (test infrastructure).
"""
import ctypes as C

import numpy as np
import torch

from ._lib import VflipError, load
from .solver import _p


class UNet:
    def __init__(self, device=None, seed=0):
        self.lib = load()
        self.device = torch.device("cuda", torch.cuda.current_device() if device is None else device)
        stream = torch.cuda.current_stream(self.device).cuda_stream
        h = C.c_void_p()
        rc = self.lib.vflip_unet_create(C.byref(h), self.device.index, C.c_void_p(stream or None), seed)
        if rc < 0:
            msg = self.lib.vflip_unet_last_error(h).decode() if h.value else "create failed"
            if h.value:
                self.lib.vflip_unet_destroy(h)
            raise VflipError(rc, msg)
        self.h = h
        self.nparams = self.lib.vflip_unet_num_params()

    def close(self):
        if getattr(self, "h", None) is not None and self.h.value:
            self.lib.vflip_unet_destroy(self.h)
            self.h = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _check(self, rc):
        if rc < 0:
            raise VflipError(rc, self.lib.vflip_unet_last_error(self.h).decode())
        return rc

    @property
    def launch_count(self):
        return self.lib.vflip_unet_launch_count(self.h)

    # parameters
    def get_params(self):
        p = np.empty(self.nparams, np.float32)
        self._check(self.lib.vflip_unet_get_params(self.h, p.ctypes.data))
        return p

    def set_output_scale(self, s0, s1):
        self._check(self.lib.vflip_unet_set_output_scale(self.h, float(s0), float(s1)))

    def set_params(self, p):
        p = np.ascontiguousarray(p, np.float32)
        assert p.size == self.nparams
        self._check(self.lib.vflip_unet_set_params(self.h, p.ctypes.data))

    # network
    def forward(self, in2, out2=None):
        Z, Y, X = in2.shape[:3]
        if out2 is None:
            out2 = torch.empty((Z, Y, X, 2), dtype=torch.float32, device=in2.device)
        self._check(self.lib.vflip_unet_forward(self.h, X, Y, Z, _p(in2), _p(out2)))
        return out2

    def gradients(self, in2, target2, weight, cw0=1.0, cw1=1.0):
        Z, Y, X = in2.shape[:3]
        g = torch.empty(self.nparams, dtype=torch.float32, device=in2.device)
        loss = C.c_double()
        self._check(self.lib.vflip_unet_gradients(self.h, X, Y, Z, _p(in2), _p(target2), _p(weight), cw0, cw1,
                                                  _p(g), C.byref(loss)))
        return loss.value, g

    def train_step(self, in2, target2, weight, lr, cw0=1.0, cw1=1.0, want_loss=True):
        Z, Y, X = in2.shape[:3]
        loss = C.c_double()
        self._check(self.lib.vflip_unet_train_step(self.h, X, Y, Z, _p(in2), _p(target2), _p(weight), cw0, cw1,
                                                   float(lr), C.byref(loss) if want_loss else None))
        return loss.value if want_loss else None

    # single operations (BF16 channels-last tensors [Z, Y, X, C])
    def conv3(self, x, w, layer_cin, layer_cout, backward_data=False, bias=None, relu=False, mask=None,
              in_coff=0, mask_coff=0, out=None, out_coff=0, outf=None, outf_valid=None):
        Z, Y, X, ctot = x.shape
        cout = layer_cin if backward_data else layer_cout
        if out is None and outf is None:
            outf = torch.empty((Z, Y, X, cout), dtype=torch.float32, device=x.device)
        self._check(self.lib.vflip_unet_conv3(
            self.h, X, Y, Z, _p(x), ctot, in_coff, _p(w), layer_cin, layer_cout, int(backward_data), _p(bias),
            int(relu), _p(mask), mask.shape[3] if mask is not None else 0, mask_coff, _p(out),
            out.shape[3] if out is not None else 0, out_coff, _p(outf), outf.shape[3] if outf is not None else 0,
            (outf.shape[3] if outf_valid is None else outf_valid) if outf is not None else 0))
        return outf if outf is not None else out

    def conv3_wgrad(self, x, dy, cin=None, cout=None, x_coff=0, dy_coff=0):
        Z, Y, X = x.shape[:3]
        cin = x.shape[3] - x_coff if cin is None else cin
        cout = dy.shape[3] - dy_coff if cout is None else cout
        dw = torch.empty((cout, cin, 27), dtype=torch.float32, device=x.device)
        self._check(self.lib.vflip_unet_conv3_wgrad(self.h, X, Y, Z, _p(x), x.shape[3], x_coff, cin, _p(dy),
                                                    dy.shape[3], dy_coff, cout, _p(dw)))
        return dw


CAPTURE, SOLVE, NO_VB, PREV, NO_NET, RESID = 1, 2, 4, 8, 16, 32


def SWEEPS(k):
    return int(k) << 8


class LearnedPreconditioner:
    """The learned warm start + coarse correction for a plume's projection.

    Phase 1 (``capturing``): projections run plain MGPCG and record one
    (features, targets, weight) triple each on the network grid of multigrid
    level ``level``.  ``train()`` fits the U-Net to the recorded triples with
    Adam on the GPU.  Phase 2: projections use the network inside flexible
    PCG (``vflip_project_learned``), which converges to the same tolerance and
    falls back to plain MGPCG when the residual stalls.
    """

    def __init__(self, solver, level=1, seed=0, net=None, use_vb=True, sweeps=2, use_prev=False, use_net=True,
                 residual=False):
        self.s = solver
        self.level = level
        self.net = net if net is not None else UNet(device=solver.device.index, seed=seed)
        self.samples = []
        self.capturing = True
        self.use_vb = use_vb
        self.sweeps = sweeps
        self.use_prev = use_prev
        self.use_net = use_net
        # residual: the network corrects the previous pressure from its
        # residual (VFLIP_LEARNED_RESID) instead of predicting the pressure
        self.residual = residual
        self.sigma = None
        self.last = None

    def _grid(self, sim):
        n = sim.p.n
        return self.s.learned_grid(n, n, n, self.level)

    def project(self, sim):
        """Projection of sim's current state; returns (converged, SolveStats)."""
        if self.capturing:
            X, Y, Z = self._grid(sim)
            dev = self.s.device
            sample = (torch.empty((Z, Y, X, 2), dtype=torch.float32, device=dev),
                      torch.empty((Z, Y, X, 2), dtype=torch.float32, device=dev),
                      torch.empty((Z, Y, X), dtype=torch.float32, device=dev))
            conv, _, st, ls = sim.project_learned(None, CAPTURE | (RESID if self.residual else 0), self.level,
                                                  sample=sample)
            self.samples.append(sample)
        else:
            mode = self.mode()
            conv, _, st, ls = sim.project_learned(self.net, mode, self.level)
        self.last = ls
        return conv, st

    def mode(self):
        if self.residual:
            return SOLVE | RESID | (0 if self.use_net else NO_NET) | SWEEPS(self.sweeps)
        return (SOLVE | (0 if self.use_vb else NO_VB) | (PREV if self.use_prev else 0) |
                (0 if self.use_net else NO_NET) | SWEEPS(self.sweeps))

    def train(self, epochs=8, lr=1e-3, seed=0, log=None):
        """Adam over the recorded triples (one sample per step, shuffled per
        epoch, cosine-decayed learning rate).  Each target channel is divided
        by its weighted RMS over the set so the network learns O(1) outputs
        (the solve's Ritz step is invariant to the outputs' scale).  Returns
        the mean loss of each epoch."""
        if not self.samples:
            raise RuntimeError("no captured samples to train on")
        m = torch.zeros(2, dtype=torch.float64, device=self.s.device)
        wsum = 0.0
        for _, t, w in self.samples:
            m += (w[..., None].double() * t.double() ** 2).sum(dim=(0, 1, 2))
            wsum += float(w.sum())
        self.sigma = torch.sqrt(m / max(wsum, 1e-30)).clamp_min(1e-30).float()
        self.net.set_output_scale(float(self.sigma[0]), float(self.sigma[1]))
        targets = [(t / self.sigma).contiguous() for _, t, _ in self.samples]
        rng = np.random.default_rng(seed)
        total = epochs * len(self.samples)
        losses, step = [], 0
        for ep in range(epochs):
            acc = 0.0
            for i in rng.permutation(len(self.samples)):
                in2, _, w = self.samples[i]
                lr_t = lr * 0.5 * (1.0 + np.cos(np.pi * step / total))
                acc += self.net.train_step(in2, targets[i], w, lr_t, 1.0, 1.0)
                step += 1
            losses.append(acc / len(self.samples))
            if log:
                log(ep, losses[-1])
        self.capturing = False
        return losses

    def prediction_error(self, sample):
        """Weighted relative L2 error of the network's two outputs on one
        captured triple (targets normalised as in training)."""
        in2, t, w = sample
        out = self.net.forward(in2)
        tn = t / self.sigma
        num = (w[..., None] * (out - tn) ** 2).sum(dim=(0, 1, 2))
        den = (w[..., None] * tn ** 2).sum(dim=(0, 1, 2))
        return tuple(float(x) for x in torch.sqrt(num / den))
