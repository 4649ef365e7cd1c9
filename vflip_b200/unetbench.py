"""Timing of the learned preconditioner's U-Net (forward and one training
step) on S^3 network grids; also the target of the convolution kernels'
ncu profiles.

    python -m vflip_b200.unetbench [--sizes 32 64 128] [--iters 10] [--no-train]
"""
import argparse

import torch

from .learned import UNet

LEVEL = {"E0A": 0, "E0B": 0, "E1A": 1, "E1B": 1, "E2A": 2, "E2B": 2, "B1": 3, "B2": 3, "D2A": 2, "D2B": 2, "D1A": 1,
         "D1B": 1, "D0A": 0, "D0B": 0, "OUT": 0}
LAYERS = [("E0A", 16, 16), ("E0B", 16, 16), ("E1A", 16, 32), ("E1B", 32, 32), ("E2A", 32, 64), ("E2B", 64, 64),
          ("B1", 64, 128), ("B2", 128, 128), ("D2A", 192, 64), ("D2B", 64, 64), ("D1A", 96, 32), ("D1B", 32, 32),
          ("D0A", 48, 16), ("D0B", 16, 16), ("OUT", 16, 16)]


def forward_flops(S):
    """2 * 27 * cin * cout per voxel and layer (OUT counted at its 16 computed channels)."""
    return sum(2 * 27 * ci * co * (S >> LEVEL[n]) ** 3 for n, ci, co in LAYERS)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--sizes", type=int, nargs="+", default=[32, 64, 128])
    ap.add_argument("--iters", type=int, default=10)
    ap.add_argument("--no-train", action="store_true")
    a = ap.parse_args()
    net = UNet(seed=0)
    ev = lambda: (torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))  # noqa: E731
    for S in a.sizes:
        g = torch.Generator(device="cuda").manual_seed(S)
        in2 = torch.randn((S, S, S, 2), device="cuda", generator=g)
        for _ in range(3):
            net.forward(in2)
        torch.cuda.synchronize()
        e0, e1 = ev()
        e0.record()
        for _ in range(a.iters):
            net.forward(in2)
        e1.record()
        torch.cuda.synchronize()
        fwd = e0.elapsed_time(e1) / a.iters
        line = f"S={S}: forward {fwd:.3f} ms, {forward_flops(S) / fwd / 1e9:.1f} TFLOP/s"
        if not a.no_train:
            t2 = torch.randn((S, S, S, 2), device="cuda", generator=g)
            w = torch.ones((S, S, S), device="cuda")
            for _ in range(2):
                net.train_step(in2, t2, w, 1e-5, want_loss=False)
            torch.cuda.synchronize()
            e0.record()
            for _ in range(a.iters):
                net.train_step(in2, t2, w, 1e-5, want_loss=False)
            e1.record()
            torch.cuda.synchronize()
            line += f"; train step {e0.elapsed_time(e1) / a.iters:.3f} ms"
        print(line, flush=True)


if __name__ == "__main__":
    main()
