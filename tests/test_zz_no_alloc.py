"""GPU: vflip_rbgs_noalloc, the smoother entry point for callers that cannot
allocate device memory (stream-captured CUDA graphs, allocation-free
real-time loops, applications that own every device byte), called through
the C ABI.  Its result must equal vflip_rbgs's (the allocating entry point)
bit for bit - the FP64 smoother tolerance used throughout these tests - on
two calls in a row, which share the library's fixed scratch array.  This
file is collected last so that a run stopping at the first failure has run
every other test; it also passes alone in a fresh process."""
import ctypes as C

import numpy as np
import pytest

from vflip_b200 import scenes

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

MAX_CELLS = 64 * 64 * 64  # VFLIP_NOALLOC_MAX_CELLS


def _ptr(t):
    return C.c_void_p(t.data_ptr())


def _problem(dims, seed):
    ni, nj, nk = dims
    pr = scenes.projection_problem(ni, nj, nk, seed=seed, inflow=True, solid_velocity=True)
    rng = np.random.default_rng(seed)
    h = np.float32(pr["h"])
    phi = pr["phi"]
    # operator of the plume projection (face weights from the solid level set)
    import oracle

    uw, vw, ww = oracle.oracle().face_weights(ni, nj, nk, h, phi)
    st = scenes.poisson_stencil(ni, nj, nk, h, uw, vw, ww)
    four = np.stack([st[0], st[2], st[4], st[6]])
    b = rng.standard_normal((nk, nj, ni))
    x0 = rng.standard_normal((nk, nj, ni))
    return four, b, x0


def test_noalloc_smoother_matches_allocating_entry_point():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from vflip_b200 import build
    from vflip_b200._lib import load
    from vflip_b200.solver import Solver

    build.build()
    lib = load()
    dev = "cuda:0"
    stream = torch.cuda.current_stream()
    with Solver(precision=0) as s:
        for call, (dims, seed, iters) in enumerate((((40, 36, 30), 1, 3), ((33, 47, 21), 2, 4))):
            four, b, x0 = (torch.from_numpy(np.ascontiguousarray(a)).to(dev) for a in _problem(dims, seed))
            ni, nj, nk = dims
            want = s.rbgs(four, b, x0.clone(), iters)
            got = x0.clone()
            torch.cuda.synchronize()
            free0 = torch.cuda.mem_get_info()[0]
            rc = lib.vflip_rbgs_noalloc(C.c_void_p(stream.cuda_stream), ni, nj, nk, _ptr(four[0]), _ptr(four[1]),
                                        _ptr(four[2]), _ptr(four[3]), _ptr(b), _ptr(got), iters)
            assert rc == 0, f"call {call}: status {rc}"
            torch.cuda.synchronize()
            assert torch.equal(got, want), f"call {call} differs from vflip_rbgs"
            if call > 0:  # (the first call may load the library's kernels, which the driver places on the device)
                assert torch.cuda.mem_get_info()[0] == free0, "the call changed the device's free memory"


def test_noalloc_rejects_grids_beyond_its_scratch():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from vflip_b200._lib import load

    lib = load()
    t = torch.zeros(1, dtype=torch.float64, device="cuda:0")
    p = _ptr(t)
    # 65 x 64 x 64 cells exceed the 64^3 scratch: rejected before any launch
    rc = lib.vflip_rbgs_noalloc(None, 65, 64, 64, p, p, p, p, p, p, 1)
    assert rc == -6
    assert MAX_CELLS == 262144
