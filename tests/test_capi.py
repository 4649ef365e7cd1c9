"""CPU: the C-ABI library loads and exports every entry point that
include/vflip.h declares; the host-only calls behave without a GPU."""
import ctypes as C
import os
import re

import pytest

from conftest import ROOT


def declared():
    src = open(os.path.join(ROOT, "include", "vflip.h")).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(vflip_[a-z0-9_]+)\s*\(", src)))


@pytest.fixture(scope="module")
def lib():
    from vflip_b200 import build
    from vflip_b200._lib import load

    build.build()
    return load()


def test_every_declared_symbol_is_exported(lib):
    names = declared()
    assert len(names) >= 20
    for n in names:
        assert hasattr(lib, n), n


def test_binding_table_matches_header():
    from vflip_b200._lib import SIGNATURES

    assert sorted(SIGNATURES) == declared()


def test_config_defaults_are_the_reference_constants(lib):
    from vflip_b200._lib import ConfigC

    cfg = ConfigC()
    lib.vflip_config_default(C.byref(cfg))
    # AlgebraicMultigrid.h:156,160,164 and GeometricLevelGen.h:46
    # 0 = automatic (the reference's 4096 / 200 in FP64, 512 / 100 in FP32 and MIXED)
    assert (cfg.pre_sweeps, cfg.post_sweeps, cfg.coarse_sweeps, cfg.coarsest_max_unknowns) == (4, 4, 0, 0)


def test_bad_arguments_fail_without_a_device(lib):
    from vflip_b200._lib import ConfigC

    assert lib.vflip_create(None, None) < 0
    assert lib.vflip_destroy(None) < 0
    cfg = ConfigC()
    lib.vflip_config_default(C.byref(cfg))
    cfg.coarsest_max_unknowns = 5000  # the coarsest level must fit one CTA
    ctx = C.c_void_p()
    assert lib.vflip_create(C.byref(ctx), C.byref(cfg)) < 0


def test_nested_and_subdomain_calls_reject_a_null_context(lib):
    """The nested-subdomain and subdomain entry points fail with an argument
    error before touching the device when the context is missing."""
    from vflip_b200._lib import SubdomainC

    sub = SubdomainC(8, 8, 8, 0.125, (C.c_float * 3)(0.0, 0.0, 0.0), None, None, None, None)
    n = C.c_int(0)
    assert lib.vflip_halo_select(None, None, 0, 0.1, C.byref(sub), None, 0, C.byref(n)) < 0
    assert lib.vflip_advect_flip_nested(None, 8, 8, 8, 0.1, None, 0, None, None, None, None, 0.01, C.byref(sub)) < 0
    assert lib.vflip_reorder_flip_nested(None, 8, 8, 8, 0.1, None, 0, None, None, None, None, 0, None, 0,
                                         C.byref(n), C.byref(sub)) < 0
    assert lib.vflip_advect_tracers_nested(None, 8, 8, 8, 0.1, None, 0, None, None, None, None, 0.01, 0.0,
                                           C.byref(sub)) < 0
    assert lib.vflip_emit_tracers_nested(None, None, 0, 0.1, 1.0, 1.0, 1.0, 0.5, 0.5, 0.5, 0.1, 0, 0, 8, 8, 8, None,
                                         C.byref(sub), None, 0, C.byref(n)) < 0
    assert lib.vflip_sub_particle_cells(None, 8, 8, 8, 0.1, 0.0, 0.0, 0.0, None, 0, None) < 0
    assert lib.vflip_sub_g2p(None, 8, 8, 8, 0.1, 0.0, 0.0, 0.0, None, 0, None, None, None) < 0


def test_no_cpu_fallback_without_library(monkeypatch, tmp_path):
    import vflip_b200._lib as L

    monkeypatch.setattr(L, "_lib", None)
    monkeypatch.setattr(L, "HERE", str(tmp_path))
    with pytest.raises(FileNotFoundError):
        L.load()
