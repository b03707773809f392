"""Host-side checks of the product library that need no GPU: it loads, it
exports every entry point include/bm3d_b200.h declares, its parameter
defaults equal the reference's, and it fails cleanly without a device."""
import ctypes
import os
import re

import numpy as np
import pytest

from conftest import ROOT, gpu_available

HEADER = os.path.join(ROOT, "include", "bm3d_b200.h")


def declared_symbols():
    text = open(HEADER).read()
    return sorted(set(re.findall(r"\b(bm3d_[a-z0-9_]+)\s*\(", text)))


def test_exports_every_declared_symbol(bm3d_lib):
    names = declared_symbols()
    assert len(names) >= 14
    for n in names:
        assert hasattr(bm3d_lib, n), n


def test_python_binding_lists_exports(bm3d_lib):
    import isp_mw_b200
    assert sorted(isp_mw_b200.EXPORTS) == declared_symbols()


@pytest.mark.parametrize("profile", ["fast", "lc", "np", "high", "vn"])
@pytest.mark.parametrize("wiener", [False, True])
def test_profile_defaults_match_reference(bm3d_lib, oracle_mod, profile, wiener):
    import isp_mw_b200
    sig = (17.0, 9.0, 4.0)
    got = isp_mw_b200.stage_params_default(profile, wiener, sig).as_dict()
    if not oracle_mod.reference_available():
        pytest.skip("reference build absent")
    want = oracle_mod.reference_stage_default(profile, wiener, sig)
    if wiener:  # the reference never initialises the final stage's lambda
        got.pop("lambda")
        want.pop("lambda")
    assert got == want


def test_unknown_profile_rejected(bm3d_lib):
    import isp_mw_b200
    with pytest.raises(ValueError):
        isp_mw_b200.stage_params_default("nope")


def test_ref_block_count_matches_scan(bm3d_lib):
    import isp_mw_b200
    p = isp_mw_b200.stage_params_default("fast", False)
    assert bm3d_lib.bm3d_ref_block_count(ctypes.byref(p), 1920, 1080) == 32400
    q = isp_mw_b200.stage_params_default("fast", True)
    assert bm3d_lib.bm3d_ref_block_count(ctypes.byref(q), 1920, 1080) == 42625
    assert bm3d_lib.bm3d_ref_block_count(ctypes.byref(p), 7, 100) == -1


def test_null_arguments_rejected(bm3d_lib):
    import isp_mw_b200
    p = isp_mw_b200.stage_params_default("fast", False)
    rc = bm3d_lib.bm3d_stage(None, ctypes.byref(p), 0, None, None, None, 64, 64, 64, 1.0, 0, None)
    assert rc == isp_mw_b200.BM3D_ERR_INVALID
    assert bm3d_lib.bm3d_ctx_create(None, 0) == isp_mw_b200.BM3D_ERR_INVALID


@pytest.mark.skipif(gpu_available(), reason="checks the no-device path")
def test_no_device_fails_cleanly(bm3d_lib):
    import isp_mw_b200
    with pytest.raises(isp_mw_b200.BM3DError) as e:
        isp_mw_b200.Context(0)
    assert e.value.code == isp_mw_b200.BM3D_ERR_CUDA
