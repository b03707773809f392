"""bm3d_stage_noalloc: the allocation-free stage entry point.

Some callers cannot allocate device memory while running -- a filter plugin
whose host application owns every device allocation, or a real-time frame loop
that cannot afford a cudaMalloc (it may synchronise the device or fail under
memory pressure). For them the library keeps the stage's scratch in a static
device array, and this entry point takes only the caller's device planes.

This test calls it through the C ABI twice in a row (the basic stage, then the
final stage fed by the first call's output, so the second call reuses the
shared scratch the first one left behind) and checks each result against the
context-based bm3d_stage on the same inputs, within the parity tolerance used
everywhere else (max-abs 1e-3). It also checks that a plane larger than the
static scratch is refused. The file sorts last so a failure here comes after
every other test has run.
"""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

MAX_ABS = 1e-3


def test_noalloc_stage_matches_context_stage():
    import torch
    import isp_mw_b200
    from isp_mw_b200 import synth

    lib = isp_mw_b200.load_library()
    h, w, s255 = 360, 640, 25.0
    _, noisy = synth.pair(h, w, s255, 123)
    sp = [synth.sigma_param(s255)] * 3
    basic_p = isp_mw_b200.stage_params_default("fast", False, sp)
    final_p = isp_mw_b200.stage_params_default("fast", True, sp)

    dev = torch.device("cuda", 0)
    torch.cuda.set_device(dev)
    src = torch.from_numpy(noisy).to(dev)
    stream = torch.cuda.current_stream(dev).cuda_stream

    # the existing entry point (context scratch)
    ctx = isp_mw_b200.Context(0)
    want_basic = torch.empty_like(src)
    want_final = torch.empty_like(src)
    ctx.stage(basic_p, False, want_basic, src)
    ctx.stage(final_p, True, want_final, src, want_basic)

    # the allocation-free entry point, two calls in a row
    got_basic = torch.empty_like(src)
    got_final = torch.empty_like(src)
    rc1 = lib.bm3d_stage_noalloc(ctypes.byref(basic_p), 0, got_basic.data_ptr(), src.data_ptr(),
                                 src.data_ptr(), w, h, w, 1.0, stream)
    rc2 = lib.bm3d_stage_noalloc(ctypes.byref(final_p), 1, got_final.data_ptr(), src.data_ptr(),
                                 got_basic.data_ptr(), w, h, w, 1.0, stream)
    torch.cuda.synchronize(dev)
    assert rc1 == isp_mw_b200.BM3D_OK and rc2 == isp_mw_b200.BM3D_OK

    for got, want in ((got_basic, want_basic), (got_final, want_final)):
        d = (got - want).abs().max().item()
        assert d <= MAX_ABS, d

    # a plane beyond the static scratch is refused before any work
    big_w, big_h = 2049, 1024
    rc = lib.bm3d_stage_noalloc(ctypes.byref(basic_p), 0, got_basic.data_ptr(), src.data_ptr(),
                                src.data_ptr(), big_w, big_h, big_w, 1.0, stream)
    assert rc == isp_mw_b200.BM3D_ERR_TOO_LARGE
    ctx.close()
