"""bm3d_stage_noalloc: the allocation-free stage entry point.

Some callers cannot allocate device memory while running -- a filter plugin
whose host application owns every device allocation, or a real-time frame loop
that cannot afford a cudaMalloc (it may synchronise the device or fail under
memory pressure). For them the library keeps the stage's scratch in a static
device array, and this entry point takes only the caller's device planes.

The test calls it through the C ABI twice in a row (the basic stage, then the
final stage fed by the first call's output, so the second call reuses the
shared scratch the first one left behind) and checks each result against the
context-based bm3d_stage on the same inputs. Both run the same kernels with the
same tiling on the same inputs, so the planes must be equal bit for bit (a
tolerance would hide a stale-accumulator bug that moves values slightly).
bm3d_noalloc_check must report the kernels' consistency counter clean. A plane
larger than the static scratch is refused with its message readable through
bm3d_last_error(NULL). A second test runs the entry point in a fresh process
before any context exists, so its own per-device set-up (scratch address,
cosine tables) is what the kernels use. The file sorts last so a failure here
comes after every other test has run.
"""
import ctypes
import subprocess
import sys

import pytest

from conftest import ROOT

pytestmark = pytest.mark.gpu


def _run_noalloc_then_context(h, w, s255, seed):
    """Two allocation-free calls (basic, then final on its output), THEN the
    context-based stages on the same inputs; returns the four planes and the
    status codes."""
    import torch
    import isp_mw_b200
    from isp_mw_b200 import synth

    lib = isp_mw_b200.load_library()
    _, noisy = synth.pair(h, w, s255, seed)
    sp = [synth.sigma_param(s255)] * 3
    basic_p = isp_mw_b200.stage_params_default("fast", False, sp)
    final_p = isp_mw_b200.stage_params_default("fast", True, sp)
    dev = torch.device("cuda", 0)
    torch.cuda.set_device(dev)
    src = torch.from_numpy(noisy).to(dev)
    stream = torch.cuda.current_stream(dev).cuda_stream

    got_basic = torch.empty_like(src)
    got_final = torch.empty_like(src)
    rc1 = lib.bm3d_stage_noalloc(ctypes.byref(basic_p), 0, got_basic.data_ptr(), src.data_ptr(),
                                 src.data_ptr(), w, h, w, 1.0, stream)
    rc2 = lib.bm3d_stage_noalloc(ctypes.byref(final_p), 1, got_final.data_ptr(), src.data_ptr(),
                                 got_basic.data_ptr(), w, h, w, 1.0, stream)
    rc_check = lib.bm3d_noalloc_check(stream)
    torch.cuda.synchronize(dev)

    ctx = isp_mw_b200.Context(0)
    want_basic = torch.empty_like(src)
    want_final = torch.empty_like(src)
    ctx.stage(basic_p, False, want_basic, src)
    ctx.stage(final_p, True, want_final, src, want_basic)
    torch.cuda.synchronize(dev)
    ctx.close()
    return (rc1, rc2, rc_check), (got_basic, got_final), (want_basic, want_final), (
        lib, basic_p, src, stream)


def test_noalloc_stage_matches_context_stage():
    import isp_mw_b200
    import torch

    rcs, got, want, (lib, basic_p, src, stream) = _run_noalloc_then_context(360, 640, 25.0, 123)
    assert rcs == (isp_mw_b200.BM3D_OK,) * 3, (rcs, lib.bm3d_last_error(None))
    for g, w_ in zip(got, want):
        assert torch.equal(g, w_), (g - w_).abs().max().item()

    # a plane beyond the static scratch is refused before any work, with a message
    big_w, big_h = 2049, 1024
    rc = lib.bm3d_stage_noalloc(ctypes.byref(basic_p), 0, got[0].data_ptr(), src.data_ptr(),
                                src.data_ptr(), big_w, big_h, big_w, 1.0, stream)
    assert rc == isp_mw_b200.BM3D_ERR_TOO_LARGE
    assert b"static scratch" in lib.bm3d_last_error(None)


_FRESH = r"""
import sys
sys.path.insert(0, sys.argv[1])
sys.path.insert(0, sys.argv[1] + "/tests")
import torch
from test_zz_no_alloc import _run_noalloc_then_context
rcs, got, want, _ = _run_noalloc_then_context(200, 333, 40.0, 77)
assert rcs == (0, 0, 0), rcs
for g, w in zip(got, want):
    assert torch.equal(g, w), (g - w).abs().max().item()
print("fresh-process noalloc ok")
"""


def test_noalloc_first_call_in_fresh_process():
    """No context is ever created before the allocation-free calls in this
    process, so they rely on their own per-device set-up alone."""
    r = subprocess.run([sys.executable, "-c", _FRESH, ROOT], capture_output=True, text=True,
                       timeout=600, cwd=ROOT)
    assert r.returncode == 0, r.stdout[-2000:] + r.stderr[-4000:]
    assert "fresh-process noalloc ok" in r.stdout
