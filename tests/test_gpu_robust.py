"""Inputs outside the usual range, against the oracle, and device-memory
exhaustion.

The FP32 stages aggregate in 64-bit fixed point whose scale comes from the
plane's largest finite |src|. Two properties keep that faithful to the
reference's float sums (source/BM3D.cpp:89-135):

* Resolution: pixels outside block (0, 0) use a scale set by the terms that
  can really reach them (reference positions within BlockSize + 2 BMrange,
  GroupSize terms each), so a single huge outlier leaves the rest of the plane
  at ~2^-20 of that outlier's magnitude or finer. Far from the outliers the
  strict bar (max-abs 1e-3) holds; near them the bar is float-relative to the
  largest |src| that can enter the pixel's groups.
* NaN / Inf: the reference's float sums turn non-finite wherever a NaN or an
  Inf term reaches them. The kernels mark such pixels and write NaN there, so
  the non-finite output pixels must be exactly the reference's.

The allocation-failure test injects BM3D_ERR_NOMEM on the host
(bm3d_inject_alloc_failures) and checks that the call fails cleanly and the
context keeps working.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

MAX_ABS = 1e-3


@pytest.fixture(scope="module")
def ctx(bm3d_lib):
    import isp_mw_b200
    c = isp_mw_b200.Context(0)
    yield c
    c.close()


def _params(s255):
    import isp_mw_b200
    from isp_mw_b200 import synth
    sp = [synth.sigma_param(s255)] * 3
    return (isp_mw_b200.stage_params_default("fast", False, sp),
            isp_mw_b200.stage_params_default("fast", True, sp))


def _reach(plane_abs, radius):
    """max over the (2 radius + 1)^2 neighbourhood of each pixel."""
    from numpy.lib.stride_tricks import sliding_window_view
    pad = np.pad(plane_abs, radius, mode="constant")
    return sliding_window_view(pad, (2 * radius + 1, 2 * radius + 1)).max(axis=(2, 3))


def _oracle(oracle_mod):
    kind = "reference" if oracle_mod.reference_available() else "port"
    return oracle_mod.backend(kind, np.float32)


@pytest.mark.parametrize("shape", [(512, 512), (1080, 1920)])
def test_outlier_pixels(ctx, oracle_mod, shape):
    from isp_mw_b200 import synth
    _, noisy = synth.pair(shape[0], shape[1], 25.0, 31)
    noisy = noisy.copy()
    noisy[100, 200] = 1.0e4
    noisy[300, 400] = 1.0e8
    b, f = _params(25.0)
    orc = _oracle(oracle_mod)
    # the pixels whose groups can hold an outlier's block: within 2 BMrange + 2 BS
    radius = 2 * b.bm_range + 2 * b.block_size
    near_max = _reach(np.where(np.abs(noisy) > 10.0, np.abs(noisy), 0.0), radius)
    far = near_max == 0
    tol = MAX_ABS + 2.0 ** -20 * near_max

    rb = orc.stage(False, b.as_dict(), noisy)
    gb = np.empty_like(noisy)
    ctx.stage(b, False, gb, noisy)
    d = np.abs(gb.astype(np.float64) - rb)
    assert d[far].max() <= MAX_ABS, float(d[far].max())
    assert np.all(d <= tol), float((d - tol).max())

    rf = orc.stage(True, f.as_dict(), noisy, rb)
    gf = np.empty_like(noisy)
    ctx.stage(f, True, gf, noisy, rb)
    d = np.abs(gf.astype(np.float64) - rf)
    assert d[far].max() <= MAX_ABS, float(d[far].max())
    assert np.all(d <= tol), float((d - tol).max())


def test_nan_and_inf_pixels(ctx, oracle_mod):
    import isp_mw_b200
    from isp_mw_b200 import synth
    _, noisy = synth.pair(256, 320, 25.0, 32)
    noisy = noisy.copy()
    noisy[50, 60] = np.nan
    noisy[120, 300] = np.inf
    noisy[200, 30] = -np.inf
    b, f = _params(25.0)
    orc = _oracle(oracle_mod)

    rb = orc.stage(False, b.as_dict(), noisy)
    gb = np.empty_like(noisy)
    ctx.stage(b, False, gb, noisy)
    bad = ~np.isfinite(rb)
    assert bad.any()
    assert np.array_equal(~np.isfinite(gb), bad)
    assert np.isnan(gb[bad]).all()
    assert np.abs(gb[~bad].astype(np.float64) - rb[~bad]).max() <= MAX_ABS

    # final stage on identical inputs (the reference's basic estimate, NaN included)
    rf = orc.stage(True, f.as_dict(), noisy, rb)
    gf = np.empty_like(noisy)
    ctx.stage(f, True, gf, noisy, rb)
    bad = ~np.isfinite(rf)
    assert np.array_equal(~np.isfinite(gf), bad)
    assert np.abs(gf[~bad].astype(np.float64) - rf[~bad]).max() <= MAX_ABS

    # the combined entry: the non-finite regions are decided by the inputs alone
    full = np.empty_like(noisy)
    ctx.full(b, f, full, noisy)
    assert np.array_equal(~np.isfinite(full), bad)

    # a batch holding the same plane gives the same plane, bit for bit
    import torch
    src = torch.from_numpy(noisy).cuda()
    dst = torch.empty_like(src)
    batch = isp_mw_b200.Batch(ctx, [b], [f], [dst], [src])
    batch.run()
    torch.cuda.synchronize()
    got = dst.cpu().numpy()
    assert np.array_equal(np.isnan(got), np.isnan(full))
    assert np.array_equal(got[np.isfinite(full)], full[np.isfinite(full)])
    batch.check()
    batch.close()


def test_nonfinite_pixel_stays_in_its_plane(ctx):
    """A NaN in one plane of a three-plane image touches that plane only."""
    from isp_mw_b200 import synth
    planes = [synth.pair(96, 128, 20.0, 40 + c)[1].copy() for c in range(3)]
    b, f = _params(20.0)
    planes[1][40, 40] = np.nan
    out = [np.empty_like(p) for p in planes]
    ctx.full3(b, f, out, planes)
    assert np.isfinite(out[0]).all() and np.isfinite(out[2]).all()
    assert not np.isfinite(out[1]).all()


def test_allocation_failure_is_reported_and_recoverable(bm3d_lib):
    import isp_mw_b200
    from isp_mw_b200 import synth
    lib = bm3d_lib
    _, noisy = synth.pair(64, 80, 25.0, 5)
    b, f = _params(25.0)
    c = isp_mw_b200.Context(0)
    out = np.empty_like(noisy)
    try:
        assert lib.bm3d_inject_alloc_failures(1) == isp_mw_b200.BM3D_OK
        with pytest.raises(isp_mw_b200.BM3DError) as e:
            c.full(b, f, out, noisy)
        assert e.value.code == isp_mw_b200.BM3D_ERR_NOMEM
        assert "injected" in str(e.value)
        # the context recovers: the next call allocates and filters
        c.full(b, f, out, noisy)
        want = np.empty_like(noisy)
        isp_mw_b200.Context(0).full(b, f, want, noisy)
        assert np.array_equal(out, want)
        # a batch whose buffers cannot be allocated fails at creation
        import torch
        src = torch.from_numpy(noisy).cuda()
        dst = torch.empty_like(src)
        lib.bm3d_inject_alloc_failures(1)
        with pytest.raises(isp_mw_b200.BM3DError) as e:
            isp_mw_b200.Batch(c, [b], [f], [dst], [src])
        assert e.value.code == isp_mw_b200.BM3D_ERR_NOMEM
    finally:
        lib.bm3d_inject_alloc_failures(0)
        c.close()
