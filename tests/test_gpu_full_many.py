"""bm3d_full_many: host planes with copies overlapped with the filtering give
exactly the per-plane bm3d_full results, synchronously and in consecutive
asynchronous calls."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _planes(n, seed):
    from isp_mw_b200 import synth
    rng = np.random.default_rng(seed)
    out = []
    for i in range(n):
        h, w = int(rng.integers(24, 200)), int(rng.integers(24, 260))
        s = float(rng.uniform(5, 50))
        out.append((synth.pair(h, w, s, seed * 100 + i)[1], s))
    return out


def _params(s255):
    import isp_mw_b200
    from isp_mw_b200 import synth
    sp = [synth.sigma_param(s255)] * 3
    return (isp_mw_b200.stage_params_default("fast", False, sp),
            isp_mw_b200.stage_params_default("fast", True, sp))


def test_full_many_matches_full(bm3d_lib):
    import torch
    import isp_mw_b200
    ctx = isp_mw_b200.Context(0)
    planes = _planes(5, 1)
    pb, pf = zip(*[_params(s) for _, s in planes])
    want = []
    for (x, _), b, f in zip(planes, pb, pf):
        y = np.empty_like(x)
        ctx.full(b, f, y, x)
        want.append(y)
    # pageable numpy planes, synchronous
    got = [np.full_like(x, -1.0) for x, _ in planes]
    ctx.full_many(pb, pf, got, [x for x, _ in planes])
    for g, w in zip(got, want):
        assert np.array_equal(g, w)
    # page-locked tensors with a row pitch wider than the plane, two async calls
    src = []
    for x, _ in planes:
        t = torch.zeros((x.shape[0], x.shape[1] + 5), dtype=torch.float32).pin_memory()
        t[:, :x.shape[1]] = torch.from_numpy(x)
        src.append(t[:, :x.shape[1]])
    outs = [[torch.full((x.shape[0], x.shape[1] + 5), -1.0).pin_memory()[:, :x.shape[1]]
             for x, _ in planes] for _ in range(2)]
    stream = torch.cuda.current_stream().cuda_stream
    ctx.full_many(pb, pf, outs[0], src, asynchronous=True, stream=stream)
    ctx.full_many(pb[::-1], pf[::-1], outs[1][::-1], src[::-1], asynchronous=True, stream=stream)
    torch.cuda.synchronize()
    for k in range(2):
        for g, w in zip(outs[k], want):
            assert np.array_equal(g.numpy(), w)
    ctx.close()


def test_full_many_empty_and_invalid(bm3d_lib):
    import isp_mw_b200
    ctx = isp_mw_b200.Context(0)
    assert ctx.full_many([], [], [], []) == isp_mw_b200.BM3D_OK
    b, f = _params(20.0)
    x = np.zeros((8, 8), np.float32)
    with pytest.raises(ValueError):
        ctx.full_many([b], [f], [np.zeros((8, 9), np.float32)], [x])
    ctx.close()
