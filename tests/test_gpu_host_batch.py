"""bm3d_host_batch: a batch fed from host planes through two device slots
gives exactly the per-plane bm3d_full results (per-image bm3d_full3 for
three-plane images), run after run, synchronously and with overlapped
asynchronous runs."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_host_batch_matches_full(bm3d_lib):
    import torch
    import isp_mw_b200
    from isp_mw_b200 import synth
    ctx = isp_mw_b200.Context(0)
    shapes = [(90, 130), (64, 64), (150, 101)]
    sig = [12.0, 30.0, 45.0]
    pb, pf = [], []
    for s in sig:
        sp = [synth.sigma_param(s)] * 3
        pb.append(isp_mw_b200.stage_params_default("fast", False, sp))
        pf.append(isp_mw_b200.stage_params_default("fast", True, sp))
    hb = isp_mw_b200.HostBatch(ctx, pb, pf, shapes, autotune=True)
    runs = []
    for r in range(4):  # distinct inputs per run
        planes = [synth.pair(h, w, s, 900 + 10 * r + k)[1]
                  for k, ((h, w), s) in enumerate(zip(shapes, sig))]
        want = []
        for x, b, f in zip(planes, pb, pf):
            y = np.empty_like(x)
            ctx.full(b, f, y, x)
            want.append(y)
        runs.append((planes, want))
    # synchronous, pageable numpy planes
    for planes, want in runs[:2]:
        out = [np.full_like(x, -1.0) for x in planes]
        hb.run(out, planes)
        for o, w_ in zip(out, want):
            assert np.array_equal(o, w_)
    # asynchronous, page-locked tensors with a wider row pitch, four runs in flight
    stream = torch.cuda.current_stream().cuda_stream
    ins, outs = [], []
    for planes, _ in runs:
        ins.append([_pinned(x, 3) for x in planes])
        outs.append([_pinned(np.full_like(x, -1.0), 3) for x in planes])
    for r in range(4):
        hb.run(outs[r], ins[r], asynchronous=True if r < 2 else "overlap", stream=stream)
    hb.join(stream)
    torch.cuda.synchronize()
    for r in range(4):
        for o, w_ in zip(outs[r], runs[r][1]):
            assert np.array_equal(o.numpy(), w_)
    hb.close()
    ctx.close()


def test_host_batch3_matches_full3(bm3d_lib):
    import torch
    import isp_mw_b200
    from isp_mw_b200 import synth
    ctx = isp_mw_b200.Context(0)
    shapes = [(72, 120), (96, 88)]
    sig = [(20.0, 10.0, 12.0), (35.0, 15.0, 15.0)]
    pb, pf = [], []
    for s in sig:
        sp = [synth.sigma_param(x, c) for c, x in enumerate(s)]
        pb.append(isp_mw_b200.stage_params_default("fast", False, sp))
        pf.append(isp_mw_b200.stage_params_default("fast", True, sp))
    hb = isp_mw_b200.HostBatch(ctx, pb, pf, shapes, autotune=False, planes=3)
    runs = []
    for r in range(3):
        imgs = [[synth.pair(h, w, s[c], 700 + 31 * r + 3 * k + c)[1] for c in range(3)]
                for k, ((h, w), s) in enumerate(zip(shapes, sig))]
        want = []
        for img, b, f in zip(imgs, pb, pf):
            y = [np.empty_like(p) for p in img]
            ctx.full3(b, f, y, img)
            want.append(y)
        runs.append((imgs, want))
    imgs, want = runs[0]
    out = [[np.full_like(p, -1.0) for p in img] for img in imgs]
    hb.run(out, imgs)
    for o3, w3 in zip(out, want):
        for o, w_ in zip(o3, w3):
            assert np.array_equal(o, w_)
    stream = torch.cuda.current_stream().cuda_stream
    ins = [[[_pinned(p, 5) for p in img] for img in imgs] for imgs, _ in runs]
    outs = [[[_pinned(np.full_like(p, -1.0), 5) for p in img] for img in imgs] for imgs, _ in runs]
    for r in range(3):
        hb.run(outs[r], ins[r], asynchronous="overlap", stream=stream)
    hb.join(stream)
    torch.cuda.synchronize()
    for r in range(3):
        for o3, w3 in zip(outs[r], runs[r][1]):
            for o, w_ in zip(o3, w3):
                assert np.array_equal(o.numpy(), w_)
    with pytest.raises(ValueError):
        hb.run(out[:1], imgs[:1])
    hb.close()
    ctx.close()


def _pinned(x, pad):
    import torch
    t = torch.zeros((x.shape[0], x.shape[1] + pad), dtype=torch.float32).pin_memory()
    t[:, :x.shape[1]] = torch.from_numpy(x)
    return t[:, :x.shape[1]]
