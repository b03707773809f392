"""Batched BM3D (bm3d_batch_*): planes of different sizes and noise levels in
one persistent launch per stage, replayed from a CUDA graph, give exactly the
per-plane results."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("autotune", [False, True])
def test_batch_equals_per_plane(bm3d_lib, autotune):
    import torch
    import isp_mw_b200
    from isp_mw_b200 import synth
    ctx = isp_mw_b200.Context(0)
    rng = np.random.default_rng(7)
    shapes = [(130, 97), (300, 256), (64, 64), (220, 180), (33, 250), (401, 123)]
    srcs, dsts, pbs, pfs, want = [], [], [], [], []
    for k, (h, w) in enumerate(shapes):
        s255 = float(rng.uniform(5, 50))
        _, noisy = synth.pair(h, w, s255, 300 + k)
        sp = [synth.sigma_param(s255)] * 3
        pb = isp_mw_b200.stage_params_default("fast", False, sp)
        pf = isp_mw_b200.stage_params_default("fast", True, sp)
        if k == 2:
            pb.sigma[0] = pf.sigma[0] = 0.0  # guard: copied through, as the reference does
        src = torch.from_numpy(noisy).cuda()
        ref = torch.empty_like(src)
        ctx.full(pb, pf, ref, src)
        srcs.append(src)
        dsts.append(torch.full_like(src, -1.0))
        pbs.append(pb)
        pfs.append(pf)
        want.append(ref)
    batch = isp_mw_b200.Batch(ctx, pbs, pfs, dsts, srcs, autotune=autotune)
    for _ in range(2):  # replays reuse the captured graph and its scratch
        for d in dsts:
            d.fill_(-1.0)
        batch.run()
        torch.cuda.synchronize()
        for k, (d, r) in enumerate(zip(dsts, want)):
            assert torch.equal(d, r), k
    assert torch.equal(dsts[2], srcs[2])
    t = batch.tuning()
    assert all(v > 0 for v in t["basic"] + t["final"])
    batch.close()
    ctx.close()
