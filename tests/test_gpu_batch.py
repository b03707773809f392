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
    batch.check()  # bm3d_batch_check: the kernels' consistency counter stayed 0
    t = batch.tuning()
    assert all(v > 0 for v in t["basic"] + t["final"])
    batch.close()
    ctx.close()


@pytest.mark.parametrize("autotune", [False, True])
def test_batch3_equals_per_image(bm3d_lib, autotune):
    """Three-plane images (groups matched on Y, reused by U and V) in one
    batch equal per-image bm3d_full3, including an image whose chroma sigma
    is 0 (that plane passes through) and one whose stages are guarded."""
    import torch
    import isp_mw_b200
    from isp_mw_b200 import synth
    ctx = isp_mw_b200.Context(0)
    shapes = [(120, 160), (97, 211), (64, 72), (180, 140)]
    srcs, dsts, pbs, pfs, want = [], [], [], [], []
    for k, (h, w) in enumerate(shapes):
        planes = [torch.from_numpy(synth.pair(h, w, s, 500 + 3 * k + c)[1]).cuda()
                  for c, s in enumerate((15.0, 10.0, 10.0))]
        sp = [synth.sigma_param(15.0, 0), synth.sigma_param(10.0, 1), synth.sigma_param(10.0, 2)]
        pb = isp_mw_b200.stage_params_default("fast", False, sp)
        pf = isp_mw_b200.stage_params_default("fast", True, sp)
        if k == 1:
            pb.sigma[2] = pf.sigma[2] = 0.0  # V passes through
        if k == 2:
            for c in range(3):  # guard: every sigma 0, all planes copied
                pb.sigma[c] = pf.sigma[c] = 0.0
        ref = [torch.empty_like(p) for p in planes]
        ctx.full3(pb, pf, ref, planes)
        srcs.append(planes)
        dsts.append([torch.full_like(p, -1.0) for p in planes])
        pbs.append(pb)
        pfs.append(pf)
        want.append(ref)
    batch = isp_mw_b200.Batch(ctx, pbs, pfs, dsts, srcs, autotune=autotune)
    for _ in range(2):
        for d in dsts:
            for p in d:
                p.fill_(-1.0)
        batch.run()
        torch.cuda.synchronize()
        for k in range(len(shapes)):
            for c in range(3):
                assert torch.equal(dsts[k][c], want[k][c]), (k, c)
    assert torch.equal(dsts[1][2], srcs[1][2])
    batch.close()
    ctx.close()


def _custom(profile, wiener, sp, bm_step):
    import isp_mw_b200
    p = isp_mw_b200.stage_params_default(profile, wiener, sp)
    if bm_step:
        p.bm_step = bm_step
    return p


@pytest.mark.parametrize("profile,bm_step", [("lc", 0), ("np", 0), ("high", 0), ("vn", 0),
                                             ("fast", 2), ("np", 3)])
def test_batch_other_profiles_equal_per_plane(bm3d_lib, profile, bm_step):
    """Batches of the other profiles (generic kernel for GroupSize 32 and
    BlockSize 11) and of matching steps above 1 (single-row matching
    strips), one and three planes per image, equal per-plane bm3d_full /
    per-image bm3d_full3 bit for bit."""
    import torch
    import isp_mw_b200
    from isp_mw_b200 import synth
    ctx = isp_mw_b200.Context(0)
    shapes = [(70, 96), (101, 83), (64, 130)]
    srcs, dsts, pbs, pfs, want = [], [], [], [], []
    srcs3, dsts3, want3 = [], [], []
    for k, (h, w) in enumerate(shapes):
        s255 = (12.0, 30.0, 45.0)[k]
        src = torch.from_numpy(synth.pair(h, w, s255, 610 + k)[1]).cuda()
        sp = [synth.sigma_param(s255)] * 3
        pb, pf = _custom(profile, False, sp, bm_step), _custom(profile, True, sp, bm_step)
        ref = torch.empty_like(src)
        ctx.full(pb, pf, ref, src)
        srcs.append(src)
        dsts.append(torch.full_like(src, -1.0))
        pbs.append(pb)
        pfs.append(pf)
        want.append(ref)
        planes = [src] + [torch.from_numpy(synth.pair(h, w, 10.0, 640 + 3 * k + c)[1]).cuda()
                          for c in (1, 2)]
        r3 = [torch.empty_like(p) for p in planes]
        ctx.full3(pb, pf, r3, planes)
        srcs3.append(planes)
        dsts3.append([torch.full_like(p, -1.0) for p in planes])
        want3.append(r3)
    batch = isp_mw_b200.Batch(ctx, pbs, pfs, dsts, srcs, autotune=True)
    batch3 = isp_mw_b200.Batch(ctx, pbs, pfs, dsts3, srcs3, autotune=False)
    for _ in range(2):
        batch.run()
        batch3.run()
        torch.cuda.synchronize()
        for k in range(len(shapes)):
            assert torch.equal(dsts[k], want[k]), k
            for c in range(3):
                assert torch.equal(dsts3[k][c], want3[k][c]), (k, c)
    batch.close()
    batch3.close()
    ctx.close()


def test_batch_rejects_bad_planes(bm3d_lib):
    """A plane smaller than a block, or stages whose geometry differs between
    planes, make batch creation fail with BM3D_ERR_INVALID (no launch)."""
    import torch
    import isp_mw_b200
    from isp_mw_b200 import synth
    ctx = isp_mw_b200.Context(0)
    sp = [synth.sigma_param(20.0)] * 3
    pb = isp_mw_b200.stage_params_default("fast", False, sp)
    pf = isp_mw_b200.stage_params_default("fast", True, sp)
    ok = torch.from_numpy(synth.pair(64, 64, 20.0, 1)[1]).cuda()
    tiny = torch.zeros((7, 40), dtype=torch.float32, device="cuda")
    for planes in ([ok, tiny], [tiny]):
        dsts = [torch.empty_like(p) for p in planes]
        with pytest.raises(isp_mw_b200.BM3DError) as e:
            isp_mw_b200.Batch(ctx, [pb] * len(planes), [pf] * len(planes), dsts, planes)
        assert e.value.code == isp_mw_b200.BM3D_ERR_INVALID
    other = isp_mw_b200.stage_params_default("lc", False, sp)  # another block step
    with pytest.raises(isp_mw_b200.BM3DError) as e:
        isp_mw_b200.Batch(ctx, [pb, other], [pf, pf], [torch.empty_like(ok)] * 2, [ok, ok])
    assert e.value.code == isp_mw_b200.BM3D_ERR_INVALID
    ctx.close()


@pytest.mark.parametrize("planes", [1, 3])
def test_final_only_batch_equals_per_plane_final(bm3d_lib, planes):
    """A batch given reference planes (bm3d_batch_final_create /
    bm3d_batch3_final_create: the pilot's estimates in the learned-pilot
    pipeline) runs the final stage only and equals per-plane bm3d_stage
    (wiener = 1) / bm3d_stage3 on the same reference, bit for bit; its stage
    timing reports no basic stage."""
    import torch
    import isp_mw_b200
    from isp_mw_b200 import synth
    ctx = isp_mw_b200.Context(0)
    shapes = [(130, 97), (64, 200), (181, 150)]
    srcs, refs, dsts, pfs, want = [], [], [], [], []
    for k, (h, w) in enumerate(shapes):
        s255 = 12.0 + 9.0 * k
        sp = [synth.sigma_param(s255)] * 3
        pb = isp_mw_b200.stage_params_default("fast", False, sp)
        pf = isp_mw_b200.stage_params_default("fast", True, sp)
        src = [torch.from_numpy(synth.pair(h, w, s255, 500 + 3 * k + c)[1]).cuda()
               for c in range(planes)]
        # any reference plane will do; a smoothed copy of the basic estimate
        basic = [torch.empty_like(x) for x in src]
        if planes == 1:
            ctx.stage(pb, False, basic[0], src[0])
        else:
            ctx.stage3(pb, False, basic, src)
        ref = [(0.9 * b + 0.1 * x).contiguous() for b, x in zip(basic, src)]
        out = [torch.empty_like(x) for x in src]
        if planes == 1:
            ctx.stage(pf, True, out[0], src[0], ref[0])
        else:
            ctx.stage3(pf, True, out, src, ref)
        srcs.append(src if planes == 3 else src[0])
        refs.append(ref if planes == 3 else ref[0])
        dsts.append([torch.full_like(x, -1.0) for x in src] if planes == 3
                    else torch.full_like(src[0], -1.0))
        pfs.append(pf)
        want.append(out)
    batch = isp_mw_b200.Batch(ctx, pfs, pfs, dsts, srcs, autotune=False, ref=refs)
    for _ in range(2):
        batch.run()
        torch.cuda.synchronize()
        for k in range(len(shapes)):
            got = dsts[k] if planes == 3 else [dsts[k]]
            for c in range(planes):
                assert torch.equal(got[c], want[k][c]), (k, c)
    tb, tf = batch.stage_times()
    assert tb < 0.05 and tf > 0.0
    batch.check()
    batch.close()
    ctx.close()
