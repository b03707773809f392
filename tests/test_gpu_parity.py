"""GPU parity: the CUDA path, called through the C ABI, against the oracle.

Bars (from the task's north star): matched group indices agree on >= 99.9 %
of reference blocks (here exactly on identical inputs), and outputs agree
within max-abs 1e-3 and >= 60 dB PSNR-to-reference on a [0, 1] scale. Every
test also states the error of the FP32 kernels against an FP64 run of the
same kernels where that is meaningful.
"""
import glob
import json
import os

import numpy as np
import pytest

from conftest import ROOT

pytestmark = pytest.mark.gpu

MAX_ABS = 1e-3
MIN_PSNR = 60.0
GOLDEN = sorted(glob.glob(os.path.join(ROOT, "tests", "golden", "*.npz")))
INT_GOLDEN = [p for p in GOLDEN if os.path.basename(p).startswith("int_")]
GOLDEN = [p for p in GOLDEN if p not in INT_GOLDEN]  # float planes
# one JSON line per comparison; PARITY_REPORT chooses the file
REPORT = os.environ.get("PARITY_REPORT",
                        os.path.join(ROOT, "tests", "_build", "parity_report.jsonl"))


def report(**kw):
    try:
        os.makedirs(os.path.dirname(REPORT), exist_ok=True)
        with open(REPORT, "a") as f:
            f.write(json.dumps(kw) + "\n")
    except OSError:
        pass


@pytest.fixture(scope="module")
def ctx(bm3d_lib):
    import isp_mw_b200
    c = isp_mw_b200.Context(0)
    yield c
    c.close()


def P(d):
    import isp_mw_b200
    return isp_mw_b200.StageParams.from_dict(d)


def psnr_to(a, b):
    from isp_mw_b200.synth import psnr
    return psnr(a, b)


def assert_close(name, got, want):
    d = np.abs(got.astype(np.float64) - want.astype(np.float64))
    p = psnr_to(got, want)
    report(test=name, max_abs=float(d.max()), psnr=p, n_over=int((d > MAX_ABS).sum()))
    assert d.max() <= MAX_ABS, (name, float(d.max()), int((d > MAX_ABS).sum()))
    assert p >= MIN_PSNR, (name, p)


def group_match(name, gpu, ref, keys=True):
    """Fraction of reference blocks whose group (positions in order, and the
    keys bit for bit when `keys`) equals the oracle's."""
    gc, gp, gk = gpu
    rc, rp, rk = ref
    assert len(gc) == len(rc)
    same = 0
    for r in range(len(rc)):
        n = rc[r]
        if gc[r] == n and np.array_equal(gp[r, :n], rp[r, :n]) and (
                not keys or np.array_equal(gk[r, :n], rk[r, :n])):
            same += 1
    frac = same / len(rc)
    report(test=name, groups=len(rc), group_match=frac)
    return frac


@pytest.mark.parametrize("path", [p for p in GOLDEN if "fast3" not in p],
                         ids=lambda p: os.path.basename(p))
def test_golden_groups_exact(ctx, path):
    """Groups on identical inputs equal the reference's, ties included."""
    z = np.load(path)
    prm = json.loads(str(z["params"]))
    for stage, plane in (("basic", z["noisy"]), ("final", z["basic"])):
        gpu = ctx.debug_groups(P(prm[stage]), stage == "final", plane)
        ref = (z[f"{stage}_counts"], z[f"{stage}_pos"], z[f"{stage}_keys"])
        frac = group_match(os.path.basename(path) + ":" + stage, gpu, ref)
        assert frac == 1.0


@pytest.mark.parametrize("path", [p for p in GOLDEN if "fast3" not in p],
                         ids=lambda p: os.path.basename(p))
def test_golden_outputs(ctx, path):
    z = np.load(path)
    prm = json.loads(str(z["params"]))
    noisy = z["noisy"]
    basic = np.empty_like(noisy)
    ctx.stage(P(prm["basic"]), False, basic, noisy)
    assert_close(os.path.basename(path) + ":basic", basic, z["basic"])
    # final stage on the reference's own basic estimate: isolates the stage
    final = np.empty_like(noisy)
    ctx.stage(P(prm["final"]), True, final, noisy, z["basic"])
    assert_close(os.path.basename(path) + ":final", final, z["final"])
    # the combined entry point, end to end
    full = np.empty_like(noisy)
    ctx.full(P(prm["basic"]), P(prm["final"]), full, noisy)
    assert_close(os.path.basename(path) + ":full", full, z["final"])


def test_golden_three_planes(ctx):
    z = np.load(os.path.join(ROOT, "tests", "golden", "fast3_52x40.npz"))
    prm = json.loads(str(z["params"]))
    src = [np.ascontiguousarray(p) for p in z["noisy"]]
    basic = [np.empty_like(s) for s in src]
    ctx.stage3(P(prm["basic"]), False, basic, src)
    for c in range(3):
        assert_close(f"fast3:basic:{c}", basic[c], z["basic"][c])
    final = [np.empty_like(s) for s in src]
    ctx.stage3(P(prm["final"]), True, final, src, [np.ascontiguousarray(b) for b in z["basic"]])
    for c in range(3):
        assert_close(f"fast3:final:{c}", final[c], z["final"][c])
    full = [np.empty_like(s) for s in src]
    ctx.full3(P(prm["basic"]), P(prm["final"]), full, src)
    for c in range(3):
        assert_close(f"fast3:full:{c}", full[c], z["final"][c])


def _oracle(oracle_mod, dtype=np.float32):
    kind = "reference" if oracle_mod.reference_available() else "port"
    return oracle_mod.backend(kind, dtype)


# The chained pipeline's bar. Its final stage matches blocks on the basic
# estimate, so a basic estimate that differs from the reference's in the 7th
# digit flips matches between nearly equal keys, and each flip moves a few
# pixels by up to ~1e-2. The reference does the same to itself: run with its
# transform evaluated in FP32 (three summation orders, oracle/dct_ref.h modes
# 1-3) instead of the double-accumulating default, its own chained output moves
# by up to 1.1e-2 at 1080p (CPU test in test_oracle.py; the envelope is also
# measured here and reported). Such flips are rare events, so an envelope of a
# few samples is no bound: where the chained max-abs is above 1e-3 the test
# instead explains every excess pixel. Each pixel over 1e-3 must lie in the
# footprint of a final-stage group that differs between the two chains, and
# each such difference must be a near-tie: at every rank the two groups' keys
# agree within NEAR_TIE relative, and a member only one chain keeps sits within
# NEAR_TIE of the matching threshold.
from chain_parity import NEAR_TIE, explain_chain_divergence  # noqa: E402

ENV_MODES = (1, 2, 3)


def chain_envelope(oracle_mod, orc, b, f, noisy, rf0):
    """Divergence of the reference's chain from itself (mode 0) when only its
    FP32 transform rounding changes: max over modes 1-3 of max-abs and pixel
    count over 1e-3, and the largest MSE."""
    env = {"max_abs": 0.0, "n_over": 0, "mse": 0.0}
    try:
        for mode in ENV_MODES:
            oracle_mod.set_f32_transform_mode("reference", mode)
            rb = orc.stage(False, b, noisy)
            rf = orc.stage(True, f, noisy, rb)
            d = np.abs(rf.astype(np.float64) - rf0.astype(np.float64))
            env["max_abs"] = max(env["max_abs"], float(d.max()))
            env["n_over"] = max(env["n_over"], int((d > MAX_ABS).sum()))
            env["mse"] = max(env["mse"], float(np.mean(d * d)))
    finally:
        oracle_mod.set_f32_transform_mode("reference", 0)
    return env


@pytest.mark.parametrize("shape,s255,seed", [((512, 512), 25.0, 0), ((1080, 1920), 25.0, 1),
                                             ((1080, 1920), 5.0, 2), ((1080, 1920), 50.0, 3),
                                             ((1080, 1920), 10.0, 7), ((301, 257), 10.0, 4),
                                             ((512, 512), 50.0, 6)])
def test_against_oracle(ctx, oracle_mod, shape, s255, seed):
    """Seeded workloads of the benchmark's shapes.

    Each stage is held to the strict bar on identical inputs: group lists
    (>= 99.9 %, exact in practice) and max-abs <= 1e-3 / >= 60 dB. The chained
    pipeline (final stage fed by our own basic estimate) against the
    reference's own chain: max-abs <= 1e-3, or, where that is exceeded, every
    excess pixel explained by a near-tie final-stage match flip (NEAR_TIE
    above), and always >= 60 dB with >= 99.9 % of final groups matched. The error of the FP32
    result against an FP64 run of the same kernels is reported too."""
    from isp_mw_b200 import synth
    import isp_mw_b200
    clean, noisy = synth.pair(shape[0], shape[1], s255, seed)
    sp = [synth.sigma_param(s255)] * 3
    b = isp_mw_b200.stage_params_default("fast", False, sp)
    f = isp_mw_b200.stage_params_default("fast", True, sp)
    orc = _oracle(oracle_mod)
    name = f"{shape[1]}x{shape[0]}_s{s255:g}"
    # basic stage, identical inputs
    rb = orc.stage(False, b.as_dict(), noisy)
    gb = ctx.debug_groups(b, False, noisy)
    assert group_match(name + ":basic_groups", gb, orc.groups(False, b.as_dict(), noisy)) >= 0.999
    basic = np.empty_like(noisy)
    ctx.stage(b, False, basic, noisy)
    assert_close(name + ":basic", basic, rb)
    # final stage, identical inputs (the oracle's final on our basic estimate)
    rf_on_ours = orc.stage(True, f.as_dict(), noisy, basic)
    gf = ctx.debug_groups(f, True, basic)
    assert group_match(name + ":final_groups", gf, orc.groups(True, f.as_dict(), basic)) >= 0.999
    final = np.empty_like(noisy)
    ctx.stage(f, True, final, noisy, basic)
    assert_close(name + ":final", final, rf_on_ours)
    # chained pipeline against the reference's own chain
    rf = orc.stage(True, f.as_dict(), noisy, rb)
    full = np.empty_like(noisy)
    ctx.full(b, f, full, noisy)
    rgf = orc.groups(True, f.as_dict(), rb)
    frac = group_match(name + ":final_groups_chained", gf, rgf, keys=False)
    d = np.abs(full.astype(np.float64) - rf)
    max_abs, n_over, mse = float(d.max()), int((d > MAX_ABS).sum()), float(np.mean(d * d))
    p_ref = psnr_to(full, rf)
    rec = dict(test=name + ":full_chained", max_abs=max_abs, psnr=p_ref, n_over=n_over,
               frac_over=float((d > MAX_ABS).mean()))
    if max_abs > MAX_ABS:
        unexplained, worst, flips = explain_chain_divergence(d, gf, rgf, f)
        rec.update(flipped_groups=flips, worst_key_gap=worst, unexplained=unexplained)
        if orc.kind == "reference":
            env = chain_envelope(oracle_mod, orc, b.as_dict(), f.as_dict(), noisy, rf)
            rec.update(env_max_abs=env["max_abs"], env_n_over=env["n_over"], env_mse=env["mse"])
        report(**rec)
        assert unexplained == 0, (name, rec)
        assert worst <= NEAR_TIE, (name, rec)
    else:
        report(**rec)
    assert p_ref >= MIN_PSNR and frac >= 0.999, (name, p_ref, frac)
    assert np.array_equal(full, final)  # bm3d_full == stage + stage, bit for bit
    # FP64 run of the same kernels: error of the FP32 result against it
    n64 = noisy.astype(np.float64)
    b64 = np.empty_like(n64)
    ctx.stage(b, False, b64, n64)
    f64 = np.empty_like(n64)
    ctx.stage(f, True, f64, n64, b64)
    report(test=name + ":fp32_vs_fp64", max_abs=float(np.abs(full - f64).max()),
           psnr=psnr_to(full, f64), psnr_clean_fp32=psnr_to(full, clean),
           psnr_clean_ref=psnr_to(rf, clean), psnr_noisy=psnr_to(noisy, clean))


def test_fp64_kernels_match_fp64_oracle(ctx, oracle_mod):
    from isp_mw_b200 import synth
    import isp_mw_b200
    _, noisy = synth.pair(128, 160, 25.0, 9)
    sp = [synth.sigma_param(25.0)] * 3
    b = isp_mw_b200.stage_params_default("fast", False, sp)
    f = isp_mw_b200.stage_params_default("fast", True, sp)
    orc = _oracle(oracle_mod, np.float64)
    rb, rf = orc.full(b.as_dict(), f.as_dict(), noisy.astype(np.float64))
    n64 = noisy.astype(np.float64)
    gb = np.empty_like(n64)
    ctx.stage(b, False, gb, n64)
    gf = np.empty_like(n64)
    ctx.stage(f, True, gf, n64, gb)
    d = np.abs(gf - rf).max()
    report(test="fp64_vs_fp64_oracle", max_abs=float(d))
    assert d < 1e-9


def test_device_mode_matches_host_mode(ctx):
    import torch
    from isp_mw_b200 import synth
    import isp_mw_b200
    _, noisy = synth.pair(200, 333, 25.0, 21)
    sp = [synth.sigma_param(25.0)] * 3
    b = isp_mw_b200.stage_params_default("fast", False, sp)
    f = isp_mw_b200.stage_params_default("fast", True, sp)
    host = np.empty_like(noisy)
    ctx.full(b, f, host, noisy)
    # pitched device planes: stride > width
    big = torch.zeros((200, 352), dtype=torch.float32, device="cuda")
    big[:, :333] = torch.from_numpy(noisy).cuda()
    src = big[:, :333]
    dst_big = torch.full((200, 352), -7.0, dtype=torch.float32, device="cuda")
    dst = dst_big[:, :333]
    ctx.full(b, f, dst, src)
    torch.cuda.synchronize()
    got = dst.cpu().numpy()
    assert np.abs(got - host).max() <= 1e-5
    assert torch.all(dst_big[:, 333:] == -7.0)
    ctx.check()  # bm3d_check: the asynchronous calls' consistency counter stayed 0


def test_param_guard_copies_src(ctx):
    import isp_mw_b200
    from isp_mw_b200 import synth
    _, noisy = synth.pair(48, 48, 10.0, 1)
    p = isp_mw_b200.stage_params_default("fast", False, (0.0, 0.0, 0.0))
    dst = np.zeros_like(noisy)
    assert ctx.stage(p, False, dst, noisy) == isp_mw_b200.BM3D_COPIED
    assert np.array_equal(dst, noisy)


def test_invalid_and_unsupported(ctx):
    import isp_mw_b200
    p = isp_mw_b200.stage_params_default("fast", False, (20.0, 20.0, 20.0))
    small = np.zeros((7, 40), np.float32)
    with pytest.raises(isp_mw_b200.BM3DError) as e:
        ctx.stage(p, False, np.empty_like(small), small)
    assert e.value.code == isp_mw_b200.BM3D_ERR_INVALID
    q = isp_mw_b200.stage_params_default("vn", True, (20.0, 20.0, 20.0))
    q.block_size = 17  # beyond the largest block size built (16)
    x = np.zeros((64, 64), np.float32)
    with pytest.raises(isp_mw_b200.BM3DError) as e:
        ctx.stage(q, True, np.empty_like(x), x, x)
    assert e.value.code == isp_mw_b200.BM3D_ERR_UNSUPPORTED


def test_tiling_and_reruns_are_bit_identical(ctx, oracle_mod):
    """Integer aggregation makes results independent of the tile shape, warp
    count and scheduling: every configuration gives the same bits."""
    from isp_mw_b200 import synth
    import isp_mw_b200
    _, noisy = synth.pair(150, 170, 25.0, 31)
    sp = [synth.sigma_param(25.0)] * 3
    b = isp_mw_b200.stage_params_default("fast", False, sp)
    f = isp_mw_b200.stage_params_default("fast", True, sp)
    rb, rf = _oracle(oracle_mod).full(b.as_dict(), f.as_dict(), noisy)
    outs = []
    try:
        for tiling in [(8, 8, 16), (1, 1, 1), (3, 5, 4), (16, 4, 8), (8, 8, 16)]:
            ctx.set_tiling(*tiling)
            out = np.empty_like(noisy)
            ctx.full(b, f, out, noisy)
            outs.append(out)
    finally:
        ctx.set_tiling(8, 8, 16)
    for o in outs[1:]:
        assert np.array_equal(o, outs[0])
    report(test="tiling_full_vs_oracle", max_abs=float(np.abs(outs[0] - rf).max()),
           psnr=psnr_to(outs[0], rf))
    assert psnr_to(outs[0], rf) >= MIN_PSNR


def test_value_range_scales_matching(ctx, oracle_mod):
    """A plane on a 0..255 scale with ValueRange 255 (include/Block.h:582)."""
    from isp_mw_b200 import synth
    import isp_mw_b200
    _, noisy = synth.pair(96, 96, 25.0, 41)
    noisy = (noisy * 255).astype(np.float32)
    sp = [synth.sigma_param(25.0)] * 3
    b = isp_mw_b200.stage_params_default("fast", False, sp)
    orc = _oracle(oracle_mod)
    ref = orc.stage(False, b.as_dict(), noisy, value_range=255.0)
    out = np.empty_like(noisy)
    ctx.stage(b, False, out, noisy, value_range=255.0)
    d = np.abs(out - ref).max() / 255.0
    report(test="value_range_255", max_abs_scaled=float(d))
    assert d <= MAX_ABS


@pytest.mark.parametrize("profile,shape,s255", [("lc", (200, 256), 15.0), ("np", (128, 160), 20.0),
                                                ("high", (96, 120), 35.0), ("vn", (128, 160), 15.0)])
def test_profiles_against_oracle(ctx, oracle_mod, profile, shape, s255):
    """Every reference profile (include/BM3D.h:27-151): np/high final and both vn
    stages (GroupSize 32, BlockSize 11, BMrange 16) run on the generic kernel."""
    from isp_mw_b200 import synth
    import isp_mw_b200
    _, noisy = synth.pair(shape[0], shape[1], s255, 50)
    sp = [synth.sigma_param(s255)] * 3
    b = isp_mw_b200.stage_params_default(profile, False, sp)
    f = isp_mw_b200.stage_params_default(profile, True, sp)
    orc = _oracle(oracle_mod)
    name = f"{profile}_{shape[1]}x{shape[0]}_s{s255:g}"
    rb = orc.stage(False, b.as_dict(), noisy)
    assert group_match(name + ":basic_groups", ctx.debug_groups(b, False, noisy),
                       orc.groups(False, b.as_dict(), noisy)) >= 0.999
    basic = np.empty_like(noisy)
    ctx.stage(b, False, basic, noisy)
    assert_close(name + ":basic", basic, rb)
    assert group_match(name + ":final_groups", ctx.debug_groups(f, True, basic),
                       orc.groups(True, f.as_dict(), basic)) >= 0.999
    final = np.empty_like(noisy)
    ctx.stage(f, True, final, noisy, basic)
    assert_close(name + ":final", final, orc.stage(True, f.as_dict(), noisy, basic))


@pytest.mark.parametrize("shape", [(8, 8), (8, 40), (40, 8), (9, 9), (16, 300), (300, 16),
                                   (0, 0)], ids=lambda s: f"{s[1]}x{s[0]}")
def test_edge_sizes_against_oracle(ctx, oracle_mod, shape):
    """Planes of one block, one block row or column, and thin strips: each
    stage on identical inputs against the oracle (groups exact, outputs within
    the bar), one and three planes. An empty plane is rejected."""
    import isp_mw_b200
    from isp_mw_b200 import synth
    sp = [synth.sigma_param(25.0)] * 3
    b = isp_mw_b200.stage_params_default("fast", False, sp)
    f = isp_mw_b200.stage_params_default("fast", True, sp)
    h, w = shape
    if h == 0:  # straight through the C ABI: the Python wrapper refuses empty arrays itself
        import ctypes
        buf = np.zeros(64, np.float32)
        for w0, h0 in ((0, 0), (0, 8), (8, 0)):
            rc = ctx.lib.bm3d_stage(ctx.h, ctypes.byref(b), 0, buf.ctypes.data, buf.ctypes.data,
                                    buf.ctypes.data, w0, h0, 8, 1.0, isp_mw_b200.MEM_HOST, None)
            assert rc == isp_mw_b200.BM3D_ERR_INVALID
        return
    orc = _oracle(oracle_mod)
    _, noisy = synth.pair(h, w, 25.0, 60 + h + w)
    name = f"edge_{w}x{h}"
    gb = ctx.debug_groups(b, False, noisy)
    assert group_match(name + ":basic_groups", gb, orc.groups(False, b.as_dict(), noisy)) == 1.0
    basic = np.empty_like(noisy)
    ctx.stage(b, False, basic, noisy)
    assert_close(name + ":basic", basic, orc.stage(False, b.as_dict(), noisy))
    final = np.empty_like(noisy)
    ctx.stage(f, True, final, noisy, basic)
    assert_close(name + ":final", final, orc.stage(True, f.as_dict(), noisy, basic))
    planes = [synth.pair(h, w, 25.0, 70 + c)[1] for c in range(3)]
    b3 = [p.copy() for p in planes]
    ctx.stage3(b, False, b3, planes)
    want = orc.stage3(False, b.as_dict(), planes)
    for c in range(3):
        assert_close(name + f":basic3_{c}", b3[c], want[c])


@pytest.mark.parametrize("profile", ["fast", "np", "vn"])
def test_three_planes_against_oracle(ctx, oracle_mod, profile):
    """Three planes sharing luma groups on the register-resident kernel (fast,
    planes run one at a time) and the generic kernel (np: GroupSize 32; vn:
    BlockSize 11), each stage on identical inputs against the oracle."""
    import isp_mw_b200
    from isp_mw_b200 import synth
    h, w = 96, 136
    planes = [synth.pair(h, w, s, 80 + c)[1] for c, s in enumerate((15.0, 10.0, 10.0))]
    sp = [synth.sigma_param(15.0, 0), synth.sigma_param(10.0, 1), synth.sigma_param(10.0, 2)]
    b = isp_mw_b200.stage_params_default(profile, False, sp)
    f = isp_mw_b200.stage_params_default(profile, True, sp)
    orc = _oracle(oracle_mod)
    basic = [p.copy() for p in planes]
    ctx.stage3(b, False, basic, planes)
    rb = orc.stage3(False, b.as_dict(), planes)
    for c in range(3):
        assert_close(f"{profile}3:basic:{c}", basic[c], rb[c])
    final = [p.copy() for p in planes]
    ctx.stage3(f, True, final, planes, basic)
    rf = orc.stage3(True, f.as_dict(), planes, basic)
    for c in range(3):
        assert_close(f"{profile}3:final:{c}", final[c], rf[c])


def test_every_group_length_against_oracle(ctx, oracle_mod):
    """Groups of every length 1..16 (σ 50 on a 256x192 plane makes them all,
    in both stages) through the FP32 group-axis transforms: butterflies for 8
    and 16, one runtime-length loop for the others. Both stages on identical
    inputs meet the strict bar, and the group lists are the oracle's."""
    from isp_mw_b200 import synth
    import isp_mw_b200
    s255 = 50.0
    _, noisy = synth.pair(192, 256, s255, 77)
    sp = [synth.sigma_param(s255)] * 3
    b = isp_mw_b200.stage_params_default("fast", False, sp)
    f = isp_mw_b200.stage_params_default("fast", True, sp)
    orc = _oracle(oracle_mod)
    rb = orc.stage(False, b.as_dict(), noisy)
    for wiener, p, ref in ((False, b, noisy), (True, f, rb)):
        name = "every_length:" + ("final" if wiener else "basic")
        g = ctx.debug_groups(p, wiener, ref)
        lengths = set(np.unique(g[0]).tolist())
        assert lengths == set(range(1, 17)), sorted(lengths)
        assert group_match(name + "_groups", g, orc.groups(wiener, p.as_dict(), ref)) == 1.0
        want = orc.stage(wiener, p.as_dict(), noisy, ref if wiener else None)
        got = np.empty_like(noisy)
        ctx.stage(p, wiener, got, noisy, ref if wiener else None)
        assert_close(name, got, want)
