"""The CPU oracle: the C restatement (oracle/bm3d_oracle_impl.h) is pinned
bit for bit against the reference's own BM3D compiled in place
(oracle/_ref), live when that build exists and always against the committed
golden fixtures that build produced (tests/golden/make_golden.py)."""
import ctypes
import glob
import json
import os
import subprocess

import numpy as np
import pytest

from conftest import ROOT

GOLDEN = sorted(glob.glob(os.path.join(ROOT, "tests", "golden", "*.npz")))
INT_GOLDEN = [p for p in GOLDEN if os.path.basename(p).startswith("int_")]
GOLDEN = [p for p in GOLDEN if p not in INT_GOLDEN]  # float planes


def load(path):
    z = np.load(path)
    return z, json.loads(str(z["params"]))


@pytest.mark.parametrize("path", [p for p in GOLDEN if "fast3" not in p],
                         ids=lambda p: os.path.basename(p))
def test_port_matches_golden(oracle_mod, path):
    z, prm = load(path)
    port = oracle_mod.backend("port", np.float32)
    basic, final = port.full(prm["basic"], prm["final"], z["noisy"])
    assert np.array_equal(basic, z["basic"])
    assert np.array_equal(final, z["final"])
    for stage, plane in (("basic", z["noisy"]), ("final", z["basic"])):
        counts, pos, keys = port.groups(stage == "final", prm[stage], plane)
        assert np.array_equal(counts, z[f"{stage}_counts"])
        assert np.array_equal(pos, z[f"{stage}_pos"])
        assert np.array_equal(keys, z[f"{stage}_keys"])


def test_port_matches_golden_three_planes(oracle_mod):
    z, prm = load(os.path.join(ROOT, "tests", "golden", "fast3_52x40.npz"))
    port = oracle_mod.backend("port", np.float32)
    basic = port.stage3(False, prm["basic"], list(z["noisy"]))
    final = port.stage3(True, prm["final"], list(z["noisy"]), basic)
    assert np.array_equal(np.stack(basic), z["basic"])
    assert np.array_equal(np.stack(final), z["final"])


def test_golden_covers_ties(oracle_mod):
    """The tie fixture really has equal keys inside kept groups."""
    z, _ = load(os.path.join(ROOT, "tests", "golden", "fast_ties_48x40.npz"))
    keys, counts = z["basic_keys"], z["basic_counts"]
    ties = sum(int(np.any(np.diff(keys[r, 1:counts[r]]) == 0)) for r in range(len(counts)))
    assert ties > 0


@pytest.mark.parametrize("dtype", [np.float32, np.float64])
@pytest.mark.parametrize("shape,s255,profile", [((57, 83), 25.0, "fast"), ((40, 31), 5.0, "lc"),
                                               ((24, 24), 50.0, "fast")])
def test_port_matches_reference_live(oracle_mod, dtype, shape, s255, profile):
    if not oracle_mod.reference_available():
        pytest.skip("reference build absent")
    from isp_mw_b200 import synth
    _, noisy = synth.pair(shape[0], shape[1], s255, 77)
    sp = [synth.sigma_param(s255)] * 3
    b = oracle_mod.reference_stage_default(profile, False, sp)
    f = oracle_mod.reference_stage_default(profile, True, sp)
    ref = oracle_mod.backend("reference", dtype)
    port = oracle_mod.backend("port", dtype)
    rb, rf = ref.full(b, f, noisy)
    pb, pf = port.full(b, f, noisy)
    assert np.array_equal(rb, pb) and np.array_equal(rf, pf)


def test_port_param_guard_copies(oracle_mod):
    """Rejected parameters copy src (source/BM3D.cpp:82-87)."""
    from isp_mw_b200 import synth
    _, noisy = synth.pair(32, 32, 10.0, 5)
    port = oracle_mod.backend("port", np.float32)
    p = {"block_size": 8, "block_step": 8, "group_size": 16, "bm_range": 9, "bm_step": 1,
         "thMSE": 1000.0, "lambda": 2.7, "sigma": [0.0, 0.0, 0.0]}
    assert np.array_equal(port.stage(False, p, noisy), noisy)


@pytest.fixture(scope="module")
def std_sort():
    out = os.path.join(ROOT, "tests", "_build")
    os.makedirs(out, exist_ok=True)
    so = os.path.join(out, "libpsort.so")
    src = os.path.join(ROOT, "tests", "cpp", "partial_sort_std.cpp")
    subprocess.run(["g++", "-O2", "-shared", "-fPIC", src, "-o", so], check=True)
    return ctypes.CDLL(so)


def test_partial_sort_emulation_matches_libstdcxx(oracle_mod, std_sort):
    """The heap-select emulation (used by the oracle and, for tied groups, by
    the GPU kernel) reproduces std::partial_sort including its placement of
    equal keys."""
    rng = np.random.default_rng(3)
    for trial in range(400):
        n = int(rng.integers(2, 400))
        m = int(rng.integers(1, min(n, 33) + 1))
        keys = rng.integers(0, max(2, n // int(rng.integers(1, 20))), n).astype(np.float32)
        payload = np.arange(n, dtype=np.int32)
        ek, ep = oracle_mod.partial_sort_f32(keys, payload, m)
        sk, sp = keys.copy(), payload.copy()
        std_sort.std_partial_sort_f32(sk.ctypes.data_as(ctypes.c_void_p),
                                      sp.ctypes.data_as(ctypes.c_void_p), m, n)
        assert np.array_equal(ek[:m], sk[:m]) and np.array_equal(ep[:m], sp[:m]), trial


@pytest.mark.parametrize("path", INT_GOLDEN, ids=lambda p: os.path.basename(p))
def test_port_matches_golden_int(oracle_mod, path):
    """Integer planes and RGB frames: the restatement against the reference's
    BM3D on Plane / Frame (conversions, three stages' outputs), bit for bit."""
    z, prm = load(path)
    port = oracle_mod.backend("port", np.float32)
    src = list(z["src"])
    b, f = prm["basic"], prm["final"]
    if prm["kind"] == "frame":
        bits, pc = prm["bits"], prm["pc"]
        assert np.array_equal(np.stack(port.frame(b, f, src, bits, pc)), z["full"])
        basic = port.stage_frame(False, b, src, None, bits, pc)
        assert np.array_equal(np.stack(basic), z["basic"])
        final = port.stage_frame(True, f, src, list(z["basic"]), bits, pc)
        assert np.array_equal(np.stack(final), z["final"])
    else:
        q = tuple(int(v) for v in z["quant"])
        assert np.array_equal(port.plane_int(b, f, src[0], q), z["full"][0])
        assert np.array_equal(port.stage_int(False, b, src[0], None, q), z["basic"][0])
        assert np.array_equal(port.stage_int(True, f, src[0], z["basic"][0], q), z["final"][0])


@pytest.mark.parametrize("group_size", [0, 1])
def test_port_int_guards(oracle_mod, group_size):
    """GroupSize 1 trips the integer / Frame filters' own guard (exact copy,
    source/BM3D.cpp:250-256, 286-293); GroupSize 0 passes it and trips the
    stage's (a conversion round trip, source/BM3D.cpp:82-87)."""
    z, prm = load(os.path.join(ROOT, "tests", "golden", "int_rgb8_pc_48x56.npz"))
    ref = oracle_mod.backend("reference" if oracle_mod.reference_available() else "port")
    port = oracle_mod.backend("port")
    b = dict(prm["basic"], group_size=group_size)
    src = list(z["src"])
    got = port.stage_frame(False, b, src)
    assert np.array_equal(np.stack(got), np.stack(ref.stage_frame(False, b, src)))
    q = (0, 0, 255)
    assert np.array_equal(port.stage_int(False, b, src[0], None, q),
                          ref.stage_int(False, b, src[0], None, q))
    if group_size == 1:
        assert np.array_equal(np.stack(got), z["src"])


def test_chain_self_divergence_under_fp32_transform(oracle_mod):
    """The reference's own chained basic -> final output is not stable to 1e-3
    under a change of FP32 transform rounding alone, while each stage on
    identical inputs is: evaluating the 3-D DCT in float (three summation
    orders, oracle/dct_ref.h modes 1-3) instead of with double accumulation
    moves the basic estimate by < 1e-6, the final stage on a fixed basic
    estimate by < 1e-5, and the chained final output by several 1e-3 (at
    512x512, sigma 50), because the final stage's block matching on the
    basic estimate flips between nearly equal keys. This is the envelope the
    GPU chain's parity bar is measured against (tests/test_gpu_parity.py)."""
    from isp_mw_b200 import synth
    import isp_mw_b200
    _, noisy = synth.pair(512, 512, 50.0, 6)
    sp = [synth.sigma_param(50.0)] * 3
    b = isp_mw_b200.stage_params_default("fast", False, sp).as_dict()
    f = isp_mw_b200.stage_params_default("fast", True, sp).as_dict()
    port = oracle_mod.backend("port", np.float32)
    rb0, rf0 = port.full(b, f, noisy)
    worst = 0.0
    try:
        for mode in (1, 2, 3):
            oracle_mod.set_f32_transform_mode("port", mode)
            rb, rf = port.full(b, f, noisy)
            fixed = port.stage(True, f, noisy, rb0)
            assert np.abs(rb - rb0).max() < 1e-6
            assert np.abs(fixed - rf0).max() < 1e-5
            d = float(np.abs(rf.astype(np.float64) - rf0).max())
            assert synth.psnr(rf, rf0) >= 60.0
            worst = max(worst, d)
    finally:
        oracle_mod.set_f32_transform_mode("port", 0)
    assert worst > 1e-3, worst


def test_chain_self_divergence_is_near_tie_match_flips(oracle_mod):
    """The reference's own chain, run with its FP32 transform summed in
    another order, exceeds 1e-3 only at pixels of final-stage groups that
    changed between the two runs, and every change is a near-tie (keys within
    1e-3 relative, in practice ~1e-6): the property the GPU chain is held to
    where it exceeds the strict bar (tests/test_gpu_parity.py)."""
    from chain_parity import NEAR_TIE, explain_chain_divergence
    from isp_mw_b200 import synth
    import isp_mw_b200
    _, noisy = synth.pair(512, 512, 50.0, 6)
    sp = [synth.sigma_param(50.0)] * 3
    b = isp_mw_b200.stage_params_default("fast", False, sp)
    f = isp_mw_b200.stage_params_default("fast", True, sp)
    port = oracle_mod.backend("port", np.float32)
    rb0, rf0 = port.full(b.as_dict(), f.as_dict(), noisy)
    g0 = port.groups(True, f.as_dict(), rb0)
    try:
        oracle_mod.set_f32_transform_mode("port", 1)
        rb, rf = port.full(b.as_dict(), f.as_dict(), noisy)
        g1 = port.groups(True, f.as_dict(), rb)
    finally:
        oracle_mod.set_f32_transform_mode("port", 0)
    d = np.abs(rf.astype(np.float64) - rf0)
    assert (d > 1e-3).sum() > 0
    unexplained, worst, flips = explain_chain_divergence(d, g1, g0, f)
    assert unexplained == 0 and worst <= NEAR_TIE and 0 < flips <= 20, (unexplained, worst, flips)
