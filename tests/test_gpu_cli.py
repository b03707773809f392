"""The command-line front end (isp_mw --bm3d ..., the reference's
`ISP_MW --bm3d` with raw files in place of images) gives the same result as
the library calls it wraps."""
import os
import subprocess

import numpy as np
import pytest

from conftest import ROOT

pytestmark = pytest.mark.gpu

CLI = os.path.join(ROOT, "isp_mw_b200", "lib", "isp_mw")


def run(args):
    r = subprocess.run([CLI, "--bm3d"] + args, capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    return r.stdout.strip()


def params(s255):
    import isp_mw_b200
    return (isp_mw_b200.stage_params_default("fast", False, [s255] * 3),
            isp_mw_b200.stage_params_default("fast", True, [s255] * 3))


def test_cli_rgb8(tmp_path, bm3d_lib):
    import isp_mw_b200
    from isp_mw_b200.synth import int_planes
    h, w = 72, 96
    src = int_planes(h, w, 20.0, 31, 0, 255, 3)
    path = tmp_path / "img.raw"
    np.stack(src).astype(np.uint8).tofile(path)
    out = run(["-S", "34.64", "-W", str(w), "-H", str(h), str(path)])
    assert out == str(tmp_path / "img.BM3D.raw")
    got = np.fromfile(out, np.uint8).reshape(3, h, w)
    ctx = isp_mw_b200.Context(0)
    b, f = params(34.64)
    want = [np.empty_like(p) for p in src]
    ctx.frame(b, f, want, src, 0, 255)
    ctx.close()
    assert np.array_equal(got, np.stack(want).astype(np.uint8))


def test_cli_gray16_tv_with_ref_and_tag(tmp_path, bm3d_lib):
    import isp_mw_b200
    from isp_mw_b200.synth import int_planes
    h, w = 64, 80
    lo, hi = 16 << 8, 235 << 8
    src = int_planes(h, w, 15.0, 32, lo, hi, 1)[0]
    ref = int_planes(h, w, 5.0, 32, lo, hi, 1)[0]
    sp, rp = tmp_path / "y.raw", tmp_path / "r.raw"
    src.astype("<u2").tofile(sp)
    ref.astype("<u2").tofile(rp)
    out = run(["--type", "gray", "--depth", "16", "--tv", "-S", "25", "-T", ".dn", "-F", ".u16",
               "--ref", str(rp), "-W", str(w), "-H", str(h), str(sp)])
    assert out == str(tmp_path / "y.dn.u16")
    got = np.fromfile(out, "<u2").reshape(h, w).astype(np.int32)
    ctx = isp_mw_b200.Context(0)
    b, f = params(25.0)
    want = np.empty_like(src)
    ctx.plane_int(b, f, want, src, (lo, lo, hi), ref=ref)
    ctx.close()
    assert np.array_equal(got, want)


def test_cli_float_profile_and_stage_overrides(tmp_path, bm3d_lib):
    import isp_mw_b200
    from isp_mw_b200 import synth
    h, w = 60, 70
    _, noisy = synth.pair(h, w, 25.0, 33)
    path = tmp_path / "f.f32"
    noisy.astype(np.float32).tofile(path)
    out = run(["--type", "float", "-P", "lc", "-S", "43.3", "-MR1", "6", "-GS2", "8",
               "-W", str(w), "-H", str(h), str(path)])
    got = np.fromfile(out, np.float32).reshape(h, w)
    b = isp_mw_b200.stage_params_default("lc", False, [43.3] * 3)
    f = isp_mw_b200.stage_params_default("lc", True, [43.3] * 3)
    b.bm_range = 6
    f.group_size = 8
    ctx = isp_mw_b200.Context(0)
    want = np.empty_like(noisy)
    ctx.full(b, f, want, noisy)
    ctx.close()
    assert np.array_equal(got, want)
