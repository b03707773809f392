"""The C++ drop-in header (include/bm3d_b200/BM3D.hpp) used the way the
reference's own classes are used: a C++ program written against the
reference's API compiles unchanged, runs on the GPU, and matches the oracle."""
import os
import subprocess

import numpy as np
import pytest

from conftest import ROOT

pytestmark = pytest.mark.gpu


def test_cpp_dropin_program(bm3d_lib, oracle_mod, tmp_path):
    from isp_mw_b200 import synth
    exe = tmp_path / "dropin_main"
    libdir = os.path.join(ROOT, "isp_mw_b200", "lib")
    subprocess.run(["g++", "-std=c++17", "-O2", "-I", os.path.join(ROOT, "include"),
                    os.path.join(ROOT, "tests", "cpp", "dropin_main.cpp"), "-o", str(exe),
                    "-L", libdir, "-lisp_mw_b200", f"-Wl,-rpath,{libdir}"], check=True)
    h, w, s255 = 120, 176, 25.0
    _, noisy = synth.pair(h, w, s255, 17)
    inp = tmp_path / "in.f32"
    noisy.tofile(inp)
    sp = synth.sigma_param(s255)
    r = subprocess.run([str(exe), str(inp), str(w), str(h), repr(sp), str(tmp_path / "b.f32"),
                        str(tmp_path / "f.f32")], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, (r.returncode, r.stderr)
    basic = np.fromfile(tmp_path / "b.f32", np.float32).reshape(h, w)
    final = np.fromfile(tmp_path / "f.f32", np.float32).reshape(h, w)
    kind = "reference" if oracle_mod.reference_available() else "port"
    orc = oracle_mod.backend(kind, np.float32)
    b = oracle_mod.reference_stage_default("fast", False, [sp] * 3) if kind == "reference" else None
    if b is None:
        import isp_mw_b200
        b = isp_mw_b200.stage_params_default("fast", False, [sp] * 3).as_dict()
        f = isp_mw_b200.stage_params_default("fast", True, [sp] * 3).as_dict()
    else:
        f = oracle_mod.reference_stage_default("fast", True, [sp] * 3)
    rb, rf = orc.full(b, f, noisy)
    assert np.abs(basic - rb).max() <= 1e-3
    assert np.abs(final - rf).max() <= 1e-3


def test_cpp_dropin_frame_and_plane(bm3d_lib, tmp_path):
    """Frame and integer Plane through the C++ drop-in equal the C ABI calls
    they wrap (bm3d_frame, bm3d_stage_frame, bm3d_plane_int)."""
    import isp_mw_b200
    from isp_mw_b200.synth import int_planes
    exe = tmp_path / "dropin_frame"
    libdir = os.path.join(ROOT, "isp_mw_b200", "lib")
    subprocess.run(["g++", "-std=c++17", "-O2", "-I", os.path.join(ROOT, "include"),
                    os.path.join(ROOT, "tests", "cpp", "dropin_frame.cpp"), "-o", str(exe),
                    "-L", libdir, "-lisp_mw_b200", f"-Wl,-rpath,{libdir}"], check=True)
    h, w, s = 72, 104, 30.0
    src = int_planes(h, w, 20.0, 23, 0, 255, 3)
    inp = tmp_path / "in.i32"
    np.stack(src).astype(np.int32).tofile(inp)
    out = tmp_path / "out.i32"
    r = subprocess.run([str(exe), str(inp), str(w), str(h), repr(s), str(out)],
                       capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, (r.returncode, r.stderr)
    got = np.fromfile(out, np.int32).reshape(10, h, w)
    ctx = isp_mw_b200.Context(0)
    b = isp_mw_b200.stage_params_default("fast", False, [s] * 3)
    f = isp_mw_b200.stage_params_default("fast", True, [s] * 3)
    full = [np.empty_like(p) for p in src]
    ctx.frame(b, f, full, src, 0, 255)
    basic = [np.empty_like(p) for p in src]
    ctx.stage_frame(b, False, basic, src, None, 0, 255)
    fin = [np.empty_like(p) for p in src]
    ctx.stage_frame(f, True, fin, src, basic, 0, 255)
    one = np.empty_like(src[0])
    ctx.plane_int(b, f, one, src[0], (0, 0, 255))
    ctx.close()
    want = np.stack(full + basic + fin + [one])
    assert np.array_equal(got, want)
