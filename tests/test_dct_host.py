"""The kernels' DCT building blocks (csrc/dct.cuh), compiled for the host,
against scipy's unnormalised DCT-II / DCT-III, which are FFTW's REDFT10 /
REDFT01 (the transforms the reference plans at source/BM3D.cpp:13-23)."""
import ctypes
import os
import subprocess

import numpy as np
import pytest
import scipy.fft

from conftest import ROOT

BUILD = os.path.join(ROOT, "tests", "_build")


@pytest.fixture(scope="module")
def dctlib():
    os.makedirs(BUILD, exist_ok=True)
    so = os.path.join(BUILD, "libdct_host.so")
    src = os.path.join(ROOT, "tests", "cpp", "dct_host.cpp")
    hdr = os.path.join(ROOT, "isp_mw_b200", "csrc", "dct.cuh")
    if not os.path.exists(so) or os.path.getmtime(so) < max(os.path.getmtime(src),
                                                             os.path.getmtime(hdr)):
        subprocess.run(["g++", "-O2", "-std=c++17", "-ffp-contract=off", "-shared", "-fPIC",
                        "-x", "c++", "-I", os.path.dirname(hdr), src, "-o", so], check=True)
    return ctypes.CDLL(so)


def _run(lib, name, x):
    x = np.ascontiguousarray(x).copy()
    getattr(lib, name)(x.ctypes.data_as(ctypes.c_void_p))
    return x


@pytest.mark.parametrize("n", [8, 16])
@pytest.mark.parametrize("dtype,tol", [(np.float64, 1e-12), (np.float32, 2e-5)])
def test_fast_transforms_match_scipy(dctlib, n, dtype, tol):
    rng = np.random.default_rng(n)
    sfx = "f32" if dtype == np.float32 else "f64"
    for _ in range(50):
        x = rng.standard_normal(n).astype(dtype)
        f = _run(dctlib, f"host_redft10_{n}_{sfx}", x)
        i = _run(dctlib, f"host_redft01_{n}_{sfx}", x)
        ref_f = scipy.fft.dct(x.astype(np.float64), type=2, norm=None)
        ref_i = scipy.fft.dct(x.astype(np.float64), type=3, norm=None)
        scale = np.abs(x).sum() * 2
        assert np.max(np.abs(f - ref_f)) <= tol * scale
        assert np.max(np.abs(i - ref_i)) <= tol * scale
        rt = _run(dctlib, f"host_redft01_{n}_{sfx}", f)
        assert np.max(np.abs(rt - 2 * n * x)) <= 4 * tol * scale * n


@pytest.mark.parametrize("n", range(1, 17))
def test_matrix_transform_lengths(dctlib, n):
    """Every group length 1..16 through the symmetric matrix form the kernels
    instantiate per length (two pencils at once), with the cosine matrices
    the library uploads (row k = output k), against scipy."""
    k = np.arange(n)[:, None]
    j = np.arange(n)[None, :]
    fwd = 2 * np.cos(np.pi * (2 * j + 1) * k / (2 * n))
    inv = np.where(j == 0, 1.0, 2 * np.cos(np.pi * j * (2 * k + 1) / (2 * n)))
    rng = np.random.default_rng(100 + n)
    for mat, typ in ((fwd, 2), (inv, 3)):
        xs = [np.zeros(16), np.zeros(16)]
        for x in xs:
            x[:n] = rng.standard_normal(n)
        a, b = xs[0].copy(), xs[1].copy()
        m = np.ascontiguousarray(mat.ravel())
        dctlib.host_dct_pair_f64(a.ctypes.data_as(ctypes.c_void_p),
                                 b.ctypes.data_as(ctypes.c_void_p), ctypes.c_int(n),
                                 m.ctypes.data_as(ctypes.c_void_p), ctypes.c_int(typ == 3))
        for got, x in ((a, xs[0]), (b, xs[1])):
            ref = scipy.fft.dct(x[:n], type=typ, norm=None)
            assert np.allclose(got[:n], ref, rtol=0, atol=1e-12 * max(1, np.abs(x).sum()) * 4)
            assert np.all(got[n:] == x[n:])


def test_line_transform_32(dctlib):
    """The length-32 symmetric line forms (full GroupSize-32 groups) against
    scipy's DCT-II / DCT-III."""
    n = 32
    k = np.arange(n)[:, None]
    j = np.arange(n)[None, :]
    fwd = 2 * np.cos(np.pi * (2 * j + 1) * k / (2 * n))
    inv = np.where(j == 0, 1.0, 2 * np.cos(np.pi * j * (2 * k + 1) / (2 * n)))
    rng = np.random.default_rng(32)
    for mat, typ in ((fwd, 2), (inv, 3)):
        x = rng.standard_normal(n)
        a = x.copy()
        m = np.ascontiguousarray(mat.ravel())
        dctlib.host_dct_line32_f64(a.ctypes.data_as(ctypes.c_void_p),
                                   m.ctypes.data_as(ctypes.c_void_p), ctypes.c_int(typ == 3))
        ref = scipy.fft.dct(x, type=typ, norm=None)
        assert np.allclose(a, ref, rtol=0, atol=1e-12 * np.abs(x).sum() * 8)


@pytest.mark.parametrize("n", [16, 32])
@pytest.mark.parametrize("dtype,tol", [(np.float64, 1e-12), (np.float32, 2e-6)])
def test_pow2_transforms_match_scipy(dctlib, n, dtype, tol):
    """Lengths 16 and 32 by recursive even/odd splits (the DCT-IV halves as a
    pre-scaled DCT-II plus adjacent sums), as the generic kernel runs full
    GroupSize-32 groups: against scipy's DCT-II / DCT-III, relative to the
    largest output, and the forward-inverse round trip."""
    rng = np.random.default_rng(7 * n)
    sfx = "f32" if dtype == np.float32 else "f64"
    for _ in range(200):
        x = rng.standard_normal(n).astype(dtype)
        f = _run(dctlib, f"host_pow2_redft10_{n}_{sfx}", x)
        i = _run(dctlib, f"host_pow2_redft01_{n}_{sfx}", x)
        ref_f = scipy.fft.dct(x.astype(np.float64), type=2, norm=None)
        ref_i = scipy.fft.dct(x.astype(np.float64), type=3, norm=None)
        assert np.max(np.abs(f - ref_f)) <= tol * np.abs(ref_f).max()
        assert np.max(np.abs(i - ref_i)) <= tol * np.abs(ref_i).max()
        rt = _run(dctlib, f"host_pow2_redft01_{n}_{sfx}", f)
        assert np.max(np.abs(rt - 2 * n * x)) <= 4 * tol * 2 * n * np.abs(x).max()
