"""CPU oracle for the BM3D path (test infrastructure only).

Loads, through ctypes:

* ``oracle/_ref/libbm3d_ref_{f32,f64}.so`` -- the reference's own
  ``source/BM3D.cpp`` + ``source/Image_Type.cpp`` compiled in place by
  ``oracle/Makefile`` (present only where the reference tree was available at
  build time; the built files travel with the repository snapshot);
* ``oracle/_build/libbm3d_oracle.so`` -- the C restatement in
  ``oracle/bm3d_oracle_impl.h``, pinned bit-for-bit against the former.

Only ``tests/``, ``__graft_entry__.smoke()`` and the CPU-baseline leg of
``bench.py`` import this package, as the checker. The product
(``isp_mw_b200``) never does.
"""
from __future__ import annotations

import ctypes
import os
import subprocess
from typing import Optional, Sequence

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REF_DIR = os.path.join(HERE, "_ref")
BUILD_DIR = os.path.join(HERE, "_build")
# where the reference checkout lives (read-only; only oracle/Makefile compiles from it)
REFERENCE_TREE = os.environ.get("ISP_MW_REFERENCE", "/root/reference")


class StageParams(ctypes.Structure):
    """Numeric fields of BM3D_Para_Base (include/BM3D.h:15-45)."""

    _fields_ = [
        ("block_size", ctypes.c_int),
        ("block_step", ctypes.c_int),
        ("group_size", ctypes.c_int),
        ("bm_range", ctypes.c_int),
        ("bm_step", ctypes.c_int),
        ("thMSE", ctypes.c_double),
        ("lambda_", ctypes.c_double),
        ("sigma", ctypes.c_double * 3),
    ]

    def as_dict(self) -> dict:
        return {
            "block_size": self.block_size,
            "block_step": self.block_step,
            "group_size": self.group_size,
            "bm_range": self.bm_range,
            "bm_step": self.bm_step,
            "thMSE": self.thMSE,
            "lambda": self.lambda_,
            "sigma": list(self.sigma),
        }


def make_params(d: dict) -> StageParams:
    p = StageParams()
    p.block_size = d["block_size"]
    p.block_step = d["block_step"]
    p.group_size = d["group_size"]
    p.bm_range = d["bm_range"]
    p.bm_step = d["bm_step"]
    p.thMSE = d["thMSE"]
    p.lambda_ = d.get("lambda", 0.0)
    for i in range(3):
        p.sigma[i] = d["sigma"][i]
    return p


def build(reference: bool = True) -> None:
    """Compile the restatement, and the reference when its tree is present."""
    targets = ["port"]
    if reference and os.path.isdir(REFERENCE_TREE):
        targets.append("ref")
    subprocess.run(["make", "-s", "-C", HERE, f"REF={REFERENCE_TREE}"] + targets, check=True)


_libs: dict = {}


def _load(path: str) -> ctypes.CDLL:
    if path not in _libs:
        _libs[path] = ctypes.CDLL(path)
    return _libs[path]


def reference_available() -> bool:
    return os.path.exists(os.path.join(REF_DIR, "libbm3d_ref_f32.so"))


def _ptr(a: np.ndarray):
    return a.ctypes.data_as(ctypes.c_void_p)


class _Backend:
    """One oracle library (reference build or restatement) at one precision."""

    def __init__(self, kind: str, dtype):
        self.kind = kind
        self.dtype = np.dtype(dtype)
        sfx = "f32" if self.dtype == np.float32 else "f64"
        if kind == "reference":
            path = os.path.join(REF_DIR, f"libbm3d_ref_{sfx}.so")
            if not os.path.exists(path):
                raise FileNotFoundError(f"reference oracle not built: {path}")
            self.lib = _load(path)
            self._stage = self.lib.ref_bm3d_stage
            self._stage3 = self.lib.ref_bm3d_stage3
            self._groups = self.lib.ref_bm3d_groups
            self._frame = self.lib.ref_bm3d_frame
            self._plane_int = self.lib.ref_bm3d_plane_int
            self._stage_int = self.lib.ref_bm3d_stage_int
            self._stage_frame = self.lib.ref_bm3d_stage_frame
        elif kind == "port":
            path = os.path.join(BUILD_DIR, "libbm3d_oracle.so")
            if not os.path.exists(path):
                build(reference=False)
            self.lib = _load(path)
            self._stage = getattr(self.lib, f"oracle_bm3d_stage_{sfx}")
            self._stage3 = getattr(self.lib, f"oracle_bm3d_stage3_{sfx}")
            self._groups = getattr(self.lib, f"oracle_bm3d_groups_{sfx}")
            self._frame = getattr(self.lib, f"oracle_bm3d_frame_{sfx}")
            self._plane_int = getattr(self.lib, f"oracle_bm3d_plane_int_{sfx}")
            self._stage_int = getattr(self.lib, f"oracle_bm3d_stage_int_{sfx}")
            self._stage_frame = getattr(self.lib, f"oracle_bm3d_stage_frame_{sfx}")
        else:
            raise ValueError(kind)
        self._stage.restype = ctypes.c_int
        self._stage3.restype = ctypes.c_int
        self._groups.restype = ctypes.c_longlong
        self._frame.restype = ctypes.c_int
        self._plane_int.restype = ctypes.c_int
        self._stage_int.restype = ctypes.c_int
        self._stage_frame.restype = ctypes.c_int

    def stage(self, wiener: bool, params: dict, src: np.ndarray, ref: Optional[np.ndarray] = None,
              value_range: float = 1.0) -> np.ndarray:
        src = np.ascontiguousarray(src, dtype=self.dtype)
        ref = src if ref is None else np.ascontiguousarray(ref, dtype=self.dtype)
        h, w = src.shape
        dst = np.empty_like(src)
        p = make_params(params)
        self._stage(int(wiener), ctypes.byref(p), _ptr(dst), _ptr(src), _ptr(ref), w, h,
                    ctypes.c_double(value_range))
        return dst

    def stage3(self, wiener: bool, params: dict, src: Sequence[np.ndarray],
               ref: Optional[Sequence[np.ndarray]] = None, value_range: float = 1.0):
        src = [np.ascontiguousarray(s, dtype=self.dtype) for s in src]
        ref = src if ref is None else [np.ascontiguousarray(r, dtype=self.dtype) for r in ref]
        h, w = src[0].shape
        dst = [s.copy() for s in src]
        arr = ctypes.c_void_p * 3
        p = make_params(params)
        self._stage3(int(wiener), ctypes.byref(p), arr(*[d.ctypes.data for d in dst]),
                     arr(*[s.ctypes.data for s in src]), arr(*[r.ctypes.data for r in ref]), w, h,
                     ctypes.c_double(value_range))
        return dst

    def groups(self, wiener: bool, params: dict, ref: np.ndarray, value_range: float = 1.0):
        """Group of every reference block: (counts[R], pos[R, G, 2] (y, x), keys[R, G])."""
        ref = np.ascontiguousarray(ref, dtype=self.dtype)
        h, w = ref.shape
        p = make_params(params)
        g = max(1, params["group_size"])
        nrefs = self._groups(int(wiener), ctypes.byref(p), _ptr(ref), w, h,
                             ctypes.c_double(value_range), 0, g, None, None, None)
        counts = np.zeros(nrefs, np.int32)
        pos = np.full((nrefs, g, 2), -1, np.int32)
        keys = np.zeros((nrefs, g), self.dtype)
        self._groups(int(wiener), ctypes.byref(p), _ptr(ref), w, h, ctypes.c_double(value_range),
                     int(nrefs), g, _ptr(counts), _ptr(pos), _ptr(keys))
        return counts, pos, keys

    def frame(self, basic: dict, final: dict, rgb: Sequence[np.ndarray], bits: int = 8,
              pc: bool = True, ref=None):
        """BM3D on an RGB frame of int32 planes (bit depth `bits`, full or
        limited range): OPP conversion, basic (matching on ref's Y when
        given), final, conversion back."""
        src = [np.ascontiguousarray(c, dtype=np.int32) for c in rgb]
        rf = None if ref is None else [np.ascontiguousarray(c, dtype=np.int32) for c in ref]
        h, w = src[0].shape
        dst = [np.empty_like(c) for c in src]
        arr = ctypes.c_void_p * 3
        pb, pf = make_params(basic), make_params(final)
        if self.kind == "reference":
            tail = (int(bits), int(pc))
        else:
            tail = frame_range(bits, pc)
        rc = self._frame(ctypes.byref(pb), ctypes.byref(pf), arr(*[d.ctypes.data for d in dst]),
                         arr(*[c.ctypes.data for c in src]),
                         None if rf is None else arr(*[c.ctypes.data for c in rf]), w, h, *tail)
        if rc != 0:
            raise RuntimeError(f"frame: {rc}")
        return dst

    def plane_int(self, basic: dict, final: dict, src: np.ndarray, quant, bits: int = 8,
                  ref=None):
        """BM3D on an int32 plane quantised as quant = (floor, neutral, ceil)."""
        src = np.ascontiguousarray(src, dtype=np.int32)
        rp = None if ref is None else np.ascontiguousarray(ref, dtype=np.int32)
        h, w = src.shape
        dst = np.empty_like(src)
        q = tuple(int(v) for v in quant)
        tail = ((int(bits),) if self.kind == "reference" else ()) + q
        pb, pf = make_params(basic), make_params(final)
        rc = self._plane_int(ctypes.byref(pb), ctypes.byref(pf), _ptr(dst), _ptr(src),
                             None if rp is None else _ptr(rp), w, h, *tail)
        if rc != 0:
            raise RuntimeError(f"plane_int: {rc}")
        return dst

    def stage_int(self, wiener: bool, params: dict, src: np.ndarray, ref=None, quant=(0, 0, 255),
                  bits: int = 8):
        """One stage on an int32 plane quantised as (floor, neutral, ceil)."""
        src = np.ascontiguousarray(src, dtype=np.int32)
        rp = None if ref is None else np.ascontiguousarray(ref, dtype=np.int32)
        h, w = src.shape
        dst = np.empty_like(src)
        q = tuple(int(v) for v in quant)
        tail = ((int(bits),) if self.kind == "reference" else ()) + q
        p = make_params(params)
        self._stage_int(int(wiener), ctypes.byref(p), _ptr(dst), _ptr(src),
                        None if rp is None else _ptr(rp), w, h, *tail)
        return dst

    def stage_frame(self, wiener: bool, params: dict, rgb, ref=None, bits: int = 8,
                    pc: bool = True):
        """One stage on an RGB frame of int32 planes."""
        src = [np.ascontiguousarray(c, dtype=np.int32) for c in rgb]
        rf = None if ref is None else [np.ascontiguousarray(c, dtype=np.int32) for c in ref]
        h, w = src[0].shape
        dst = [np.empty_like(c) for c in src]
        arr = ctypes.c_void_p * 3
        tail = (int(bits), int(pc)) if self.kind == "reference" else frame_range(bits, pc)
        p = make_params(params)
        self._stage_frame(int(wiener), ctypes.byref(p), arr(*[d.ctypes.data for d in dst]),
                          arr(*[c.ctypes.data for c in src]),
                          None if rf is None else arr(*[c.ctypes.data for c in rf]), w, h, *tail)
        return dst

    def full(self, basic: dict, final: dict, src: np.ndarray, value_range: float = 1.0):
        """Basic then final, tmp sized from src (the working BM3D sequence)."""
        tmp = self.stage(False, basic, src, src, value_range)
        return tmp, self.stage(True, final, src, tmp, value_range)


def frame_range(bits: int, pc: bool = True):
    """Floor and Ceil of an RGB plane (include/Image_Type.hpp:94-109, GetQuanPara):
    full range [0, 2^bits - 1], limited range [16, 235] << (bits - 8)."""
    if pc:
        return 0, (1 << bits) - 1
    return 16 << (bits - 8), 235 << (bits - 8)


def plane_quant(bits: int, pc: bool = True, chroma: bool = False):
    """(Floor, Neutral, Ceil) of an integer plane (include/Image_Type.hpp:94-109)."""
    if pc:
        lo, hi = 0, (1 << bits) - 1
    else:
        lo, hi = 16 << (bits - 8), (240 if chroma else 235) << (bits - 8)
    return lo, (1 << (bits - 1)) if chroma else lo, hi


def backend(kind: str = "port", dtype=np.float32) -> _Backend:
    return _Backend(kind, dtype)


def set_f32_transform_mode(kind: str, mode: int) -> int:
    """Select how the FP32 oracle evaluates its 3-D DCT (see
    ``oracle_dct_set_f32_mode`` in oracle/dct_ref.h): 0 = double accumulation
    (the default the fixtures were made with), 1 / 2 / 3 = float arithmetic
    per axis, terms summed forward / backward / pairwise. Returns the previous
    mode."""
    path = (os.path.join(REF_DIR, "libbm3d_ref_f32.so") if kind == "reference"
            else os.path.join(BUILD_DIR, "libbm3d_oracle.so"))
    lib = _load(path)
    old = int(lib.oracle_dct_get_f32_mode())
    lib.oracle_dct_set_f32_mode(int(mode))
    return old


def reference_stage_default(profile: str, wiener: bool, sigma: Sequence[float]) -> dict:
    """Profile defaults from the compiled reference's own parameter classes."""
    lib = _load(os.path.join(REF_DIR, "libbm3d_ref_f32.so"))
    out = StageParams()
    s = (ctypes.c_double * 3)(*sigma)
    rc = lib.ref_stage_default(profile.encode(), int(wiener), s, ctypes.byref(out))
    if rc != 0:
        raise ValueError(profile)
    return out.as_dict()


def partial_sort_f32(keys: np.ndarray, payload: np.ndarray, m: int):
    """The restatement's libstdc++ partial_sort emulation (for pinning)."""
    lib = _load(os.path.join(BUILD_DIR, "libbm3d_oracle.so"))
    k = np.ascontiguousarray(keys, dtype=np.float32).copy()
    p = np.ascontiguousarray(payload, dtype=np.int32).copy()
    lib.oracle_partial_sort_f32(_ptr(k), _ptr(p), int(m), int(k.size))
    return k, p
