"""isp_mw_b200: B200-native BM3D behind the C ABI of ``include/bm3d_b200.h``.

Python binding over ``lib/libisp_mw_b200.so`` (ctypes). It mirrors the
reference's BM3D filter API (mawen1250/ISP_MW ``include/BM3D.h``):
``BM3D_Basic_Para`` / ``BM3D_Final_Para`` / ``BM3D_Para`` with their profiles
and ``thMSE_Default``, and filters ``BM3D_Basic``, ``BM3D_Final`` and ``BM3D``
whose ``process(dst, src[, ref])`` / ``__call__(src[, ref])`` follow
``FilterIF2`` (``include/Filter.h:138-217``). Planes are numpy arrays (host
memory: copied in and out) or CUDA torch tensors (device memory: work is
enqueued on the current torch stream).

There is no CPU path: without the compiled library or a B200 every call raises.
"""
from __future__ import annotations

import ctypes
import os
from typing import Optional, Sequence

import numpy as np

PKG = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(PKG, "lib", "libisp_mw_b200.so")

BM3D_OK = 0
BM3D_COPIED = 1
BM3D_ERR_INVALID = -1
BM3D_ERR_UNSUPPORTED = -2
BM3D_ERR_CUDA = -3
BM3D_ERR_NOMEM = -4
BM3D_ERR_TOO_LARGE = -5
MEM_HOST = 0
MEM_DEVICE = 1
GROUP_STRIDE = 32  # members per reference block in bm3d_debug_groups' arrays

EXPORTS = [
    "bm3d_stage_params_default", "bm3d_stage_params_thmse_default", "bm3d_ctx_create",
    "bm3d_ctx_destroy", "bm3d_last_error", "bm3d_stage", "bm3d_stage3", "bm3d_full",
    "bm3d_full3", "bm3d_stage_f64", "bm3d_ref_block_count", "bm3d_debug_groups",
    "bm3d_last_stats", "bm3d_check", "bm3d_batch_check", "bm3d_set_tiling", "bm3d_set_kernel_timing", "bm3d_kernel_time",
    "bm3d_stage_noalloc", "bm3d_noalloc_check", "bm3d_batch_create", "bm3d_batch_run", "bm3d_batch_tuning",
    "bm3d_batch_destroy", "bm3d_plane_int", "bm3d_stage_int", "bm3d_frame", "bm3d_stage_frame",
    "bm3d_full_many", "bm3d_batch3_create", "bm3d_host_batch_create", "bm3d_host_batch3_create",
    "bm3d_host_batch_run", "bm3d_host_batch_join", "bm3d_host_batch_destroy",
    "bm3d_inject_alloc_failures", "bm3d_batch_stage_times", "bm3d_batch_final_create",
    "bm3d_batch3_final_create",
    "bm3d_pilot_param_count", "bm3d_pilot_set_conv_kernel", "bm3d_pilot_conv_kernel",
    "bm3d_pilot_set_timing", "bm3d_pilot_layer_ms",
    "bm3d_pilot_create", "bm3d_pilot_destroy", "bm3d_pilot_set_params",
    "bm3d_pilot_get_params", "bm3d_pilot_get_grad", "bm3d_pilot_save", "bm3d_pilot_load",
    "bm3d_pilot_estimate", "bm3d_pilot_train_step", "bm3d_pilot_full", "bm3d_pilot_conv48",
    "bm3d_pilot_wgrad48",
]


class BM3DError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"bm3d status {code}: {msg}")
        self.code = code


class StageParams(ctypes.Structure):
    """``bm3d_stage_params``: numeric fields of BM3D_Para_Base (include/BM3D.h:15-45)."""

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
            "block_size": self.block_size, "block_step": self.block_step,
            "group_size": self.group_size, "bm_range": self.bm_range,
            "bm_step": self.bm_step, "thMSE": self.thMSE, "lambda": self.lambda_,
            "sigma": list(self.sigma),
        }

    @classmethod
    def from_dict(cls, d: dict) -> "StageParams":
        p = cls()
        for k in ("block_size", "block_step", "group_size", "bm_range", "bm_step", "thMSE"):
            setattr(p, k, d[k])
        p.lambda_ = d.get("lambda", 0.0)
        for i in range(3):
            p.sigma[i] = d["sigma"][i]
        return p


_lib: Optional[ctypes.CDLL] = None


def load_library(path: str = LIB_PATH) -> ctypes.CDLL:
    """Load the compiled library; raises if it was not built."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(path):
        raise FileNotFoundError(
            f"{path} is missing: build it with `python -m isp_mw_b200.build` (no CPU fallback)")
    lib = ctypes.CDLL(path)
    vp, cp, ip = ctypes.c_void_p, ctypes.c_char_p, ctypes.c_int
    sp = ctypes.POINTER(StageParams)
    lib.bm3d_stage_params_default.argtypes = [cp, ip, ctypes.POINTER(ctypes.c_double), sp]
    lib.bm3d_stage_params_thmse_default.argtypes = [cp, ip, sp]
    lib.bm3d_ctx_create.argtypes = [ctypes.POINTER(vp), ip]
    lib.bm3d_ctx_destroy.argtypes = [vp]
    lib.bm3d_ctx_destroy.restype = None
    lib.bm3d_last_error.argtypes = [vp]
    lib.bm3d_last_error.restype = cp
    plane = [ip, ip, ctypes.c_size_t, ctypes.c_float, ip, vp]
    lib.bm3d_stage.argtypes = [vp, sp, ip, vp, vp, vp] + plane
    lib.bm3d_stage3.argtypes = [vp, sp, ip, vp, vp, vp] + plane
    lib.bm3d_full.argtypes = [vp, sp, sp, vp, vp, vp] + plane
    lib.bm3d_full3.argtypes = [vp, sp, sp, vp, vp, vp] + plane
    lib.bm3d_stage_f64.argtypes = [vp, sp, ip, vp, vp, vp, ip, ip, ctypes.c_size_t,
                                   ctypes.c_double, ip, vp]
    lib.bm3d_ref_block_count.argtypes = [sp, ip, ip]
    lib.bm3d_ref_block_count.restype = ctypes.c_longlong
    lib.bm3d_debug_groups.argtypes = [vp, sp, ip, vp, ip, ip, ctypes.c_size_t, ctypes.c_float,
                                      vp, vp, vp]
    lib.bm3d_last_stats.argtypes = [vp, ctypes.POINTER(ctypes.c_ulonglong)]
    lib.bm3d_check.argtypes = [vp]
    lib.bm3d_batch_check.argtypes = [vp, vp]
    lib.bm3d_set_tiling.argtypes = [vp, ip, ip, ip]
    lib.bm3d_stage_noalloc.argtypes = [sp, ip, vp, vp, vp, ip, ip, ctypes.c_size_t,
                                       ctypes.c_float, vp]
    lib.bm3d_noalloc_check.argtypes = [vp]
    lib.bm3d_inject_alloc_failures.argtypes = [ip]
    lib.bm3d_pilot_param_count.argtypes = []
    lib.bm3d_pilot_set_conv_kernel.argtypes = [ip]
    lib.bm3d_pilot_conv_kernel.argtypes = []
    lib.bm3d_pilot_set_timing.argtypes = [vp, ip]
    lib.bm3d_pilot_layer_ms.argtypes = [vp, vp]
    lib.bm3d_pilot_create.argtypes = [vp, ctypes.c_ulonglong, ctypes.POINTER(vp)]
    lib.bm3d_pilot_destroy.argtypes = [vp]
    lib.bm3d_pilot_destroy.restype = None
    lib.bm3d_pilot_set_params.argtypes = [vp, vp, ip]
    lib.bm3d_pilot_get_params.argtypes = [vp, vp, ip]
    lib.bm3d_pilot_get_grad.argtypes = [vp, vp, ip]
    lib.bm3d_pilot_save.argtypes = [vp, cp]
    lib.bm3d_pilot_load.argtypes = [vp, cp]
    lib.bm3d_pilot_estimate.argtypes = [vp, vp, vp, ip, ip, ip, ctypes.c_size_t, ctypes.c_size_t,
                                        vp, ip, vp]
    lib.bm3d_pilot_train_step.argtypes = [vp, ip, ip, ip, vp, vp, vp, ctypes.c_float,
                                          ctypes.POINTER(ctypes.c_double), vp]
    lib.bm3d_pilot_full.argtypes = [vp, vp, sp, vp, vp, ip, ip, ctypes.c_size_t, ctypes.c_float,
                                    ip, vp]
    lib.bm3d_pilot_conv48.argtypes = [vp, ip, ip, ip, vp, vp, vp, vp, ip, vp, vp]
    lib.bm3d_pilot_wgrad48.argtypes = [vp, ip, ip, ip, vp, vp, vp, vp, vp]
    lib.bm3d_batch_create.argtypes = [vp, ip, vp, vp, vp, vp, vp, vp, vp, ip,
                                      ctypes.POINTER(vp)]
    lib.bm3d_batch3_create.argtypes = [vp, ip, vp, vp, vp, vp, vp, vp, vp, ip,
                                       ctypes.POINTER(vp)]
    lib.bm3d_host_batch_create.argtypes = [vp, ip, vp, vp, vp, vp, ip, ctypes.POINTER(vp)]
    lib.bm3d_host_batch3_create.argtypes = [vp, ip, vp, vp, vp, vp, ip, ctypes.POINTER(vp)]
    lib.bm3d_host_batch_run.argtypes = [vp, vp, vp, vp, ip, vp]
    lib.bm3d_host_batch_join.argtypes = [vp, vp]
    lib.bm3d_host_batch_destroy.argtypes = [vp]
    lib.bm3d_host_batch_destroy.restype = None
    lib.bm3d_batch_run.argtypes = [vp, vp]
    lib.bm3d_batch_tuning.argtypes = [vp, ctypes.POINTER(ctypes.c_int)]
    lib.bm3d_batch_stage_times.argtypes = [vp, vp, ctypes.POINTER(ctypes.c_float)]
    lib.bm3d_batch_final_create.argtypes = [vp, ip, vp, vp, vp, vp, vp, vp, vp, ip,
                                            ctypes.POINTER(vp)]
    lib.bm3d_batch3_final_create.argtypes = [vp, ip, vp, vp, vp, vp, vp, vp, vp, ip,
                                             ctypes.POINTER(vp)]
    lib.bm3d_batch_destroy.argtypes = [vp]
    lib.bm3d_batch_destroy.restype = None
    quant = [ip, ip, ctypes.c_size_t, ip, ip, ip, ip, vp]   # w, h, stride, floor, neutral, ceil, mem, stream
    lib.bm3d_plane_int.argtypes = [vp, sp, sp, vp, vp, vp] + quant
    lib.bm3d_stage_int.argtypes = [vp, sp, ip, vp, vp, vp] + quant
    rgb = [ip, ip, ctypes.c_size_t, ip, ip, ip, vp]         # w, h, stride, floor, ceil, mem, stream
    lib.bm3d_frame.argtypes = [vp, sp, sp, vp, vp, vp] + rgb
    lib.bm3d_stage_frame.argtypes = [vp, sp, ip, vp, vp, vp] + rgb
    lib.bm3d_full_many.argtypes = [vp, ip, vp, vp, vp, vp, vp, vp, vp, ctypes.c_float, ip, vp]
    lib.bm3d_set_kernel_timing.argtypes = [vp, ip]
    lib.bm3d_kernel_time.argtypes = [vp, ip, ctypes.POINTER(ctypes.c_double),
                                     ctypes.POINTER(ctypes.c_longlong)]
    _lib = lib
    return lib


def stage_params_default(profile: str = "fast", wiener: bool = False,
                         sigma: Sequence[float] = (10.0, 10.0, 10.0)) -> StageParams:
    """Profile defaults with sigma applied and thMSE_Default() re-run."""
    lib = load_library()
    p = StageParams()
    s = (ctypes.c_double * 3)(*sigma)
    rc = lib.bm3d_stage_params_default(profile.encode(), int(wiener), s, ctypes.byref(p))
    if rc != BM3D_OK:
        raise ValueError(f"unrecognized profile {profile!r}")
    return p


def _is_torch(x) -> bool:
    return type(x).__module__.startswith("torch")


def _plane_info(x):
    """(pointer, mem kind, width, height, stride, dtype name) of a plane."""
    if _is_torch(x):
        if x.dim() != 2 or x.stride(1) != 1:
            raise ValueError("planes must be 2-D with unit column stride")
        mem = MEM_DEVICE if x.is_cuda else MEM_HOST
        return x.data_ptr(), mem, x.shape[1], x.shape[0], x.stride(0), str(x.dtype).split(".")[-1]
    a = x
    if not isinstance(a, np.ndarray) or a.ndim != 2 or a.strides[1] != a.itemsize:
        raise ValueError("planes must be 2-D numpy arrays with unit column stride")
    return a.ctypes.data, MEM_HOST, a.shape[1], a.shape[0], a.strides[0] // a.itemsize, a.dtype.name


def _stream_of(x) -> int:
    if _is_torch(x) and x.is_cuda:
        import torch
        return torch.cuda.current_stream(x.device).cuda_stream
    return 0


class Context:
    """A ``bm3d_ctx`` on one CUDA device."""

    def __init__(self, device: int = 0):
        self.lib = load_library()
        h = ctypes.c_void_p()
        rc = self.lib.bm3d_ctx_create(ctypes.byref(h), int(device))
        if rc != BM3D_OK:
            raise BM3DError(rc, self.lib.bm3d_last_error(None).decode())
        self.h = h
        self.device = device

    def close(self):
        if getattr(self, "h", None):
            self.lib.bm3d_ctx_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _check(self, rc: int, allow_copied: bool = True) -> int:
        if rc == BM3D_OK or (allow_copied and rc == BM3D_COPIED):
            return rc
        raise BM3DError(rc, self.lib.bm3d_last_error(self.h).decode())

    def set_tiling(self, tile_x: int = 0, tile_y: int = 0, warps: int = 0):
        self._check(self.lib.bm3d_set_tiling(self.h, tile_x, tile_y, warps))

    def stage(self, params: StageParams, wiener: bool, dst, src, ref=None,
              value_range: float = 1.0) -> int:
        """One stage on one plane (``bm3d_stage`` / ``bm3d_stage_f64``)."""
        ref = src if ref is None else ref
        dp, mem, w, h, stride, dt = _plane_info(dst)
        spp, mem_s, *_ = _plane_info(src)
        rp, mem_r, *_ = _plane_info(ref)
        if not (mem == mem_s == mem_r):
            raise ValueError("dst, src and ref must live in the same memory")
        stream = _stream_of(dst)
        if dt == "float64":
            rc = self.lib.bm3d_stage_f64(self.h, ctypes.byref(params), int(wiener), dp, spp, rp,
                                         w, h, stride, ctypes.c_double(value_range), mem, stream)
        else:
            rc = self.lib.bm3d_stage(self.h, ctypes.byref(params), int(wiener), dp, spp, rp, w,
                                     h, stride, value_range, mem, stream)
        return self._check(rc)

    def stage3(self, params: StageParams, wiener: bool, dst, src, ref=None,
               value_range: float = 1.0) -> int:
        ref = src if ref is None else ref
        infos = [_plane_info(x) for x in list(dst) + list(src) + list(ref)]
        w, h, stride, mem = infos[0][2], infos[0][3], infos[0][4], infos[0][1]
        arr = ctypes.c_void_p * 3
        rc = self.lib.bm3d_stage3(self.h, ctypes.byref(params), int(wiener),
                                  arr(*[i[0] for i in infos[0:3]]),
                                  arr(*[i[0] for i in infos[3:6]]),
                                  arr(*[i[0] for i in infos[6:9]]), w, h, stride, value_range,
                                  mem, _stream_of(dst[0]))
        return self._check(rc)

    def full(self, basic: StageParams, final: StageParams, dst, src,
             value_range: float = 1.0, ref=None) -> int:
        """Basic (matching on ref, default src) then final (``bm3d_full``)."""
        dp, mem, w, h, stride, _ = _plane_info(dst)
        spp, *_ = _plane_info(src)
        rp = None if ref is None else _plane_info(ref)[0]
        rc = self.lib.bm3d_full(self.h, ctypes.byref(basic), ctypes.byref(final), dp, spp, rp, w,
                                h, stride, value_range, mem, _stream_of(dst))
        return self._check(rc)

    def full3(self, basic: StageParams, final: StageParams, dst, src,
              value_range: float = 1.0, ref=None) -> int:
        planes = list(dst) + list(src) + ([] if ref is None else list(ref))
        infos = [_plane_info(x) for x in planes]
        w, h, stride, mem = infos[0][2], infos[0][3], infos[0][4], infos[0][1]
        arr = ctypes.c_void_p * 3
        rc = self.lib.bm3d_full3(self.h, ctypes.byref(basic), ctypes.byref(final),
                                 arr(*[i[0] for i in infos[0:3]]),
                                 arr(*[i[0] for i in infos[3:6]]),
                                 None if ref is None else arr(*[i[0] for i in infos[6:9]]), w, h,
                                 stride, value_range, mem, _stream_of(dst[0]))
        return self._check(rc)

    # -- integer planes and RGB frames (int32 numpy arrays or CUDA tensors) --

    @staticmethod
    def _int_planes(planes):
        infos = [_plane_info(x) for x in planes]
        if any(i[5] != "int32" for i in infos):
            raise ValueError("integer paths take int32 planes")
        w, h, stride, mem = infos[0][2], infos[0][3], infos[0][4], infos[0][1]
        if any(i[1:5] != (mem, w, h, stride) for i in infos):
            raise ValueError("planes must share memory kind, size and stride")
        return [i[0] for i in infos], w, h, stride, mem

    def plane_int(self, basic: StageParams, final: StageParams, dst, src, quant,
                  ref=None) -> int:
        """Basic then final on an int32 plane quantised as quant = (floor, neutral, ceil)."""
        ptrs, w, h, stride, mem = self._int_planes([dst, src] + ([] if ref is None else [ref]))
        lo, mid, hi = (int(v) for v in quant)
        rc = self.lib.bm3d_plane_int(self.h, ctypes.byref(basic), ctypes.byref(final), ptrs[0],
                                     ptrs[1], ptrs[2] if ref is not None else None, w, h, stride,
                                     lo, mid, hi, mem, _stream_of(dst))
        return self._check(rc)

    def stage_int(self, params: StageParams, wiener: bool, dst, src, ref=None,
                  quant=(0, 0, 255)) -> int:
        """One stage on an int32 plane (ref None = src)."""
        planes = [dst, src] + ([] if ref is None else [ref])
        ptrs, w, h, stride, mem = self._int_planes(planes)
        lo, mid, hi = (int(v) for v in quant)
        rc = self.lib.bm3d_stage_int(self.h, ctypes.byref(params), int(wiener), ptrs[0], ptrs[1],
                                     ptrs[2] if ref is not None else None, w, h, stride, lo, mid,
                                     hi, mem, _stream_of(dst))
        return self._check(rc)

    def frame(self, basic: StageParams, final: StageParams, dst, src, floor: int = 0,
              ceil: int = 255, ref=None) -> int:
        """Basic then final on an RGB frame of three int32 planes (R, G, B)."""
        planes = list(dst) + list(src) + ([] if ref is None else list(ref))
        ptrs, w, h, stride, mem = self._int_planes(planes)
        arr = ctypes.c_void_p * 3
        rc = self.lib.bm3d_frame(self.h, ctypes.byref(basic), ctypes.byref(final),
                                 arr(*ptrs[0:3]), arr(*ptrs[3:6]),
                                 arr(*ptrs[6:9]) if ref is not None else None, w, h, stride,
                                 int(floor), int(ceil), mem, _stream_of(dst[0]))
        return self._check(rc)

    def stage_frame(self, params: StageParams, wiener: bool, dst, src, ref=None, floor: int = 0,
                    ceil: int = 255) -> int:
        """One stage on an RGB frame (ref None = src)."""
        planes = list(dst) + list(src) + ([] if ref is None else list(ref))
        ptrs, w, h, stride, mem = self._int_planes(planes)
        arr = ctypes.c_void_p * 3
        rc = self.lib.bm3d_stage_frame(self.h, ctypes.byref(params), int(wiener), arr(*ptrs[0:3]),
                                       arr(*ptrs[3:6]),
                                       arr(*ptrs[6:9]) if ref is not None else None, w, h, stride,
                                       int(floor), int(ceil), mem, _stream_of(dst[0]))
        return self._check(rc)

    def full_many(self, basic: Sequence[StageParams], final: Sequence[StageParams], dst, src,
                  value_range: float = 1.0, asynchronous: bool = False,
                  stream: Optional[int] = None) -> int:
        """``bm3d_full_many``: basic then final on host planes (numpy arrays or
        CPU tensors; page-locked for overlap), copies overlapped with the
        filtering. With ``asynchronous`` the call returns once enqueued on
        ``stream`` (default: the current torch stream); synchronise it before
        reading ``dst``."""
        n = len(src)
        if not (len(basic) == len(final) == len(dst) == n):
            raise ValueError("one basic/final parameter set and dst per src plane")
        di = [_plane_info(x) for x in dst]
        si = [_plane_info(x) for x in src]
        if any(i[1] != MEM_HOST for i in di + si):
            raise ValueError("full_many takes host planes")
        for a, b in zip(di, si):
            if a[2:5] != b[2:5]:
                raise ValueError("dst and src planes must have the same size and stride")
        if stream is None:
            try:
                import torch
                stream = torch.cuda.current_stream(self.device).cuda_stream
            except Exception:
                stream = 0
        vp = ctypes.c_void_p * max(1, n)
        pb = (StageParams * max(1, n))(*basic)
        pf = (StageParams * max(1, n))(*final)
        w = (ctypes.c_int * max(1, n))(*[i[2] for i in si])
        h = (ctypes.c_int * max(1, n))(*[i[3] for i in si])
        st = (ctypes.c_size_t * max(1, n))(*[i[4] for i in si])
        rc = self.lib.bm3d_full_many(self.h, n, pb, pf, vp(*[i[0] for i in di]),
                                     vp(*[i[0] for i in si]), w, h, st, value_range,
                                     int(asynchronous), stream)
        return self._check(rc)

    def ref_block_count(self, params: StageParams, width: int, height: int) -> int:
        return int(self.lib.bm3d_ref_block_count(ctypes.byref(params), width, height))

    def debug_groups(self, params: StageParams, wiener: bool, ref: np.ndarray,
                     value_range: float = 1.0):
        """Group of every reference block: (counts[R], pos[R, 32, 2] (y, x), keys[R, 32])."""
        ref = np.ascontiguousarray(ref, dtype=np.float32)
        h, w = ref.shape
        n = self.ref_block_count(params, w, h)
        counts = np.zeros(n, np.int32)
        pos = np.full((n, GROUP_STRIDE, 2), -1, np.int32)
        keys = np.zeros((n, GROUP_STRIDE), np.float32)
        rc = self.lib.bm3d_debug_groups(self.h, ctypes.byref(params), int(wiener),
                                        ref.ctypes.data, w, h, w, value_range,
                                        counts.ctypes.data, pos.ctypes.data, keys.ctypes.data)
        self._check(rc, allow_copied=False)
        return counts, pos, keys

    def set_kernel_timing(self, on: bool):
        self._check(self.lib.bm3d_set_kernel_timing(self.h, int(on)))

    def kernel_time(self, wiener: bool):
        """(total ms, launches) of the basic / final stage kernel since timing began."""
        ms, n = ctypes.c_double(), ctypes.c_longlong()
        self._check(self.lib.bm3d_kernel_time(self.h, int(wiener), ctypes.byref(ms),
                                              ctypes.byref(n)))
        return ms.value, n.value

    def last_stats(self):
        out = (ctypes.c_ulonglong * 4)()
        self._check(self.lib.bm3d_last_stats(self.h, out))
        return [int(v) for v in out]

    def check(self):
        """``bm3d_check``: wait for the context's work and raise if the kernels'
        consistency counter moved (device-memory calls do not check it)."""
        self._check(self.lib.bm3d_check(self.h), allow_copied=False)


class Batch:
    """``bm3d_batch``: basic + final over many device planes (CUDA torch
    tensors) of any sizes and noise levels, one persistent launch per stage,
    replayed from a CUDA graph. The planes are bound at creation. When every
    element of ``src`` / ``dst`` is a triple of planes (Y, U, V), the images
    are filtered as three planes sharing luma groups (``bm3d_batch3_create``)."""

    def __init__(self, ctx: "Context", basic: Sequence[StageParams], final: Sequence[StageParams],
                 dst: Sequence, src: Sequence, autotune: bool = True, ref: Optional[Sequence] = None):
        """With `ref` (planes shaped like src), the batch runs the final stage
        only, with those planes in place of the basic estimates
        (``bm3d_batch_final_create``); `basic` is then ignored."""
        n = len(src)
        if not (len(basic) == len(final) == len(dst) == n) or n == 0:
            raise ValueError("one basic/final parameter set and dst per src image")
        self.ctx = ctx
        three = all(isinstance(x, (list, tuple)) for x in src)
        if three:
            if not all(isinstance(x, (list, tuple)) and len(x) == 3 for x in list(src) + list(dst)):
                raise ValueError("three-plane images take three src and three dst planes each")
            src = [p for x in src for p in x]
            dst = [p for x in dst for p in x]
            for i in range(n):
                shapes = {tuple(p.shape) for p in src[3 * i:3 * i + 3] + dst[3 * i:3 * i + 3]}
                if len(shapes) != 1:
                    raise ValueError("the planes of an image must have one size")
        npl = 3 if three else 1
        if ref is not None and three:
            ref = [p for x in ref for p in x]
        self._keep = (list(dst), list(src), None if ref is None else list(ref))
        infos_d = [_plane_info(d) for d in dst]
        infos_s = [_plane_info(x) for x in src]
        if any(i[1] != MEM_DEVICE for i in infos_d + infos_s):
            raise ValueError("batches take device (CUDA) planes")
        for a, b in zip(infos_d, infos_s):
            if a[2:5] != b[2:5]:
                raise ValueError("dst and src planes must have the same size and pitch")
        if npl == 3 and any(infos_s[3 * i][4] != infos_s[3 * i + c][4]
                            for i in range(n) for c in range(3)):
            raise ValueError("the planes of an image must share one row pitch")
        pb = (StageParams * n)(*basic)
        pf = (StageParams * n)(*final)
        vp = ctypes.c_void_p * (n * npl)
        first = infos_s[::npl]
        w = (ctypes.c_int * n)(*[i[2] for i in first])
        h = (ctypes.c_int * n)(*[i[3] for i in first])
        st = (ctypes.c_size_t * n)(*[i[4] for i in first])
        self.h = ctypes.c_void_p()
        if ref is None:
            create = ctx.lib.bm3d_batch3_create if npl == 3 else ctx.lib.bm3d_batch_create
            rc = create(ctx.h, n, pb, pf, vp(*[i[0] for i in infos_d]),
                        vp(*[i[0] for i in infos_s]), w, h, st, int(autotune),
                        ctypes.byref(self.h))
        else:
            infos_r = [_plane_info(x) for x in ref]
            if any(a[1:5] != b[1:5] for a, b in zip(infos_r, infos_s)):
                raise ValueError("ref planes must match src in memory, size and pitch")
            create = (ctx.lib.bm3d_batch3_final_create if npl == 3
                      else ctx.lib.bm3d_batch_final_create)
            rc = create(ctx.h, n, pf, vp(*[i[0] for i in infos_d]), vp(*[i[0] for i in infos_s]),
                        vp(*[i[0] for i in infos_r]), w, h, st, int(autotune),
                        ctypes.byref(self.h))
        ctx._check(rc, allow_copied=False)
        self.pixels = sum(i[2] * i[3] for i in first)  # image pixels (per plane for 3-plane images)

    def run(self, stream: Optional[int] = None):
        if stream is None:
            import torch
            stream = torch.cuda.current_stream().cuda_stream
        self.ctx._check(self.ctx.lib.bm3d_batch_run(self.h, stream))

    def check(self, stream: Optional[int] = None):
        """``bm3d_batch_check``: wait for ``stream`` and raise if the batch
        kernels' consistency counter moved."""
        if stream is None:
            import torch
            stream = torch.cuda.current_stream().cuda_stream
        self.ctx._check(self.ctx.lib.bm3d_batch_check(self.h, stream), allow_copied=False)

    def stage_times(self, stream: Optional[int] = None):
        """Device ms of the basic and final persistent stage launches, from one
        eager run of the pipeline (``bm3d_batch_stage_times``)."""
        if stream is None:
            import torch
            stream = torch.cuda.current_stream().cuda_stream
        out = (ctypes.c_float * 2)()
        self.ctx._check(self.ctx.lib.bm3d_batch_stage_times(self.h, stream, out))
        return float(out[0]), float(out[1])

    def tuning(self):
        out = (ctypes.c_int * 6)()
        self.ctx._check(self.ctx.lib.bm3d_batch_tuning(self.h, out))
        return {"basic": tuple(out[0:3]), "final": tuple(out[3:6])}

    def close(self):
        if getattr(self, "h", None):
            self.ctx.lib.bm3d_batch_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class HostBatch:
    """``bm3d_host_batch``: a batch fed from host planes (numpy arrays or CPU
    tensors; page-locked for overlap). Sizes and parameters are fixed at
    creation; each ``run`` uploads ``src``, filters and downloads into ``dst``.
    With ``asynchronous`` the call returns once enqueued on ``stream``
    (default: the current torch stream), and consecutive runs overlap their
    copies with one another's filtering; synchronise before reading ``dst``.
    With ``planes=3`` every image is three planes (Y, U, V) sharing luma
    groups (``bm3d_host_batch3_create``), and ``run`` takes a triple of
    planes per image."""

    def __init__(self, ctx: "Context", basic: Sequence[StageParams], final: Sequence[StageParams],
                 shapes: Sequence, autotune: bool = True, planes: int = 1):
        n = len(shapes)
        if not (len(basic) == len(final) == n) or n == 0:
            raise ValueError("one basic/final parameter set per image")
        if planes not in (1, 3):
            raise ValueError("planes must be 1 or 3")
        self.ctx = ctx
        self.npl = planes
        self.shapes = [(int(h), int(w)) for h, w in shapes]
        pb = (StageParams * n)(*basic)
        pf = (StageParams * n)(*final)
        w = (ctypes.c_int * n)(*[s[1] for s in self.shapes])
        h = (ctypes.c_int * n)(*[s[0] for s in self.shapes])
        self.h = ctypes.c_void_p()
        create = ctx.lib.bm3d_host_batch3_create if planes == 3 else ctx.lib.bm3d_host_batch_create
        rc = create(ctx.h, n, pb, pf, w, h, int(autotune), ctypes.byref(self.h))
        ctx._check(rc, allow_copied=False)
        self.pixels = sum(a * b for a, b in self.shapes)  # image pixels

    def run(self, dst, src, asynchronous=False, stream: Optional[int] = None):
        """asynchronous: False (dst written on return), True (enqueued; the
        stream completes after this run's download) or "overlap" (enqueued,
        no wait tied to the stream: call join() before synchronising)."""
        n, npl = len(self.shapes), self.npl
        if len(dst) != n or len(src) != n:
            raise ValueError("one dst and src image per batch image")
        if npl == 3:
            if not all(isinstance(x, (list, tuple)) and len(x) == 3 for x in list(dst) + list(src)):
                raise ValueError("three-plane batches take three planes per image")
            dst = [p for x in dst for p in x]
            src = [p for x in src for p in x]
        di = [_plane_info(x) for x in dst]
        si = [_plane_info(x) for x in src]
        for j, (a, b) in enumerate(zip(di, si)):
            if a[1] != MEM_HOST or b[1] != MEM_HOST:
                raise ValueError("host batches take host planes")
            k = j // npl
            if ((a[3], a[2]) != self.shapes[k] or (b[3], b[2]) != self.shapes[k] or a[4] != b[4]
                    or b[4] != si[k * npl][4]):
                raise ValueError("plane size or stride does not match the batch")
        if stream is None:
            try:
                import torch
                stream = torch.cuda.current_stream(self.ctx.device).cuda_stream
            except Exception:
                stream = 0
        vp = ctypes.c_void_p * (n * npl)
        st = (ctypes.c_size_t * n)(*[i[4] for i in si[::npl]])
        mode = 2 if asynchronous == "overlap" else int(bool(asynchronous))
        rc = self.ctx.lib.bm3d_host_batch_run(self.h, vp(*[i[0] for i in di]),
                                              vp(*[i[0] for i in si]), st, mode, stream)
        self.ctx._check(rc, allow_copied=False)

    def join(self, stream: Optional[int] = None):
        """Make ``stream`` wait for every download issued so far."""
        if stream is None:
            import torch
            stream = torch.cuda.current_stream(self.ctx.device).cuda_stream
        self.ctx._check(self.ctx.lib.bm3d_host_batch_join(self.h, stream), allow_copied=False)

    def close(self):
        if getattr(self, "h", None):
            self.ctx.lib.bm3d_host_batch_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


# ---------------------------------------------------------------------------
# Mirror of the reference's parameter and filter classes (include/BM3D.h).

class BM3D_Para_Base:
    """Fields of BM3D_Para_Base (include/BM3D.h:15-45)."""

    wiener = False

    def __init__(self, profile: str = "fast"):
        self.profile = profile
        p = stage_params_default(profile, self.wiener, (10.0, 10.0, 10.0))
        self.sigma = [10.0, 10.0, 10.0]
        self.BlockSize = p.block_size
        self.BlockStep = p.block_step
        self.GroupSize = p.group_size
        self.BMrange = p.bm_range
        self.BMstep = p.bm_step
        self.thMSE = p.thMSE
        self.lambda_ = p.lambda_

    def thMSE_Default(self):
        p = self.to_c()
        load_library().bm3d_stage_params_thmse_default(self.profile.encode(), int(self.wiener),
                                                       ctypes.byref(p))
        self.thMSE = p.thMSE

    def to_c(self) -> StageParams:
        return StageParams.from_dict({
            "block_size": self.BlockSize, "block_step": self.BlockStep,
            "group_size": self.GroupSize, "bm_range": self.BMrange, "bm_step": self.BMstep,
            "thMSE": self.thMSE, "lambda": self.lambda_, "sigma": self.sigma})


class BM3D_Basic_Para(BM3D_Para_Base):
    """include/BM3D.h:48-98."""
    wiener = False


class BM3D_Final_Para(BM3D_Para_Base):
    """include/BM3D.h:101-151."""
    wiener = True


class BM3D_Para:
    """include/BM3D.h:154-168."""

    def __init__(self, profile: str = "fast"):
        self.basic = BM3D_Basic_Para(profile)
        self.final = BM3D_Final_Para(profile)

    def thMSE_Default(self):
        self.basic.thMSE_Default()
        self.final.thMSE_Default()


_default_ctx: Optional[Context] = None


def default_context() -> Context:
    global _default_ctx
    if _default_ctx is None:
        _default_ctx = Context(0)
    return _default_ctx


def _empty_like(x):
    if _is_torch(x):
        import torch
        return torch.empty_like(x)
    return np.empty_like(x)


class _Stage:
    wiener = False

    def __init__(self, para: Optional[BM3D_Para_Base] = None, ctx: Optional[Context] = None):
        self.para = para if para is not None else (
            BM3D_Final_Para() if self.wiener else BM3D_Basic_Para())
        self.ctx = ctx

    def process(self, dst, src, ref=None, value_range: float = 1.0):
        """FilterIF2::process(dst, src[, ref]) (include/Filter.h:174-199)."""
        ctx = self.ctx or default_context()
        if isinstance(src, (list, tuple)):
            ctx.stage3(self.para.to_c(), self.wiener, dst, src, ref, value_range)
        else:
            ctx.stage(self.para.to_c(), self.wiener, dst, src, ref, value_range)
        return dst

    def __call__(self, src, ref=None, value_range: float = 1.0):
        """FilterIF2::operator()(src[, ref]) (include/Filter.h:189-216)."""
        if isinstance(src, (list, tuple)):
            dst = [s.copy() if isinstance(s, np.ndarray) else s.clone() for s in src]
        else:
            dst = _empty_like(src)
        return self.process(dst, src, ref, value_range)


class BM3D_Basic(_Stage):
    """include/BM3D.h:287-309: the hard-threshold basic estimate."""
    wiener = False


class BM3D_Final(_Stage):
    """include/BM3D.h:312-334: the Wiener final estimate (ref = basic estimate)."""
    wiener = True


class BM3D:
    """include/BM3D.h:337-357: basic then final."""

    def __init__(self, para: Optional[BM3D_Para] = None, ctx: Optional[Context] = None):
        self.para = para if para is not None else BM3D_Para()
        self.ctx = ctx

    def process(self, dst, src, ref=None, value_range: float = 1.0):
        """FilterIF2::process(dst, src[, ref]): the basic stage matches on ref."""
        ctx = self.ctx or default_context()
        if isinstance(src, (list, tuple)):
            ctx.full3(self.para.basic.to_c(), self.para.final.to_c(), dst, src, value_range, ref)
        else:
            ctx.full(self.para.basic.to_c(), self.para.final.to_c(), dst, src, value_range, ref)
        return dst

    def __call__(self, src, ref=None, value_range: float = 1.0):
        if isinstance(src, (list, tuple)):
            dst = [s.copy() if isinstance(s, np.ndarray) else s.clone() for s in src]
        else:
            dst = _empty_like(src)
        return self.process(dst, src, ref, value_range)


class Pilot:
    """``bm3d_pilot``: the learned pilot (8 layers of 3 x 3 convolutions, 48
    channels, BF16 with FP32 accumulation on the tensor cores) that stands in
    for the basic estimate feeding the final (Wiener) stage. Training data and
    the loop live in ``isp_mw_b200.pilot``."""

    def __init__(self, ctx: "Context", seed: int = 0):
        self.ctx = ctx
        self.lib = ctx.lib
        self.h = ctypes.c_void_p()
        ctx._check(self.lib.bm3d_pilot_create(ctx.h, int(seed), ctypes.byref(self.h)),
                   allow_copied=False)
        self.count = int(self.lib.bm3d_pilot_param_count())

    def close(self):
        if getattr(self, "h", None):
            self.lib.bm3d_pilot_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def params(self) -> np.ndarray:
        out = np.empty(self.count, np.float32)
        self.ctx._check(self.lib.bm3d_pilot_get_params(self.h, out.ctypes.data, self.count))
        return out

    def grad(self) -> np.ndarray:
        out = np.empty(self.count, np.float32)
        self.ctx._check(self.lib.bm3d_pilot_get_grad(self.h, out.ctypes.data, self.count))
        return out

    def set_timing(self, on: bool):
        """Record CUDA events around each layer of later forward passes."""
        self.ctx._check(self.lib.bm3d_pilot_set_timing(self.h, 1 if on else 0))

    def layer_ms(self) -> np.ndarray:
        """Device ms of the eight layers of the last timed forward pass."""
        out = np.empty(8, np.float32)
        self.ctx._check(self.lib.bm3d_pilot_layer_ms(self.h, out.ctypes.data))
        return out

    def set_params(self, values: np.ndarray):
        v = np.ascontiguousarray(values, dtype=np.float32)
        if v.size != self.count:
            raise ValueError(f"expected {self.count} parameters")
        self.ctx._check(self.lib.bm3d_pilot_set_params(self.h, v.ctypes.data, self.count))

    def save(self, path: str):
        self.ctx._check(self.lib.bm3d_pilot_save(self.h, path.encode()))

    def load(self, path: str):
        self.ctx._check(self.lib.bm3d_pilot_load(self.h, path.encode()))

    def estimate(self, dst, src, sigma):
        """dst = pilot(src): one plane (2-D) or a stack of planes (3-D, numpy
        host arrays or contiguous CUDA tensors); sigma = true noise std (0-1
        scale), one per plane."""
        if _is_torch(src):
            import torch
            if src.dim() == 2:
                src, dst = src.unsqueeze(0), dst.unsqueeze(0)
            n, h, w = src.shape
            if not (src.is_contiguous() and dst.is_contiguous()):
                raise ValueError("pilot planes must be contiguous")
            sig = torch.as_tensor(np.broadcast_to(np.asarray(sigma, np.float32), (n,)).copy(),
                                  device=src.device)
            stream = torch.cuda.current_stream(src.device)
            rc = self.lib.bm3d_pilot_estimate(self.h, dst.data_ptr(), src.data_ptr(), n, w, h, w,
                                              h * w, sig.data_ptr(), MEM_DEVICE, stream.cuda_stream)
            self.ctx._check(rc)
            stream.synchronize()
            return dst
        s3 = np.ascontiguousarray(src, np.float32)
        if s3.ndim == 2:
            s3 = s3[None]
        n, h, w = s3.shape
        out = np.empty_like(s3)
        sig = np.ascontiguousarray(np.broadcast_to(np.asarray(sigma, np.float32), (n,)))
        rc = self.lib.bm3d_pilot_estimate(self.h, out.ctypes.data, s3.ctypes.data, n, w, h, w,
                                          h * w, sig.ctypes.data, MEM_HOST, None)
        self.ctx._check(rc)
        dst[...] = out.reshape(dst.shape)
        return dst

    def train_step(self, noisy, target, sigma, lr: float, want_loss: bool = True):
        """One Adam step on CUDA tensors noisy / target [n, h, w] and sigma [n];
        returns the mean squared error (before the step) when want_loss."""
        import torch
        n, h, w = noisy.shape
        loss = ctypes.c_double(0.0)
        rc = self.lib.bm3d_pilot_train_step(
            self.h, n, h, w, noisy.data_ptr(), target.data_ptr(), sigma.data_ptr(),
            ctypes.c_float(lr), ctypes.byref(loss) if want_loss else None,
            torch.cuda.current_stream(noisy.device).cuda_stream)
        self.ctx._check(rc)
        return loss.value if want_loss else None

    def full(self, final: StageParams, dst, src, value_range: float = 1.0) -> int:
        """Pilot, then the final stage with the pilot's estimate as reference
        (``bm3d_pilot_full``)."""
        dp, mem, w, h, stride, _ = _plane_info(dst)
        spp, *_ = _plane_info(src)
        rc = self.lib.bm3d_pilot_full(self.ctx.h, self.h, ctypes.byref(final), dp, spp, w, h,
                                      stride, value_range, mem, _stream_of(dst))
        return self.ctx._check(rc)
