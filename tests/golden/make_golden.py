"""Generate tests/golden/*.npz from the reference's own BM3D, compiled in
place by oracle/Makefile (oracle/_ref/libbm3d_ref_f32.so).

Each fixture holds its inputs (so it does not depend on the generator's
floating-point behaviour on another machine), the parameters, and the
reference's basic estimate, final estimate and group lists.

    python tests/golden/make_golden.py
"""
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

import oracle  # noqa: E402
from isp_mw_b200 import synth  # noqa: E402


def params(profile, sigma_param):
    s = [sigma_param] * 3 if np.isscalar(sigma_param) else list(sigma_param)
    final = oracle.reference_stage_default(profile, True, s)
    final["lambda"] = 0.0  # never initialised by the reference (include/BM3D.h:101-151), unused
    return oracle.reference_stage_default(profile, False, s), final


def tie_plane(h, w):
    """Sawtooth ramps of exact binary fractions: every candidate at the same
    horizontal offset has exactly the same block distance, so kept groups are
    full of equal keys and std::partial_sort's tie placement decides them."""
    y, x = np.mgrid[0:h, 0:w]
    return (((x % 32) / 64.0) + ((y // 16) % 2) / 8.0).astype(np.float32)


CASES = [
    ("fast_64x64_s25", "fast", 64, 64, 25.0, 11),
    ("fast_97x70_s10", "fast", 70, 97, 10.0, 12),
    ("fast_13x21_s50", "fast", 21, 13, 50.0, 13),
    ("lc_60x44_s15", "lc", 44, 60, 15.0, 14),
    ("fast_ties_48x40", "fast", 40, 48, None, 15),
    ("np_56x72_s20", "np", 56, 72, 20.0, 16),
    ("high_48x40_s30", "high", 40, 48, 30.0, 17),
    ("vn_64x56_s15", "vn", 56, 64, 15.0, 18),
]


# (name, kind, height, width, sigma/255, bit depth, full range, chroma, seed)
INT_CASES = [
    ("int_rgb8_pc_48x56", "frame", 48, 56, 20.0, 8, True, False, 40),
    ("int_rgb10_tv_41x37", "frame", 41, 37, 30.0, 10, False, False, 41),
    ("int_y8_tv_44x60", "plane", 44, 60, 15.0, 8, False, False, 42),
    ("int_c8_pc_40x52", "plane", 40, 52, 25.0, 8, True, True, 43),
    ("int_y16_pc_36x40", "plane", 36, 40, 10.0, 16, True, False, 44),
]


def main():
    oracle.build(reference=True)
    ref = oracle.backend("reference", np.float32)
    for name, profile, h, w, s255, seed in CASES:
        if s255 is None:
            noisy = tie_plane(h, w)
            clean = noisy.copy()
            sp = synth.sigma_param(20.0)
        else:
            clean, noisy = synth.pair(h, w, s255, seed)
            sp = synth.sigma_param(s255)
        b, f = params(profile, sp)
        basic, final = ref.full(b, f, noisy)
        gb = ref.groups(False, b, noisy)
        gf = ref.groups(True, f, basic)
        np.savez_compressed(
            os.path.join(HERE, name + ".npz"), noisy=noisy, basic=basic, final=final,
            basic_counts=gb[0], basic_pos=gb[1], basic_keys=gb[2],
            final_counts=gf[0], final_pos=gf[1], final_keys=gf[2],
            params=json.dumps({"basic": b, "final": f, "profile": profile}))
        print(name, noisy.shape)
    # three planes sharing luma groups
    h, w = 40, 52
    planes = [synth.pair(h, w, s, 30 + i)[1] for i, s in enumerate((15.0, 10.0, 10.0))]
    sp = [synth.sigma_param(15.0, 0), synth.sigma_param(10.0, 1), synth.sigma_param(10.0, 2)]
    b, f = params("fast", sp)
    basic = ref.stage3(False, b, planes)
    final = ref.stage3(True, f, planes, basic)
    np.savez_compressed(os.path.join(HERE, "fast3_52x40.npz"), noisy=np.stack(planes),
                        basic=np.stack(basic), final=np.stack(final),
                        params=json.dumps({"basic": b, "final": f, "profile": "fast"}))
    print("fast3_52x40")
    # integer planes and RGB frames (int32, the reference's Plane / Frame)
    for name, kind, h, w, s255, bits, pc, chroma, seed in INT_CASES:
        b, f = params("fast", synth.sigma_param(s255))
        if kind == "frame":
            lo, hi = oracle.frame_range(bits, pc)
            src = synth.int_planes(h, w, s255, seed, lo, hi, 3)
            full = ref.frame(b, f, src, bits, pc)
            basic = ref.stage_frame(False, b, src, None, bits, pc)
            final = ref.stage_frame(True, f, src, basic, bits, pc)
            quant = (lo, lo, hi)
        else:
            quant = oracle.plane_quant(bits, pc, chroma)
            src = synth.int_planes(h, w, s255, seed, quant[0], quant[2], 1)
            full = [ref.plane_int(b, f, src[0], quant, bits)]
            basic = [ref.stage_int(False, b, src[0], None, quant, bits)]
            final = [ref.stage_int(True, f, src[0], basic[0], quant, bits)]
        np.savez_compressed(
            os.path.join(HERE, name + ".npz"), src=np.stack(src), full=np.stack(full),
            basic=np.stack(basic), final=np.stack(final), quant=np.array(quant, np.int32),
            params=json.dumps({"basic": b, "final": f, "profile": "fast", "kind": kind,
                               "bits": bits, "pc": pc}))
        print(name, (h, w))


if __name__ == "__main__":
    main()
