"""Shared by the parity tests: why a chained basic -> final result may
differ from the reference's chain by more than the strict bar, checked rather
than assumed.

The final stage matches blocks on the basic estimate (BM3D_Final,
source/BM3D.cpp:411-457, matching through include/Block.h:578-703). Two basic
estimates that differ only in float rounding give slightly different block
distances, so a candidate whose key nearly ties another (or sits at the
threshold) can change places, and the changed group moves the pixels of its
members' blocks. explain_chain_divergence checks that this, and nothing else,
is what happened: every pixel over the bar lies in a member block of a group
that differs between the two chains, and every such difference is a near-tie.
"""
import numpy as np

MAX_ABS = 1e-3
# relative key gap of a flip that counts as a near-tie
NEAR_TIE = 1e-3


def explain_chain_divergence(d, gpu_groups, ref_groups, f):
    """(pixels over MAX_ABS not explained by a near-tie group flip, worst
    relative key gap of a flip, number of flipped groups)."""
    gc, gp, gk = gpu_groups
    rc, rp, rk = ref_groups
    bs = f.block_size
    th = f.thMSE / np.sqrt(3.0)  # the matching threshold in key units (thMSE * normY)
    mask = np.zeros(d.shape, bool)
    worst, flips = 0.0, 0
    for r in range(len(rc)):
        n1, n2 = int(gc[r]), int(rc[r])
        if n1 == n2 and np.array_equal(gp[r, :n1], rp[r, :n2]):
            continue
        flips += 1
        m = min(n1, n2)
        k1 = gk[r, :m].astype(np.float64)
        k2 = rk[r, :m].astype(np.float64)
        scale = max(float(np.abs(k1).max(initial=0.0)), float(np.abs(k2).max(initial=0.0)), 1e-30)
        worst = max(worst, float(np.abs(k1 - k2).max(initial=0.0)) / scale)
        extra = np.concatenate([gk[r, m:n1], rk[r, m:n2]]).astype(np.float64)
        if extra.size:
            worst = max(worst, float(np.abs(extra - th).max()) / th)
        for y, x in list(gp[r, :n1]) + list(rp[r, :n2]):
            mask[y:y + bs, x:x + bs] = True
    unexplained = int(((d > MAX_ABS) & ~mask).sum())
    return unexplained, worst, flips
