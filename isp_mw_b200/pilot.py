"""Training data, training loop and evaluation of the learned pilot.

The pilot (``isp_mw_b200.Pilot``, kernels in ``csrc/pilot_kernels.cuh``) is an
8-layer 48-channel 3 x 3 convolutional network that stands in for the BM3D
basic estimate feeding the final (Wiener) stage. It regresses the basic
estimate this library computes:

* data: 128 x 128 crops of seeded synthetic 1920 x 1080 planes (the generator
  of ``isp_mw_b200.synth``: piecewise-smooth shapes plus a sinusoidal texture),
  each source plane with its own noise level sigma ~ U[5, 50] / 255; the
  target of a crop is the same crop of the plane's basic estimate (the basic
  stage run on the whole plane, as at inference);
* loss: squared error against the target, scaled per crop by
  (25/255 / sigma)^2 so that every noise level weighs alike; Adam with a
  warm-up and a cosine learning rate schedule, one ``bm3d_pilot_train_step``
  call per batch (forward, backward and update on the GPU).

Run ``python -m isp_mw_b200.pilot --out pilot.bin`` to train and save a
checkpoint.
"""
from __future__ import annotations

import argparse
import concurrent.futures as cf
import math
import multiprocessing as mp
import os
import time
from typing import Dict, List, Optional, Sequence

import numpy as np

from . import synth


def _plane(args):
    h, w, s255, seed = args
    return synth.pair(h, w, s255, seed)


def make_planes(count: int, shape=(1080, 1920), sigma_range=(5.0, 50.0), seed: int = 1234,
                workers: Optional[int] = None):
    """`count` seeded (clean, noisy, sigma_255) planes, generated in a process
    pool (spawned, so it is safe after CUDA is initialised)."""
    rng = np.random.default_rng(seed)
    sig = rng.uniform(sigma_range[0], sigma_range[1], count)
    jobs = [(shape[0], shape[1], float(sig[i]), seed * 1000 + i) for i in range(count)]
    workers = workers or max(1, min(count, (os.cpu_count() or 2) - 1, 32))
    if workers == 1:
        pairs = [_plane(j) for j in jobs]
    else:
        with cf.ProcessPoolExecutor(workers, mp_context=mp.get_context("spawn")) as pool:
            pairs = list(pool.map(_plane, jobs, chunksize=max(1, count // (4 * workers))))
    return [(c, n, float(s)) for (c, n), s in zip(pairs, sig)]


def make_dataset(ctx, crops: int = 20000, crop: int = 128, planes: int = 160,
                 shape=(1080, 1920), seed: int = 1234, workers: Optional[int] = None,
                 profile: str = "fast") -> Dict:
    """Crops of (noisy, basic estimate, clean) on the GPU, with each crop's
    true noise std (0-1 scale)."""
    import torch
    from . import stage_params_default
    src = make_planes(planes, shape, seed=seed, workers=workers)
    per = int(math.ceil(crops / planes))
    rng = np.random.default_rng(seed + 1)
    noisy_c, basic_c, clean_c, sig_c = [], [], [], []
    for clean, noisy, s255 in src:
        n_d = torch.from_numpy(noisy).cuda()
        b_d = torch.empty_like(n_d)
        p = stage_params_default(profile, False, [synth.sigma_param(s255)] * 3)
        ctx.stage(p, False, b_d, n_d)
        c_d = torch.from_numpy(clean).cuda()
        ys = rng.integers(0, shape[0] - crop + 1, per)
        xs = rng.integers(0, shape[1] - crop + 1, per)
        for y, x in zip(ys, xs):
            noisy_c.append(n_d[y:y + crop, x:x + crop])
            basic_c.append(b_d[y:y + crop, x:x + crop])
            clean_c.append(c_d[y:y + crop, x:x + crop])
            sig_c.append(s255 / 255.0)
    torch.cuda.synchronize()
    return {
        "noisy": torch.stack(noisy_c[:crops]).contiguous(),
        "target": torch.stack(basic_c[:crops]).contiguous(),
        "clean": torch.stack(clean_c[:crops]).contiguous(),
        "sigma": torch.tensor(sig_c[:crops], dtype=torch.float32, device="cuda"),
    }


def train(pilot, data: Dict, epochs: int = 30, batch: int = 32, lr: float = 5e-4,
          lr_min: float = 5e-6, warmup: int = 1000, seed: int = 0, log_every: int = 0) -> List:
    """Adam over shuffled batches: the rate rises linearly over the first
    `warmup` steps, then follows a cosine from `lr` to `lr_min` (a full-rate
    start can drive every ReLU of a layer negative, after which the network
    only passes the noisy plane through). Returns (step, loss) pairs (the loss
    of each batch before its update)."""
    import torch
    n = data["noisy"].shape[0]
    steps_per_epoch = n // batch
    total = epochs * steps_per_epoch
    g = torch.Generator(device="cuda").manual_seed(seed)
    hist = []
    step = 0
    for _ in range(epochs):
        perm = torch.randperm(n, device="cuda", generator=g)
        for k in range(steps_per_epoch):
            idx = perm[k * batch:(k + 1) * batch]
            rate = lr_min + 0.5 * (lr - lr_min) * (1.0 + math.cos(math.pi * step / max(1, total)))
            if step < warmup:
                rate *= (step + 1) / warmup
            loss = pilot.train_step(data["noisy"][idx].contiguous(), data["target"][idx].contiguous(),
                                    data["sigma"][idx].contiguous(), rate)
            hist.append((step, loss))
            if log_every and step % log_every == 0:
                print(f"step {step}/{total} lr {rate:.2e} loss {loss:.3e}", flush=True)
            step += 1
    return hist


def collapsed(hist: List) -> bool:
    """True when training ended no better than half its starting loss: the
    network went dead (every ReLU of a layer negative) and passes the noisy
    plane through."""
    if len(hist) < 600:
        return False
    first = float(np.mean([l for _, l in hist[:50]]))
    last = float(np.mean([l for _, l in hist[-500:]]))
    return not last < 0.5 * first


def fit(pilot, data: Dict, epochs: int = 30, batch: int = 32, lr: float = 5e-4, seed: int = 0,
        attempts: int = 3, log_every: int = 0):
    """train(), restarted from a fresh initialisation at half the rate when a
    run collapses. Returns (history of the last run, restarts)."""
    from . import Pilot
    hist: List = []
    for k in range(attempts):
        if k > 0:
            fresh = Pilot(pilot.ctx, seed=seed + 1000 * k)
            pilot.set_params(fresh.params())
            fresh.close()
        hist = train(pilot, data, epochs=epochs, batch=batch, lr=lr / (2 ** k), seed=seed + k,
                     log_every=log_every)
        if not collapsed(hist):
            return hist, k
    return hist, attempts - 1


def evaluate(ctx, pilot, sigmas: Sequence[float] = (5.0, 10.0, 25.0, 50.0), shape=(1080, 1920),
             seed: int = 99, profile: str = "fast") -> List[Dict]:
    """Plain BM3D (basic + final) against pilot + final on the same seeded
    planes: PSNR against the clean plane, and the pilot's PSNR against the
    basic estimate it stands in for."""
    from . import stage_params_default
    out = []
    for i, s255 in enumerate(sigmas):
        clean, noisy = synth.pair(shape[0], shape[1], s255, seed + i)
        sp = [synth.sigma_param(s255)] * 3
        b = stage_params_default(profile, False, sp)
        f = stage_params_default(profile, True, sp)
        basic = np.empty_like(noisy)
        ctx.stage(b, False, basic, noisy)
        plain = np.empty_like(noisy)
        ctx.stage(f, True, plain, noisy, basic)
        est = np.empty_like(noisy)
        pilot.estimate(est, noisy, np.float32(f.sigma[0] / math.sqrt(3.0) / 255.0))
        piloted = np.empty_like(noisy)
        pilot.full(f, piloted, noisy)
        out.append({
            "sigma": s255,
            "psnr_noisy": round(synth.psnr(noisy, clean), 3),
            "psnr_basic": round(synth.psnr(basic, clean), 3),
            "psnr_plain": round(synth.psnr(plain, clean), 3),
            "psnr_pilot_estimate": round(synth.psnr(est, clean), 3),
            "psnr_pilot_vs_basic": round(synth.psnr(est, basic), 3),
            "psnr_pilot_final": round(synth.psnr(piloted, clean), 3),
            "delta_db": round(synth.psnr(piloted, clean) - synth.psnr(plain, clean), 3),
        })
    return out


def main(argv=None):
    ap = argparse.ArgumentParser(description=__doc__.split("\n\n")[0])
    ap.add_argument("--out", default="pilot.bin")
    ap.add_argument("--crops", type=int, default=20000)
    ap.add_argument("--planes", type=int, default=160)
    ap.add_argument("--epochs", type=int, default=30)
    ap.add_argument("--batch", type=int, default=32)
    ap.add_argument("--lr", type=float, default=5e-4)
    ap.add_argument("--seed", type=int, default=0)
    args = ap.parse_args(argv)
    import json
    from . import Context, Pilot
    ctx = Context(0)
    t0 = time.time()
    data = make_dataset(ctx, crops=args.crops, planes=args.planes, seed=1234 + args.seed)
    t1 = time.time()
    pilot = Pilot(ctx, seed=args.seed)
    hist, restarts = fit(pilot, data, epochs=args.epochs, batch=args.batch, lr=args.lr,
                         seed=args.seed, log_every=100)
    t2 = time.time()
    pilot.save(args.out)
    res = evaluate(ctx, pilot)
    print(json.dumps({"data_s": round(t1 - t0, 1), "train_s": round(t2 - t1, 1),
                      "steps": len(hist), "restarts": restarts, "final_loss": hist[-1][1],
                      "eval": res}))


if __name__ == "__main__":
    main()
