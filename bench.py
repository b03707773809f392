"""BM3D throughput benchmark (megapixels per second).

Workload (one "step"): plain BM3D, basic + final, fast profile, on four
1920x1080 float32 luma planes -- the sigma sweep {5, 10, 25, 50}/255 --
generated by isp_mw_b200.synth (seeded piecewise-smooth planes + Gaussian
noise; synthetic, no dataset). Inputs rotate over a ring of sets whose total
size exceeds the 126 MB L2.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Our arm times K steps with CUDA events (barrier + synchronize on both sides,
max over ranks) on device-resident planes -> ``value``; then the same steps
through the C ABI with pinned host planes (host->device copy, filter,
device->host copy inside the timed region) -> ``e2e``. The roofline is taken
on the kernel the steps replay (the batch's persistent final-stage launch).
After the headline, the default run adds the 64-plane mixed batch (batch64)
and the 16-frame 4K YUV batch (yuv4k16) as extra keys. The reference arm
(--impl reference) runs the reference's own CPU BM3D (oracle/_ref, compiled
from the reference sources; the C restatement when that build is absent) on
the host cores: each step is one wave of whole 1920x1080 planes of the sweep,
one per thread (the reference is single-threaded per plane).
Multi-GPU: every rank filters its own planes (independent images, no
collective on the data path): weak scaling.
"""
from __future__ import annotations

import argparse
import concurrent.futures as cf
import json
import math
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

W, H = 1920, 1080
SIGMAS = (5.0, 10.0, 25.0, 50.0)
RING = 4
METRIC = "BM3D MP/s (basic+final, 1920x1080 luma, sigma sweep 5/10/25/50)"


def sweep_config(world: int) -> dict:
    """The headline workload's config, printed identically by both arms."""
    return {"workload": "BM3D basic+final, fast profile, 4 x 1920x1080 f32 luma planes "
                        "(sigma 5/10/25/50 per 255) per step",
            "width": W, "height": H, "planes_per_step": len(SIGMAS), "profile": "fast",
            "sigma_255": list(SIGMAS),
            "l2": f"inputs rotate over {RING} sets ({RING * len(SIGMAS) * W * H * 4 / 1e6:.0f} MB) "
                  "> 126 MB L2",
            "parallelism": f"replicas x{world} (independent planes per GPU)"}


def dist_env():
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return rank, world, local


class ClockSampler:
    """nvidia-smi samples of SM clock and throttle reasons during a region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.proc = None
        self.lines = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.index), f"--query-gpu={self.FIELDS}",
                 "--format=csv,noheader,nounits", "-lms", "50"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
            t0 = time.time()  # nvidia-smi takes a moment to start: have a sample before timing
            while not self.lines and self.proc.poll() is None and time.time() - t0 < 5.0:
                time.sleep(0.01)
        except OSError:
            self.proc = None
        return self

    def mark(self) -> int:
        """Index of the next sample (bracket a timed region with two marks)."""
        return len(self.lines)

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *exc):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()
            self.thread.join(timeout=2)

    def summary(self, lo: int = 0, hi: int | None = None):
        """Median SM clock and active throttle reasons over samples [lo, hi)
        (all samples when that range holds none)."""
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        lines = self.lines[lo:hi] or self.lines
        for ln in lines:
            parts = [p.strip() for p in ln.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                mx = float(parts[2])
            except ValueError:
                continue
            for n, v in zip(names, parts[5:9]):
                if v.lower() == "active":
                    reasons.add(n)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": mx, "reasons": sorted(reasons), "samples": 0}
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


def make_inputs(rank: int):
    from isp_mw_b200 import shard, synth
    sets = []
    for r in range(RING):
        planes = []
        for k, s in enumerate(SIGMAS):
            seed = shard.plane_seed(rank, r, k)
            _, noisy = synth.pair(H, W, s, seed)
            planes.append(noisy)
        sets.append(planes)
    return sets


def params_for(sigma_255: float):
    import isp_mw_b200
    from isp_mw_b200 import synth
    sp = [synth.sigma_param(sigma_255)] * 3
    return (isp_mw_b200.stage_params_default("fast", False, sp),
            isp_mw_b200.stage_params_default("fast", True, sp))


def algorithmic_flops(stats, wiener: bool, bs: int = 8) -> float:
    """Direct-formulation FLOPs of one stage launch from its counters:
    block matching 3 BS^2 per candidate; per group of n blocks a 3-D DCT of
    4 n BS^3 + 2 BS^2 n^2 (x2 basic: forward + inverse, x3 final: two forward
    + inverse); shrinkage 1 (hard threshold) or 5 (Wiener) per coefficient;
    aggregation 3 per pixel of every block."""
    sum_n, sum_n2, cand = stats[0], stats[1], stats[2]
    t = 3 if wiener else 2
    per_coef = 5 if wiener else 1
    dct = t * (4 * bs ** 3 * sum_n + 2 * bs ** 2 * sum_n2)
    return 3 * bs * bs * cand + dct + per_coef * bs * bs * sum_n + 3 * bs * bs * sum_n


def load_peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            return json.load(f)
    except OSError:
        return {}


BATCH_N = 64


def batch_inputs(rank: int):
    """The batched workload: 64 planes, width and height each uniform in
    [256, 2048], sigma uniform in [5, 50]/255, seeded."""
    from isp_mw_b200 import synth
    rng = np.random.default_rng(4242 + rank)
    sizes = rng.integers(256, 2049, size=(BATCH_N, 2))
    sigmas = rng.uniform(5.0, 50.0, size=BATCH_N)
    planes = []
    for k in range(BATCH_N):
        h, w = int(sizes[k, 0]), int(sizes[k, 1])
        _, noisy = synth.pair(h, w, float(sigmas[k]), 10_000 * (rank + 1) + k)
        planes.append(noisy)
    return planes, sigmas


def _timed_batch_runs(batch, dev, steps, warmup):
    import torch
    stream = torch.cuda.current_stream(dev)
    for _ in range(warmup):
        batch.run(stream.cuda_stream)
    torch.cuda.synchronize(dev)
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    ev0.record(stream)
    for _ in range(steps):
        batch.run(stream.cuda_stream)
    ev1.record(stream)
    torch.cuda.synchronize(dev)
    return ev0.elapsed_time(ev1) / steps


def measure_batch64(ctx, dev, rank, steps=10, warmup=3):
    """configs[2] on this GPU: the 64 mixed-size planes in one batch (device
    planes, CUDA-event timed steps)."""
    import torch
    import isp_mw_b200
    from isp_mw_b200 import synth
    planes, sigmas = batch_inputs(rank)
    pbs, pfs = [], []
    for s255 in sigmas:
        sp = [synth.sigma_param(float(s255))] * 3
        pbs.append(isp_mw_b200.stage_params_default("fast", False, sp))
        pfs.append(isp_mw_b200.stage_params_default("fast", True, sp))
    srcs = [torch.from_numpy(p).to(dev) for p in planes]
    dsts = [torch.empty_like(x) for x in srcs]
    batch = isp_mw_b200.Batch(ctx, pbs, pfs, dsts, srcs, autotune=True)
    ms = _timed_batch_runs(batch, dev, steps, warmup)
    mp = batch.pixels / 1e6
    out = {"workload": "64 planes, W,H ~ U[256,2048], sigma ~ U[5,50]/255, basic+final in one "
                       "persistent launch per stage from a CUDA graph (this GPU)",
           "value": round(mp / (ms / 1e3), 3), "unit": "MP/s", "steps": steps,
           "ms_per_step": round(ms, 4), "per_image_ms": round(ms / BATCH_N, 5),
           "megapixels": round(mp, 3), "tiling": batch.tuning()}
    batch.close()
    return out


def measure_yuv4k16(ctx, dev, rank, steps=3, warmup=2):
    """configs[4] (plain batched form) on this GPU: 16 YUV 4:4:4 3840x2160
    frames, luma groups reused for chroma, one batch."""
    import torch
    import isp_mw_b200
    from isp_mw_b200 import synth
    frames = yuv_inputs(rank)
    sp = [synth.sigma_param(YUV_SIGMAS[c], c) for c in range(3)]
    pb = isp_mw_b200.stage_params_default("fast", False, sp)
    pf = isp_mw_b200.stage_params_default("fast", True, sp)
    srcs = [[torch.from_numpy(p).to(dev) for p in f] for f in frames]
    dsts = [[torch.empty_like(p) for p in f] for f in srcs]
    batch = isp_mw_b200.Batch(ctx, [pb] * YUV_FRAMES, [pf] * YUV_FRAMES, dsts, srcs, autotune=True)
    ms = _timed_batch_runs(batch, dev, steps, warmup)
    mp = YUV_FRAMES * YUV_W * YUV_H / 1e6
    out = {"workload": "16 frames of 3840x2160 YUV 4:4:4 (sigma 15/10/10), luma groups reused "
                       "for chroma, basic+final in one persistent launch per stage from a CUDA "
                       "graph (this GPU); MP counts frame pixels",
           "value": round(mp / (ms / 1e3), 3), "unit": "MP/s", "steps": steps,
           "ms_per_step": round(ms, 3), "per_frame_ms": round(ms / YUV_FRAMES, 4),
           "tiling": batch.tuning()}
    batch.close()
    return out


YUV_FRAMES, YUV_W, YUV_H = 16, 3840, 2160
YUV_SIGMAS = (15.0, 10.0, 10.0)


def yuv_inputs(rank: int):
    """16 frames of 3840x2160 YUV 4:4:4: every plane generated independently
    (seeded piecewise-smooth + Gaussian noise), sigma 15/255 on luma and
    10/255 on chroma."""
    from isp_mw_b200 import synth

    def plane(k):
        c = k % 3
        return synth.pair(YUV_H, YUV_W, YUV_SIGMAS[c], 20_000 * (rank + 1) + k)[1]

    with cf.ThreadPoolExecutor(max(1, min(16, os.cpu_count() or 1))) as ex:
        flat = list(ex.map(plane, range(3 * YUV_FRAMES)))
    return [flat[3 * i:3 * i + 3] for i in range(YUV_FRAMES)]


def run_yuv(args):
    """Batched three-plane BM3D over a 4K video batch: 16 YUV 4:4:4 frames,
    block matching on luma with the groups reused for chroma, all frames in
    one persistent launch per stage from a CUDA graph."""
    import torch
    import torch.distributed as dist
    import isp_mw_b200
    from isp_mw_b200 import shard, synth

    rank, world, local = dist_env()
    torch.cuda.set_device(local)
    if world > 1:
        dist.init_process_group("nccl", timeout=__import__("datetime").timedelta(seconds=300))
    dev = torch.device("cuda", local)
    ctx = isp_mw_b200.Context(local)
    frames = yuv_inputs(rank)
    sp = [synth.sigma_param(YUV_SIGMAS[c], c) for c in range(3)]
    pb = isp_mw_b200.stage_params_default("fast", False, sp)
    pf = isp_mw_b200.stage_params_default("fast", True, sp)
    srcs = [[torch.from_numpy(p).to(dev) for p in f] for f in frames]
    dsts = [[torch.empty_like(p) for p in f] for f in srcs]
    t0 = time.perf_counter()
    batch = isp_mw_b200.Batch(ctx, [pb] * YUV_FRAMES, [pf] * YUV_FRAMES, dsts, srcs, autotune=True)
    build_s = time.perf_counter() - t0
    stream = torch.cuda.current_stream(dev)

    def barrier():
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize(dev)

    clk = ClockSampler(local).__enter__()
    for _ in range(args.warmup):
        batch.run()
    barrier()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    m0 = clk.mark()
    ev0.record(stream)
    for _ in range(args.steps):
        batch.run()
    ev1.record(stream)
    barrier()
    m1 = clk.mark()
    clk.__exit__(None, None, None)
    ms = shard.max_over_ranks(ev0.elapsed_time(ev1), dev)
    mp = YUV_FRAMES * YUV_W * YUV_H / 1e6
    value = world * mp * args.steps / (ms / 1e3)

    # end to end: page-locked host frames in, results out, every step, through
    # a three-plane host batch (bm3d_host_batch3_create): two device slots
    # let one step's uploads and downloads overlap the neighbouring steps'
    # filtering.
    pin_in = [[torch.from_numpy(p).pin_memory() for p in f] for f in frames]
    pin_out = [[torch.empty_like(p).pin_memory() for p in f] for f in pin_in]
    hb = isp_mw_b200.HostBatch(ctx, [pb] * YUV_FRAMES, [pf] * YUV_FRAMES,
                               [(YUV_H, YUV_W)] * YUV_FRAMES, autotune=True, planes=3)

    def step_e2e():
        hb.run(pin_out, pin_in, asynchronous="overlap", stream=stream.cuda_stream)

    for _ in range(2):  # builds both slots' graphs
        step_e2e()
    hb.join(stream.cuda_stream)
    barrier()
    e0 = time.perf_counter()
    ev0.record(stream)
    for _ in range(args.steps):
        step_e2e()
    hb.join(stream.cuda_stream)  # every step's download is inside the timed region
    ev1.record(stream)
    barrier()
    e_wall = (time.perf_counter() - e0) * 1e3
    e_ms = shard.max_over_ranks(max(ev0.elapsed_time(ev1), e_wall), dev)
    hb.close()
    nbytes = 3 * 4 * YUV_FRAMES * YUV_W * YUV_H
    if rank == 0:
        line = {
            "metric": "batched 3-plane BM3D MP/s (16 x 3840x2160 YUV 4:4:4, sigma 15/10/10, "
                      "luma groups reused for chroma)",
            "value": round(value, 3), "unit": "MP/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": round(ms / args.steps, 4),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic (seeded piecewise-smooth planes + Gaussian noise)",
            "config": {"workload": "batched plain BM3D basic+final, fast profile, 16 YUV 4:4:4 "
                                   "3840x2160 frames per step (MP counts frame pixels), three "
                                   "planes per frame sharing luma groups, one persistent "
                                   "launch per stage from a CUDA graph",
                       "frames": YUV_FRAMES, "width": YUV_W, "height": YUV_H,
                       "sigma_255": list(YUV_SIGMAS), "tiling": batch.tuning(),
                       "graph_build_s": round(build_s, 3), "parallelism": f"replicas x{world}",
                       "l2": "inputs 1.6 GB per step > 126 MB L2"},
            "per_frame_ms": round(ms / args.steps / YUV_FRAMES, 4),
            "e2e": {"value": round(world * mp * args.steps / (e_ms / 1e3), 3), "unit": "MP/s",
                    "h2d_bytes_per_step": nbytes, "d2h_bytes_per_step": nbytes},
            "gpu_launches": args.steps * 6,
            "clocks": clk.summary(m0, m1),
        }
        print(json.dumps(line), flush=True)
    batch.close()
    ctx.close()
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()


def run_batch(args):
    """Batched BM3D over 64 mixed-size planes: all of them in one persistent
    launch per stage, replayed from a CUDA graph; tiling from the autotuner."""
    import torch
    import torch.distributed as dist
    import isp_mw_b200
    from isp_mw_b200 import shard, synth

    rank, world, local = dist_env()
    torch.cuda.set_device(local)
    if world > 1:
        dist.init_process_group("nccl", timeout=__import__("datetime").timedelta(seconds=120))
    dev = torch.device("cuda", local)
    ctx = isp_mw_b200.Context(local)
    planes, sigmas = batch_inputs(rank)
    pbs, pfs = [], []
    for s255 in sigmas:
        sp = [synth.sigma_param(float(s255))] * 3
        pbs.append(isp_mw_b200.stage_params_default("fast", False, sp))
        pfs.append(isp_mw_b200.stage_params_default("fast", True, sp))
    srcs = [torch.from_numpy(p).to(dev) for p in planes]
    dsts = [torch.empty_like(x) for x in srcs]
    t0 = time.perf_counter()
    batch = isp_mw_b200.Batch(ctx, pbs, pfs, dsts, srcs, autotune=True)
    build_s = time.perf_counter() - t0
    stream = torch.cuda.current_stream(dev)

    def barrier():
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize(dev)

    clk = ClockSampler(local).__enter__()
    for _ in range(args.warmup):
        batch.run()
    barrier()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    m0 = clk.mark()
    ev0.record(stream)
    for _ in range(args.steps):
        batch.run()
    ev1.record(stream)
    barrier()
    m1 = clk.mark()
    clk.__exit__(None, None, None)
    ms = shard.max_over_ranks(ev0.elapsed_time(ev1), dev)
    mp = batch.pixels / 1e6
    value = world * mp * args.steps / (ms / 1e3)

    # end to end: pinned host planes in, results out, every step, through a
    # host batch (bm3d_host_batch): two device slots let one step's copies
    # overlap the neighbouring steps' filtering.
    pin_in = [torch.from_numpy(p).pin_memory() for p in planes]
    pin_out = [torch.empty(p.shape, dtype=torch.float32).pin_memory() for p in planes]
    hb = isp_mw_b200.HostBatch(ctx, pbs, pfs, [p.shape for p in planes], autotune=True)

    def step_e2e():
        hb.run(pin_out, pin_in, asynchronous="overlap", stream=stream.cuda_stream)

    for _ in range(2):  # builds both slots' graphs
        step_e2e()
    hb.join(stream.cuda_stream)
    barrier()
    e0 = time.perf_counter()
    ev0.record(stream)
    for _ in range(args.steps):
        step_e2e()
    hb.join(stream.cuda_stream)  # every step's download is inside the timed region
    ev1.record(stream)
    barrier()
    e_wall = (time.perf_counter() - e0) * 1e3
    e_ms = shard.max_over_ranks(max(ev0.elapsed_time(ev1), e_wall), dev)
    hb.close()
    nbytes = 4 * batch.pixels
    if rank == 0:
        line = {
            "metric": "batched BM3D MP/s (64 planes, W,H ~ U[256,2048], sigma ~ U[5,50]/255)",
            "value": round(value, 3), "unit": "MP/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": round(ms / args.steps, 4),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic (seeded piecewise-smooth planes + Gaussian noise)",
            "config": {"workload": "batched BM3D basic+final, fast profile, 64 planes per step "
                                   "in one persistent launch per stage from a CUDA graph",
                       "planes": BATCH_N, "megapixels": round(mp, 3),
                       "tiling": batch.tuning(), "graph_build_s": round(build_s, 3),
                       "parallelism": f"replicas x{world}"},
            "per_image_ms": round(ms / args.steps / BATCH_N, 5),
            "e2e": {"value": round(world * mp * args.steps / (e_ms / 1e3), 3), "unit": "MP/s",
                    "h2d_bytes_per_step": nbytes, "d2h_bytes_per_step": nbytes},
            "gpu_launches": args.steps * 6,
            "clocks": clk.summary(m0, m1),
        }
        print(json.dumps(line), flush=True)
    batch.close()
    ctx.close()
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()


# DRAM bytes (dram__bytes_read.sum + dram__bytes_write.sum) per persistent
# batch launch over the step's four 1920x1080 planes. Until a capture of the
# batch kernel itself is committed these are four times the per-plane
# stage_kernel captures (profiles/stage_kernel_{final,basic}_1080p_full.txt):
# the batch kernel runs the same per-tile body over the same tiles.
TRAFFIC_FINAL_1080P = 46.487e6 + 0.0e6
TRAFFIC_BASIC_1080P = 37.286e6 + 0.004e6
TRAFFIC_BATCH_FINAL_4X1080P = 4 * TRAFFIC_FINAL_1080P
TRAFFIC_BATCH_BASIC_4X1080P = 4 * TRAFFIC_BASIC_1080P
TRAFFIC_SOURCE = ("4 x the per-plane stage_kernel capture on one 1920x1080 plane, sigma 25 "
                  "(profiles/stage_kernel_final_1080p_full.txt, stage_kernel_basic_1080p_full.txt)")


def run_ours(args):
    import torch
    import torch.distributed as dist
    import isp_mw_b200

    rank, world, local = dist_env()
    torch.cuda.set_device(local)
    if world > 1:
        dist.init_process_group("nccl", timeout=__import__("datetime").timedelta(seconds=120))
    dev = torch.device("cuda", local)
    ctx = isp_mw_b200.Context(local)
    params = [params_for(s) for s in SIGMAS]
    host_sets = make_inputs(rank)
    dev_sets = [[torch.from_numpy(p).to(dev) for p in planes] for planes in host_sets]
    outs = [torch.empty((H, W), dtype=torch.float32, device=dev) for _ in SIGMAS]
    stream = torch.cuda.current_stream(dev)

    # One batch (persistent basic + final launches in a CUDA graph) per input set.
    batches = [isp_mw_b200.Batch(ctx, [p[0] for p in params], [p[1] for p in params], outs,
                                 planes, autotune=True) for planes in dev_sets]

    def step(i):
        batches[i % RING].run(stream.cuda_stream)

    def barrier():
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize(dev)

    clk = ClockSampler(local).__enter__()  # samples warm-up, timed and kernel-timing passes
    for i in range(args.warmup):
        step(i)
    barrier()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    m0 = clk.mark()
    ev0.record(stream)
    for i in range(args.steps):
        step(args.warmup + i)
    ev1.record(stream)
    barrier()
    m1 = clk.mark()
    from isp_mw_b200 import shard
    ms_max = shard.max_over_ranks(ev0.elapsed_time(ev1), dev)
    mp_step = len(SIGMAS) * W * H / 1e6
    value = world * mp_step * args.steps / (ms_max / 1e3)

    # Kernel roofline, on the kernel the timed steps replay: the batch's
    # persistent stage launches (four planes each), timed with CUDA events on
    # their stream in eager runs of the same pipeline. Algorithmic FLOPs come
    # from the kernels' own counters (group sizes, candidates) of per-plane
    # runs on the same inputs, which produce the same groups.
    ctx.set_kernel_timing(True)
    flops_set = []
    for r in range(RING):
        fl = {False: 0.0, True: 0.0}
        for k in range(len(SIGMAS)):
            b = torch.empty_like(outs[k])
            ctx.stage(params[k][0], False, b, dev_sets[r][k])
            fl[False] += algorithmic_flops(ctx.last_stats(), False)
            ctx.stage(params[k][1], True, outs[k], dev_sets[r][k], b)
            fl[True] += algorithmic_flops(ctx.last_stats(), True)
        flops_set.append(fl)
    t_basic, n_basic = ctx.kernel_time(False)  # per-plane stage_kernel launches (reported beside)
    t_final, n_final = ctx.kernel_time(True)
    ctx.set_kernel_timing(False)
    reps = max(RING, min(args.steps, 40))
    bt = {False: 0.0, True: 0.0}
    bfl = {False: 0.0, True: 0.0}
    for i in range(reps):
        tb, tf = batches[i % RING].stage_times(stream.cuda_stream)
        bt[False] += tb
        bt[True] += tf
        bfl[False] += flops_set[i % RING][False]
        bfl[True] += flops_set[i % RING][True]
    clk.__exit__(None, None, None)
    dom = bt[True] >= bt[False]
    per_launch_ms = bt[dom] / reps
    achieved = bfl[dom] / reps / (per_launch_ms / 1e3) / 1e12
    clocks = clk.summary(m0, m1)
    sm_max = clocks.get("sm_max_mhz") or 1965.0
    peak_fp32 = 148 * 128 * 2 * sm_max * 1e6 / 1e12

    # End to end through the C ABI: pinned host planes in, results out.
    pinned_in = [[torch.from_numpy(p).pin_memory() for p in planes] for planes in host_sets]
    pinned_out = [torch.empty((H, W), dtype=torch.float32).pin_memory() for _ in SIGMAS]

    # A host batch (bm3d_host_batch) on page-locked host planes: each step
    # uploads its four planes, replays the batch graph and downloads the
    # results; two device slots let one step's copies overlap the
    # neighbouring steps' filtering.
    hb = isp_mw_b200.HostBatch(ctx, [p[0] for p in params], [p[1] for p in params],
                               [(H, W)] * len(SIGMAS), autotune=True)

    def step_e2e(i):
        hb.run(pinned_out, pinned_in[i % RING], asynchronous="overlap", stream=stream.cuda_stream)

    for i in range(min(args.warmup, 3)):
        step_e2e(i)
    hb.join(stream.cuda_stream)
    barrier()
    e0 = time.perf_counter()
    ev0.record(stream)
    for i in range(args.steps):
        step_e2e(i)
    hb.join(stream.cuda_stream)  # every step's download is inside the timed region
    ev1.record(stream)
    barrier()
    e_wall = (time.perf_counter() - e0) * 1e3
    e_ms = shard.max_over_ranks(max(ev0.elapsed_time(ev1), e_wall), dev)
    e2e_value = world * mp_step * args.steps / (e_ms / 1e3)

    # configs[2] and configs[4] as extra keys, measured after the headline
    # (outside its timed region): the 64-plane mixed batch and the 16-frame
    # 4K YUV batch, device-resident, CUDA-event timed
    extras = {}
    if not args.no_extras:
        extras["batch64"] = measure_batch64(ctx, dev, rank, steps=10, warmup=3)
        extras["yuv4k16"] = measure_yuv4k16(ctx, dev, rank, steps=3, warmup=2)

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cpu = cpu_baseline(host_sets[0], budget_s=args.cpu_seconds)

    if rank == 0:
        peaks = load_peaks()
        if peaks.get("hbm_gbs"):
            hbm_peak, hbm_source = float(peaks["hbm_gbs"]), "measured (MEASURED_PEAKS.json)"
        else:  # an earlier STREAM-style copy measurement on these B200s
            hbm_peak, hbm_source = 6650.0, "fallback 6.65 TB/s (MEASURED_PEAKS.json absent)"
        traffic = (TRAFFIC_BATCH_FINAL_4X1080P if dom else TRAFFIC_BATCH_BASIC_4X1080P)
        line = {
            "metric": METRIC,
            "value": round(value, 3),
            "unit": "MP/s",
            "n_gpus": world,
            "steps": args.steps,
            "warmup": args.warmup,
            "ms_per_step": round(ms_max / args.steps, 4),
            "higher_is_better": True,
            "scaling": "weak",
            "vs_baseline": None,
            "dtype": "f32",
            "data": "synthetic (seeded piecewise-smooth planes + Gaussian noise)",
            "config": sweep_config(world),
            "step": "one batched graph replay (persistent basic + final launches over the 4 "
                    "planes) per step",
            "tiling": batches[0].tuning(),
            "e2e": {"value": round(e2e_value, 3), "unit": "MP/s",
                    "h2d_bytes_per_step": len(SIGMAS) * W * H * 4,
                    "d2h_bytes_per_step": len(SIGMAS) * W * H * 4},
            "gpu_launches": args.steps * 6,
            "roofline": {
                "bound": "fp32",
                "kernel": "batch_stage_kernel (final)" if dom else "batch_stage_kernel (basic)",
                "launch": "one persistent launch over the 4 planes of a step, the kernel the "
                          "timed steps replay; CUDA events on its stream in eager runs of the "
                          "same pipeline",
                "achieved": round(achieved, 3),
                "peak": round(peak_fp32, 2),
                "unit": "TFLOP/s",
                "frac": round(achieved / peak_fp32, 4),
                "traffic": traffic,
                "traffic_source": TRAFFIC_SOURCE,
                "peak_source": "nominal FP32 FMA rate 148 SM x 128 lanes x 2 flop x max SM clock "
                               "(MEASURED_PEAKS.json has no FP32 SIMT figure)",
                "per_launch_ms": round(per_launch_ms, 4),
                "algorithmic_gflop_per_launch": round(bfl[dom] / reps / 1e9, 3),
                "hbm_peak_gbs": hbm_peak,
                "hbm_peak_source": hbm_source,
                "dram_gbs": round(traffic / (per_launch_ms / 1e3) / 1e9, 1),
                "dram_frac": round(traffic / (per_launch_ms / 1e3) / 1e9 / hbm_peak, 4),
            },
            "batch_stage_ms_per_launch": {"basic": round(bt[False] / reps, 4),
                                          "final": round(bt[True] / reps, 4)},
            "stage_ms_per_plane": {"basic": round(t_basic / max(1, n_basic), 4),
                                   "final": round(t_final / max(1, n_final), 4),
                                   "kernel": "stage_kernel, one launch per plane"},
            "clocks": clocks,
        }
        line.update(extras)
        if cpu is not None:
            line["cpu_baseline"] = cpu
        print(json.dumps(line), flush=True)
    for b in batches:
        b.close()
    hb.close()
    ctx.close()
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()


def _ref_backend():
    import oracle
    kind = "reference" if oracle.reference_available() else "port"
    if kind == "port":
        oracle.build(reference=False)
    return kind, oracle.backend(kind, np.float32)


def _cpu_tasks(planes, rows: int, count: int = 0):
    """(plane index, strip) tasks of `rows` rows each over the step's planes,
    cycled until there are `count` of them (0: one pass)."""
    tasks = []
    for k, p in enumerate(planes):
        for y0 in range(0, H, rows):
            y1 = min(H, y0 + rows)
            if y1 - y0 >= 16:
                tasks.append((k, np.ascontiguousarray(p[y0:y1])))
    base = list(tasks)
    while len(tasks) < count:
        tasks.append(base[len(tasks) % len(base)])
    return tasks


def _plane_tasks(planes, count: int):
    """`count` whole-plane tasks cycling over the step's planes."""
    return [(k % len(planes), planes[k % len(planes)]) for k in range(count)]


def _run_cpu(backend, tasks, cores):
    px = sum(t[1].size for t in tasks)

    def one(t):
        k, plane = t
        backend.full(_PARAMS[k][0], _PARAMS[k][1], plane)

    t0 = time.perf_counter()
    with cf.ThreadPoolExecutor(max_workers=cores) as ex:
        list(ex.map(one, tasks))
    return px, time.perf_counter() - t0


_PARAMS = []


def _init_params():
    import oracle
    from isp_mw_b200 import synth
    _PARAMS.clear()
    for s in SIGMAS:
        sp = [synth.sigma_param(s)] * 3
        if oracle.reference_available():
            _PARAMS.append((oracle.reference_stage_default("fast", False, sp),
                            oracle.reference_stage_default("fast", True, sp)))
        else:
            import isp_mw_b200
            _PARAMS.append((isp_mw_b200.stage_params_default("fast", False, sp).as_dict(),
                            isp_mw_b200.stage_params_default("fast", True, sp).as_dict()))


def _bm_only(backend, plane, k):
    """Single-thread seconds of the reference's block matching alone over the
    basic and final scans of one plane (BM3D_Base::BlockMatching,
    source/BM3D.cpp:221-236, through the group dump), against the whole
    basic + final on that plane."""
    b, f = _PARAMS[k]
    t0 = time.perf_counter()
    basic = backend.stage(False, b, plane)
    t1 = time.perf_counter()
    backend.stage(True, f, plane, basic)
    t2 = time.perf_counter()
    backend.groups(False, b, plane)
    t3 = time.perf_counter()
    backend.groups(True, f, basic)
    t4 = time.perf_counter()
    return {"plane": f"1920x1080 sigma {SIGMAS[k]:g}", "threads": 1,
            "basic_s": round(t1 - t0, 3), "final_s": round(t2 - t1, 3),
            "bm_basic_s": round(t3 - t2, 3), "bm_final_s": round(t4 - t3, 3),
            "bm_fraction": round((t4 - t2) / (t2 - t0), 3)}


def cpu_baseline(planes, budget_s: float = 20.0):
    """The reference's CPU BM3D on this host's cores, on a bounded sample of
    the workload: whole 1920x1080 planes of the step (basic + final each, the
    reference being single-threaded per plane), one plane per core at a time,
    waves until about `budget_s`; plus the block-matching share of one plane."""
    kind, backend = _ref_backend()
    _init_params()
    cores = len(os.sched_getaffinity(0))
    px, t = _run_cpu(backend, _plane_tasks(planes, cores), cores)  # first wave calibrates
    waves = max(1, int(round(budget_s / t)))
    if waves > 1:
        px2, t2 = _run_cpu(backend, _plane_tasks(planes, cores * (waves - 1)), cores)
        px, t = px + px2, t + t2
    n = cores * waves
    return {"value": round(px / t / 1e6, 4), "unit": "MP/s", "cores": cores, "kind": kind,
            "sample": f"{n} whole 1920x1080 planes cycled over the step's 4 planes (sigma "
                      f"sweep), basic+final fast profile, {px / 1e6:.1f} MP in {t:.1f} s, one "
                      f"plane per thread at a time on {cores} threads",
            "bm_only": _bm_only(backend, planes[2], 2)}


def run_reference(args):
    rank, world, _ = dist_env()
    if rank != 0:
        return
    kind, backend = _ref_backend()
    _init_params()
    cores = len(os.sched_getaffinity(0))
    planes = make_inputs(0)[0]
    # a step is one wave: `cores` whole planes of the sweep, one per thread.
    # The first warm-up wave calibrates; when the run would not end within
    # about five minutes, each step is a wave of strips instead (the ratio of
    # whole-plane to strip rate measured on the same cores is reported).
    tasks = _plane_tasks(planes, cores)
    px0, t0 = _run_cpu(backend, tasks, cores)
    sample = f"one wave per step: {cores} whole 1920x1080 planes of the sweep, one per thread"
    strip_ratio = None
    if (args.steps + max(0, args.warmup - 1)) * t0 > 300.0:
        strips = _cpu_tasks(planes, 120)
        _, ts = _run_cpu(backend, strips[:cores], cores)
        per_step = cores * max(1, int(300.0 / max(1, args.steps + args.warmup) / max(1e-6, ts)))
        tasks = _cpu_tasks(planes, 120, per_step)[:per_step]
        spx, st = _run_cpu(backend, tasks, cores)
        strip_ratio = round((px0 / t0) / (spx / st), 4)
        sample = (f"{per_step} strips of 1920x120 per step (whole planes would exceed the time "
                  f"budget), on {cores} threads")
    for _ in range(max(0, args.warmup - 1)):
        _run_cpu(backend, tasks, cores)
    tot_px, tot_t = 0, 0.0
    for _ in range(args.steps):
        px, t = _run_cpu(backend, tasks, cores)
        tot_px += px
        tot_t += t
    value = tot_px / tot_t / 1e6
    line = {
        "impl": "reference",
        "metric": METRIC,
        "value": round(value, 4),
        "unit": "MP/s",
        "n_gpus": world,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": round(tot_t / args.steps * 1e3, 2),
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f32",
        "data": "synthetic (seeded piecewise-smooth planes + Gaussian noise)",
        "config": sweep_config(world),
        "cpu_baseline": {"value": round(value, 4), "unit": "MP/s", "cores": cores, "kind": kind,
                         "sample": sample},
        "e2e": {"value": round(value, 4), "unit": "MP/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
    }
    if strip_ratio is not None:
        line["cpu_baseline"]["whole_over_strip_rate"] = strip_ratio
    print(json.dumps(line), flush=True)


def _trained_pilot(ctx, args):
    """The pilot for the pilot workloads: loaded from --pilot-checkpoint when
    that file exists, else trained on 20k 128x128 crops (and saved there when
    a path is given). Returns (pilot, loss history, data s, train s)."""
    import torch
    import isp_mw_b200
    from isp_mw_b200 import pilot as pilot_mod
    t0 = time.perf_counter()
    pilot = isp_mw_b200.Pilot(ctx, seed=0)
    hist = []
    t1 = t0
    if args.pilot_checkpoint and os.path.exists(args.pilot_checkpoint):
        pilot.load(args.pilot_checkpoint)
    else:
        data = pilot_mod.make_dataset(ctx, crops=args.pilot_crops, planes=160)
        t1 = time.perf_counter()
        hist, pilot.restarts = pilot_mod.fit(pilot, data, epochs=args.pilot_epochs)
        del data
        if args.pilot_checkpoint:
            pilot.save(args.pilot_checkpoint)
    torch.cuda.synchronize()
    return pilot, hist, t1 - t0, time.perf_counter() - t1


def run_pilot_yuv(args):
    """configs[4] with the learned pilot: 16 frames of 3840x2160 YUV 4:4:4
    (sigma 15/10/10), the pilot on every plane (in chunks of four frames),
    then one final-stage-only batch over all frames with the groups matched on
    the pilot's luma estimate and reused for chroma -- against the plain
    batched form (basic + final) on the same frames, MP/s and PSNR against
    the clean planes."""
    import torch
    import isp_mw_b200
    from isp_mw_b200 import synth

    rank, world, local = dist_env()
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    ctx = isp_mw_b200.Context(local)
    pilot, hist, t_data, t_train = _trained_pilot(ctx, args)

    def plane(k):
        c = k % 3
        return synth.pair(YUV_H, YUV_W, YUV_SIGMAS[c], 20_000 * (rank + 1) + k)

    with cf.ThreadPoolExecutor(max(1, min(16, os.cpu_count() or 1))) as ex:
        pairs = list(ex.map(plane, range(3 * YUV_FRAMES)))
    src = torch.stack([torch.from_numpy(n) for _, n in pairs]).to(dev).contiguous()
    est = torch.empty_like(src)
    out = torch.empty_like(src)
    sp = [synth.sigma_param(YUV_SIGMAS[c], c) for c in range(3)]
    pb = isp_mw_b200.stage_params_default("fast", False, sp)
    pf = isp_mw_b200.stage_params_default("fast", True, sp)
    sig = torch.tensor([YUV_SIGMAS[k % 3] / 255.0 for k in range(3 * YUV_FRAMES)],
                       dtype=torch.float32, device=dev)
    frames = lambda t: [[t[3 * i + c] for c in range(3)] for i in range(YUV_FRAMES)]
    plain = isp_mw_b200.Batch(ctx, [pb] * YUV_FRAMES, [pf] * YUV_FRAMES, frames(out), frames(src),
                              autotune=True)
    fin = isp_mw_b200.Batch(ctx, [pf] * YUV_FRAMES, [pf] * YUV_FRAMES, frames(out), frames(src),
                            autotune=True, ref=frames(est))
    stream = torch.cuda.current_stream(dev)
    chunk = 12  # planes per pilot call (four frames)
    lib = ctx.lib

    def pilot_net():
        for k0 in range(0, 3 * YUV_FRAMES, chunk):
            ctx._check(lib.bm3d_pilot_estimate(pilot.h, est[k0].data_ptr(), src[k0].data_ptr(),
                                               chunk, YUV_W, YUV_H, YUV_W, YUV_W * YUV_H,
                                               sig[k0:].data_ptr(), isp_mw_b200.MEM_DEVICE,
                                               stream.cuda_stream))

    def pilot_step():
        pilot_net()
        fin.run(stream.cuda_stream)

    def timed(fn, steps, warmup):
        for _ in range(warmup):
            fn()
        torch.cuda.synchronize(dev)
        ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        ev0.record(stream)
        for _ in range(steps):
            fn()
        ev1.record(stream)
        torch.cuda.synchronize(dev)
        return ev0.elapsed_time(ev1) / steps

    clk = ClockSampler(local).__enter__()
    m0 = clk.mark()
    ms_pilot = timed(pilot_step, args.steps, args.warmup)
    m1 = clk.mark()
    ms_plain = timed(lambda: plain.run(stream.cuda_stream), args.steps, args.warmup)
    ms_net = timed(pilot_net, args.steps, args.warmup)
    clk.__exit__(None, None, None)
    plain.run(stream.cuda_stream)
    torch.cuda.synchronize(dev)
    clean = [c for c, _ in pairs]
    p_plain = [synth.psnr(out[k].cpu().numpy(), clean[k]) for k in range(3 * YUV_FRAMES)]
    pilot_step()
    torch.cuda.synchronize(dev)
    p_pilot = [synth.psnr(out[k].cpu().numpy(), clean[k]) for k in range(3 * YUV_FRAMES)]
    mp = YUV_FRAMES * YUV_W * YUV_H / 1e6
    mean = lambda v, c: round(float(np.mean([v[k] for k in range(c, len(v), 3)])), 3)
    if rank == 0:
        print(json.dumps({
            "metric": "batched learned-pilot BM3D MP/s (16 x 3840x2160 YUV 4:4:4, sigma 15/10/10, "
                      "luma groups reused for chroma)",
            "value": round(mp / (ms_pilot / 1e3), 3), "unit": "MP/s", "n_gpus": 1,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(ms_pilot, 3),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "bf16 (pilot, FP32 accumulation) + f32 (final stage)",
            "data": "synthetic (seeded piecewise-smooth planes + Gaussian noise)",
            "config": {"workload": "learned pilot on all 48 planes (12 per call), then one "
                                   "final-stage-only batch (bm3d_batch3_final_create) over the 16 "
                                   "frames with groups matched on the pilot's luma estimate; MP "
                                   "counts frame pixels", "frames": YUV_FRAMES, "width": YUV_W,
                       "height": YUV_H, "sigma_255": list(YUV_SIGMAS),
                       "train_steps": len(hist), "data_s": round(t_data, 1),
                       "train_s": round(t_train, 1)},
            "plain": {"value": round(mp / (ms_plain / 1e3), 3), "unit": "MP/s",
                      "ms_per_step": round(ms_plain, 3)},
            "pilot_over_plain": round(ms_plain / ms_pilot, 4),
            "pilot_network_ms_per_step": round(ms_net, 3),
            "psnr_vs_clean_mean": {"plain": {"Y": mean(p_plain, 0), "U": mean(p_plain, 1),
                                             "V": mean(p_plain, 2)},
                                   "pilot": {"Y": mean(p_pilot, 0), "U": mean(p_pilot, 1),
                                             "V": mean(p_pilot, 2)}},
            "gpu_launches": args.steps * (4 * 8 + 3),
            "clocks": clk.summary(m0, m1),
        }), flush=True)
    fin.close()
    plain.close()
    pilot.close()
    ctx.close()


# DRAM bytes (read + write) of one 48 -> 48 layer launch on one 1920x1080
# plane, per forward kernel, from the ncu captures named beside them
PILOT_CONV_TRAFFIC_PER_PLANE = {
    "conv48_n144_kernel": (199_203_328 + 158_855_680,
                           "profiles/conv48_n144_kernel_1080p_full.txt"),
    "conv48_tma_kernel": (199_160_576 + 156_573_952,
                          "profiles/conv48_tma_kernel_1080p_full.txt"),
}


def run_pilot(args):
    """the learned pilot in place of the basic estimate. Trains
    the pilot on 20k 128x128 crops of synthetic 1920x1080 planes (sigma ~
    U[5, 50]) regressing this library's basic estimate (untimed; its time is
    reported), then times pilot + final against plain basic + final on the
    sweep's four 1920x1080 planes on this GPU and reports PSNR against the
    clean planes for both."""
    import torch
    import isp_mw_b200
    from isp_mw_b200 import pilot as pilot_mod, synth

    rank, world, local = dist_env()
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    ctx = isp_mw_b200.Context(local)
    pilot, hist, t_data, t_train = _trained_pilot(ctx, args)
    evals = pilot_mod.evaluate(ctx, pilot)

    params = [params_for(s) for s in SIGMAS]
    clean_noisy = [synth.pair(H, W, s, 77 + k) for k, s in enumerate(SIGMAS)]
    srcs = [torch.from_numpy(n).to(dev) for _, n in clean_noisy]
    stack = torch.stack(srcs).contiguous()
    est = torch.empty_like(stack)
    outs = [torch.empty_like(x) for x in srcs]
    sig = np.array([params[k][1].sigma[0] / math.sqrt(3.0) / 255.0 for k in range(len(SIGMAS))],
                   np.float32)
    sig_d = torch.from_numpy(sig).to(dev)
    stream = torch.cuda.current_stream(dev)
    lib = ctx.lib

    def pilot_net():
        ctx._check(lib.bm3d_pilot_estimate(pilot.h, est.data_ptr(), stack.data_ptr(),
                                           len(SIGMAS), W, H, W, W * H, sig_d.data_ptr(),
                                           isp_mw_b200.MEM_DEVICE, stream.cuda_stream))

    # the pilot pipeline: the network on the step's four planes, then the
    # final stage of all four as one final-stage-only batch fed by its output
    pbatch = isp_mw_b200.Batch(ctx, [p[1] for p in params], [p[1] for p in params], outs,
                               [stack[k] for k in range(len(SIGMAS))], autotune=True,
                               ref=[est[k] for k in range(len(SIGMAS))])

    def pilot_step():
        pilot_net()
        pbatch.run(stream.cuda_stream)

    batch = isp_mw_b200.Batch(ctx, [p[0] for p in params], [p[1] for p in params], outs, srcs,
                              autotune=True)

    def timed(fn, steps, warmup):
        for _ in range(warmup):
            fn()
        torch.cuda.synchronize(dev)
        ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        ev0.record(stream)
        for _ in range(steps):
            fn()
        ev1.record(stream)
        torch.cuda.synchronize(dev)
        return ev0.elapsed_time(ev1) / steps

    clk = ClockSampler(local).__enter__()
    m0 = clk.mark()
    ms_pilot = timed(pilot_step, args.steps, args.warmup)
    m1 = clk.mark()
    ms_plain = timed(lambda: batch.run(stream.cuda_stream), args.steps, args.warmup)
    ms_cnn = timed(pilot_net, args.steps, args.warmup)
    tb = tf = tpf = 0.0
    for _ in range(8):
        a, b = batch.stage_times(stream.cuda_stream)
        tb, tf = tb + a / 8, tf + b / 8
        tpf += pbatch.stage_times(stream.cuda_stream)[1] / 8
    clk.__exit__(None, None, None)
    # PSNR on these planes: plain (the batch's output) and pilot + final
    batch.run(stream.cuda_stream)
    torch.cuda.synchronize(dev)
    plain_out = [o.cpu().numpy() for o in outs]
    pilot_step()
    torch.cuda.synchronize(dev)
    pilot_out = [o.cpu().numpy() for o in outs]
    psnr = [{"sigma": s, "plain": round(synth.psnr(plain_out[k], clean_noisy[k][0]), 3),
             "pilot": round(synth.psnr(pilot_out[k], clean_noisy[k][0]), 3)}
            for k, s in enumerate(SIGMAS)]
    for q in psnr:
        q["delta_db"] = round(q["pilot"] - q["plain"], 3)
    mp = len(SIGMAS) * W * H / 1e6
    flops_cnn = len(SIGMAS) * W * H * 2 * 9 * (2 * 48 + 6 * 48 * 48 + 48)
    peaks = load_peaks()
    bf16_peak = float(peaks.get("bf16_tflops", 1590.0))
    # the dominant kernel: the six 48 -> 48 layers of the pilot's forward
    # pass over the step's four planes, each one launch, timed with CUDA
    # events recorded around each layer on the launching stream
    pilot.set_timing(True)
    lay = np.zeros(8)
    for _ in range(10):
        pilot_net()
        lay += pilot.layer_ms() / 10
    pilot.set_timing(False)
    ms_conv = float(lay[1:7].mean())
    conv_kernel = {3: "conv48_n144_kernel", 2: "conv48_tma_kernel", 1: "conv48_kernel"}.get(
        int(lib.bm3d_pilot_conv_kernel()), "none")
    flops_conv = len(SIGMAS) * W * H * 2 * 9 * 48 * 48
    if rank == 0:
        line = {
            "metric": "BM3D MP/s with the learned pilot in place of the basic estimate "
                      "(pilot + final, 4 x 1920x1080, sigma 5/10/25/50)",
            "value": round(mp / (ms_pilot / 1e3), 3), "unit": "MP/s", "n_gpus": 1,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(ms_pilot, 4),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "bf16 (pilot, FP32 accumulation) + f32 (final stage)",
            "data": "synthetic (seeded piecewise-smooth planes + Gaussian noise)",
            "config": {"workload": "learned pilot (8 x 3x3 conv, 48 ch, BF16 tensor cores) on the "
                                   "sweep's 4 planes, then their final Wiener stage as one "
                                   "final-stage-only batch fed by the pilot",
                       "train_crops": args.pilot_crops, "train_epochs": args.pilot_epochs,
                       "train_batch": 32, "data_s": round(t_data, 1),
                       "train_s": round(t_train, 1), "train_steps": len(hist),
                       "train_restarts": getattr(pilot, "restarts", 0),
                       "final_loss": hist[-1][1] if hist else None},
            "plain": {"value": round(mp / (ms_plain / 1e3), 3), "unit": "MP/s",
                      "ms_per_step": round(ms_plain, 4),
                      "basic_ms_per_launch": round(tb, 4), "final_ms_per_launch": round(tf, 4)},
            "pilot_over_plain": round(ms_plain / ms_pilot, 4),
            "pilot_network_ms_per_step": round(ms_cnn, 4),
            "pilot_final_ms_per_launch": round(tpf, 4),
            "ceiling": {"formula": "(T_basic + T_final) / (T_pilot + T_final), batch kernels",
                        "value": round((tb + tf) / (ms_cnn + tf), 4), "target": 2.0},
            "roofline": {"bound": "tensor", "kernel": conv_kernel,
                         "launch": "one 48 -> 48 layer over the step's four 1920x1080 planes "
                                   "(the six such layers are 98 % of the network's FLOPs)",
                         "per_launch_ms": round(ms_conv, 4),
                         "algorithmic_gflop_per_launch": round(flops_conv / 1e9, 2),
                         "achieved": round(flops_conv / (ms_conv / 1e3) / 1e12, 2),
                         "peak": bf16_peak, "unit": "TFLOP/s",
                         "frac": round(flops_conv / (ms_conv / 1e3) / 1e12 / bf16_peak, 4),
                         "peak_source": "MEASURED_PEAKS.json bf16_tflops (burst)",
                         "traffic": (PILOT_CONV_TRAFFIC_PER_PLANE[conv_kernel][0] * len(SIGMAS)
                                     if conv_kernel in PILOT_CONV_TRAFFIC_PER_PLANE else None),
                         "traffic_source": (f"4 x the one-plane capture "
                                            f"({PILOT_CONV_TRAFFIC_PER_PLANE[conv_kernel][1]})"
                                            if conv_kernel in PILOT_CONV_TRAFFIC_PER_PLANE
                                            else None),
                         "network_tflops": round(flops_cnn / (ms_cnn / 1e3) / 1e12, 2),
                         "layer_ms": [round(float(x), 4) for x in lay]},
            "psnr_vs_clean": psnr,
            "eval_1080p": evals,
            "gpu_launches": args.steps * (8 + 6),
            "clocks": clk.summary(m0, m1),
        }
        print(json.dumps(line), flush=True)
    pbatch.close()
    batch.close()
    pilot.close()
    ctx.close()


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=100)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-extras", action="store_true",
                    help="skip the batch64 / yuv4k16 figures the default run adds")
    ap.add_argument("--cpu-seconds", type=float, default=20.0)
    ap.add_argument("--pilot-crops", type=int, default=20000)
    ap.add_argument("--pilot-epochs", type=int, default=30)
    ap.add_argument("--pilot-checkpoint", default="",
                    help="pilot workload: load this checkpoint if it exists, else train and save")
    ap.add_argument("--workload", default="sweep1080",
                    choices=["sweep1080", "batch64", "yuv4k16", "pilot1080", "pilotyuv4k16"],
                    help="sweep1080: 4 x 1920x1080 sigma sweep (headline); batch64: 64 uneven "
                         "planes; yuv4k16: 16 3840x2160 YUV 4:4:4 frames, three planes each")
    args = ap.parse_args()
    if args.warmup < 3 and args.impl == "ours":
        args.warmup = 3
    if args.impl == "reference":
        run_reference(args)
    elif args.workload == "batch64":
        run_batch(args)
    elif args.workload == "yuv4k16":
        run_yuv(args)
    elif args.workload == "pilot1080":
        run_pilot(args)
    elif args.workload == "pilotyuv4k16":
        run_pilot_yuv(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
