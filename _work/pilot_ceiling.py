"""Ceiling of the learned-pilot pipeline, measured rather than estimated.

The pilot (8 layers of 3x3 convolutions, 48 channels, ReLU, BF16 with FP32
accumulation, input = noisy plane + noise-level map, residual output) would
replace only the basic estimate; the Wiener stage keeps its own block
matching and transforms. This times the pilot's convolution stack with
cuDNN (a library stand-in, channels-last BF16, best algorithm picked by
cuDNN's benchmark mode) at the given plane size and the plain basic and
final stages of this library on the same plane, and prints the pipeline
speed-up bound (T_basic + T_final) / (T_cnn + T_final). Weights are random:
only the time matters here.

    python -m isp_mw_b200.pilot_ceiling [--width 1920] [--height 1080] [--sigma 25]
"""
from __future__ import annotations

import argparse
import json


def time_ms(fn, reps: int = 50, warmup: int = 5) -> float:
    import torch
    for _ in range(warmup):
        fn()
    torch.cuda.synchronize()
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    a.record()
    for _ in range(reps):
        fn()
    b.record()
    torch.cuda.synchronize()
    return a.elapsed_time(b) / reps


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--width", type=int, default=1920)
    ap.add_argument("--height", type=int, default=1080)
    ap.add_argument("--sigma", type=float, default=25.0)
    ap.add_argument("--layers", type=int, default=8)
    ap.add_argument("--channels", type=int, default=48)
    args = ap.parse_args()

    import torch
    import isp_mw_b200
    from isp_mw_b200 import synth

    torch.backends.cudnn.benchmark = True
    dev = torch.device("cuda", 0)
    c, n = args.channels, args.layers
    chans = [2] + [c] * (n - 1) + [1]
    layers = []
    for i in range(n):
        conv = torch.nn.Conv2d(chans[i], chans[i + 1], 3, padding=1, bias=True)
        layers.append(conv)
        if i < n - 1:
            layers.append(torch.nn.ReLU(inplace=True))
    net = torch.nn.Sequential(*layers).to(dev, torch.bfloat16).to(memory_format=torch.channels_last)
    x = torch.randn(1, 2, args.height, args.width, device=dev, dtype=torch.bfloat16)
    x = x.to(memory_format=torch.channels_last)

    def pilot():
        with torch.no_grad():
            return x[:, :1] + net(x)  # residual output

    t_cnn = time_ms(pilot)
    flop = 2 * 9 * sum(chans[i] * chans[i + 1] for i in range(n)) * args.width * args.height

    _, noisy = synth.pair(args.height, args.width, args.sigma, 2024)
    sp = [synth.sigma_param(args.sigma)] * 3
    pb = isp_mw_b200.stage_params_default("fast", False, sp)
    pf = isp_mw_b200.stage_params_default("fast", True, sp)
    ctx = isp_mw_b200.Context(0)
    src = torch.from_numpy(noisy).to(dev)
    basic = torch.empty_like(src)
    out = torch.empty_like(src)
    t_basic = time_ms(lambda: ctx.stage(pb, False, basic, src))
    t_final = time_ms(lambda: ctx.stage(pf, True, out, src, basic))
    ctx.close()
    print(json.dumps({
        "plane": f"{args.width}x{args.height}", "sigma_255": args.sigma,
        "pilot": f"{n} layers 3x3, {c} channels, bf16 channels-last, cuDNN",
        "pilot_gflop": round(flop / 1e9, 1), "t_cnn_ms": round(t_cnn, 4),
        "pilot_tflops": round(flop / (t_cnn / 1e3) / 1e12, 1),
        "t_basic_ms": round(t_basic, 4), "t_final_ms": round(t_final, 4),
        "speedup_bound": round((t_basic + t_final) / (t_cnn + t_final), 3),
    }))


if __name__ == "__main__":
    main()
