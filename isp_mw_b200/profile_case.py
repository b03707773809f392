"""A fixed workload for profiler captures: warm-up launches, then `--launches`
launches of one BM3D stage on one seeded synthetic plane (device memory).

    python -m isp_mw_b200.profile_case --stage final --width 1920 --height 1080

With `--time`, the launches are timed with CUDA events instead (for the
profile tables): `--profile np --time` prints ms per launch of each stage.
With `--batch N`, N planes of the sigma sweep (5/10/25/50, cycled) go through
one batch (default tiling, no autotuning) and each launch is one eager run of
its pipeline (the persistent batch_stage_kernel launches the benchmark's graph
replays). With `--pilot`, each launch is the learned pilot on the plane
(conv_in, six tensor-core conv48 layers, conv_out).
"""
from __future__ import annotations

import argparse


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--stage", choices=["basic", "final"], default="final")
    ap.add_argument("--width", type=int, default=1920)
    ap.add_argument("--height", type=int, default=1080)
    ap.add_argument("--sigma", type=float, default=25.0)
    ap.add_argument("--warmup", type=int, default=2)
    ap.add_argument("--launches", type=int, default=2)
    ap.add_argument("--groups-only", action="store_true",
                    help="run the stage's block matching alone (bm3d_debug_groups)")
    ap.add_argument("--planes", type=int, choices=[1, 3], default=1,
                    help="3: Y/U/V planes (sigma 15/10/10) sharing luma groups (bm3d_stage3)")
    ap.add_argument("--profile", default="fast", choices=["fast", "lc", "np", "high", "vn"])
    ap.add_argument("--time", action="store_true",
                    help="time both stages (CUDA events, --launches each) and print ms and MP/s")
    ap.add_argument("--batch", type=int, default=0,
                    help="N > 0: one batch of N sweep planes, launches = eager pipeline runs")
    ap.add_argument("--pilot", action="store_true", help="launches = pilot estimates of the plane")
    args = ap.parse_args()
    if args.batch > 0:
        return batch_case(args)
    if args.pilot:
        return pilot_case(args)
    if args.time:
        return time_stages(args)
    if args.planes == 3:
        return three_planes(args)

    import torch
    import isp_mw_b200
    from isp_mw_b200 import synth

    _, noisy = synth.pair(args.height, args.width, args.sigma, 2024)
    sp = [synth.sigma_param(args.sigma)] * 3
    b = isp_mw_b200.stage_params_default(args.profile, False, sp)
    f = isp_mw_b200.stage_params_default(args.profile, True, sp)
    ctx = isp_mw_b200.Context(0)
    src = torch.from_numpy(noisy).cuda()
    basic = torch.empty_like(src)
    out = torch.empty_like(src)
    ctx.stage(b, False, basic, src)
    ref_plane = noisy if args.stage == "basic" else basic.cpu().numpy()
    for _ in range(args.warmup + args.launches):
        if args.groups_only:
            ctx.debug_groups(b if args.stage == "basic" else f, args.stage == "final", ref_plane)
        elif args.stage == "basic":
            ctx.stage(b, False, out, src)
        else:
            ctx.stage(f, True, out, src, basic)
    torch.cuda.synchronize()
    st = ctx.last_stats()
    print(f"stage={args.stage} {args.width}x{args.height} groups_sum_n={st[0]} candidates={st[2]}")
    ctx.close()


def time_stages(args):
    """Basic then final of the chosen profile on one seeded plane (or, with
    `--planes 3`, three Y/U/V planes at sigma 15/10/10 sharing luma groups),
    each timed over `--launches` launches after `--warmup`."""
    import json
    import torch
    import isp_mw_b200
    from isp_mw_b200 import synth

    ctx = isp_mw_b200.Context(0)
    if args.planes == 3:
        sig = (15.0, 10.0, 10.0)
        src = [torch.from_numpy(synth.pair(args.height, args.width, s, 50 + c)[1]).cuda()
               for c, s in enumerate(sig)]
        sp = [synth.sigma_param(s, c) for c, s in enumerate(sig)]
        basic = [torch.empty_like(p) for p in src]
        out = [torch.empty_like(p) for p in src]
        stage = ctx.stage3
    else:
        _, noisy = synth.pair(args.height, args.width, args.sigma, 2024)
        sp = [synth.sigma_param(args.sigma)] * 3
        src = torch.from_numpy(noisy).cuda()
        basic = torch.empty_like(src)
        out = torch.empty_like(src)
        stage = ctx.stage
    b = isp_mw_b200.stage_params_default(args.profile, False, sp)
    f = isp_mw_b200.stage_params_default(args.profile, True, sp)
    ms = {}
    for name, run in (("basic", lambda: stage(b, False, basic, src)),
                      ("final", lambda: stage(f, True, out, src, basic))):
        for _ in range(args.warmup):
            run()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(max(1, args.launches)):
            run()
        e1.record()
        torch.cuda.synchronize()
        ms[name] = e0.elapsed_time(e1) / max(1, args.launches)
    ctx.close()
    mp = args.width * args.height / 1e6
    print(json.dumps({"profile": args.profile, "plane": f"{args.width}x{args.height}",
                      "planes": args.planes,
                      "sigma_255": [15.0, 10.0, 10.0] if args.planes == 3 else args.sigma,
                      "basic_ms": round(ms["basic"], 4),
                      "final_ms": round(ms["final"], 4),
                      "mp_per_s": round(mp / ((ms["basic"] + ms["final"]) / 1e3), 1)}))


def three_planes(args):
    """Three seeded planes (sigma 15, 10, 10 on Y, U, V), one basic
    three-plane stage, then the requested stage `--launches + --warmup` times."""
    import torch
    import isp_mw_b200
    from isp_mw_b200 import synth

    sig = (15.0, 10.0, 10.0)
    planes = [torch.from_numpy(synth.pair(args.height, args.width, s, 7 + c)[1]).cuda()
              for c, s in enumerate(sig)]
    sp = [synth.sigma_param(s, c) for c, s in enumerate(sig)]
    b = isp_mw_b200.stage_params_default("fast", False, sp)
    f = isp_mw_b200.stage_params_default("fast", True, sp)
    ctx = isp_mw_b200.Context(0)
    basic = [p.clone() for p in planes]
    out = [p.clone() for p in planes]
    ctx.stage3(b, False, basic, planes)
    for _ in range(args.warmup + args.launches):
        if args.stage == "basic":
            ctx.stage3(b, False, out, planes)
        else:
            ctx.stage3(f, True, out, planes, basic)
    torch.cuda.synchronize()
    print(f"stage={args.stage} planes=3 {args.width}x{args.height}")
    ctx.close()



def batch_case(args):
    import torch
    import isp_mw_b200
    from isp_mw_b200 import synth
    sig = [(5.0, 10.0, 25.0, 50.0)[k % 4] for k in range(args.batch)]
    ctx = isp_mw_b200.Context(0)
    srcs, pbs, pfs = [], [], []
    for k, s in enumerate(sig):
        srcs.append(torch.from_numpy(synth.pair(args.height, args.width, s, 3000 + k)[1]).cuda())
        sp = [synth.sigma_param(s)] * 3
        pbs.append(isp_mw_b200.stage_params_default(args.profile, False, sp))
        pfs.append(isp_mw_b200.stage_params_default(args.profile, True, sp))
    dsts = [torch.empty_like(x) for x in srcs]
    batch = isp_mw_b200.Batch(ctx, pbs, pfs, dsts, srcs, autotune=False)
    times = [batch.stage_times() for _ in range(args.warmup + args.launches)]
    t = times[args.warmup:]
    print(f"batch of {args.batch} {args.width}x{args.height}: basic "
          f"{sum(x[0] for x in t) / len(t):.4f} ms, final {sum(x[1] for x in t) / len(t):.4f} ms "
          f"per persistent launch")
    if args.time:  # whole pipeline from its CUDA graph, 20 replays after the runs above
        ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        ev0.record()
        for _ in range(20):
            batch.run()
        ev1.record()
        torch.cuda.synchronize()
        print(f"graph replay: {ev0.elapsed_time(ev1) / 20:.4f} ms per run of the {args.batch} planes")
    batch.close()
    ctx.close()


def pilot_case(args):
    import torch
    import isp_mw_b200
    from isp_mw_b200 import synth
    _, noisy = synth.pair(args.height, args.width, args.sigma, 2024)
    ctx = isp_mw_b200.Context(0)
    p = isp_mw_b200.Pilot(ctx, seed=1)
    src = torch.from_numpy(noisy).cuda()
    out = torch.empty_like(src)
    for _ in range(args.warmup):
        p.estimate(out, src, args.sigma / 255.0)
    torch.cuda.synchronize()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    ev0.record()
    for _ in range(args.launches):
        p.estimate(out, src, args.sigma / 255.0)
    ev1.record()
    torch.cuda.synchronize()
    ms = ev0.elapsed_time(ev1) / max(1, args.launches)
    print(f"pilot {args.width}x{args.height}: {ms:.3f} ms per estimate (CUDA events)")
    p.close()
    ctx.close()


if __name__ == "__main__":
    main()
