#!/usr/bin/env python
"""TV-L1 frame pairs/s at 1024x436 on B200 (5 scales x 5 warps x <= 50 inner
iterations, lambda 0.15, tau 0.25, theta 0.3, epsilon 0.01).

One step = one batch of --batch synthetic pairs (seeded generator of the
1024x436 workload: textured noise, affine background, moving disc, N(0,2)
noise, uint8 frames) solved through the library.  Prints one JSON line on
rank 0.

  python bench.py [--gpus N --steps K --warmup W --batch P]
  python bench.py --impl reference ...   # the reference's sequential C++ TV-L1
                                         # (compiled in place) on the host cores

Under torchrun (N > 1) every rank solves its own batch (pairs are independent,
no data-path collective: weak scaling); the step time is the max over ranks.
"""
from __future__ import annotations

import argparse
import datetime
import json
import os
import subprocess
import sys
import tempfile
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
PKG = os.path.join(ROOT, "sycl-optic-flow_b200")
for _p in (ROOT, PKG):
    if _p not in sys.path:
        sys.path.insert(0, _p)

W, H = 1024, 436
METRIC = "TV-L1 pairs/s @1024x436: learned warm-start vs plain at equal EPE; HBM GB/s"
PARAMS = dict(nscales=5, max_iterations=50)  # other parameters: reference defaults
BYTES_PER_PX_ITER = 60  # read u1,u2,p11,p12,p21,p22,I1wx,I1wy,rho_c; write u1,u2,p x4


def log(*a):
    print(*a, file=sys.stderr, flush=True)


def make_pairs_seeds(seeds):
    from oflow import synth
    out = []
    for s in seeds:
        p = synth.tvl1_pair(seed=s, w=W, h=H)
        out.append((synth.quantize(p.I0), synth.quantize(p.I1), p))
    return out


def make_pairs(n, seed0):
    return make_pairs_seeds(range(seed0, seed0 + n))


def measured_peak():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(path) as f:
            v = json.load(f)["hbm_gbs"]
        return float(v), "measured"
    except Exception:
        return 6650.0, "fallback"


TRAFFIC_PROFILE = os.path.join(ROOT, "profiles", "k_tvl1_q_1024x436.md")


def ncu_traffic():
    """DRAM bytes per pair-iteration of the finest-scale inner iterations, from
    the committed ncu summary (a line 'traffic_bytes_per_pair_iteration: N'),
    or None."""
    try:
        for line in open(TRAFFIC_PROFILE):
            if line.startswith("traffic_bytes_per_pair_iteration:"):
                return float(line.split(":")[1].split()[0])
    except OSError:
        pass
    return None


class Clocks:
    """nvidia-smi sampled every 200 ms while the timed region runs."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu):
        self.gpu = gpu
        self.f = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
        self.p = None

    def __enter__(self):
        try:
            self.p = subprocess.Popen(["nvidia-smi", "-i", str(self.gpu), f"--query-gpu={self.Q}",
                                       "--format=csv,noheader,nounits", "-lms", "200"],
                                      stdout=self.f, stderr=subprocess.DEVNULL)
        except OSError:
            self.p = None
        return self

    def __exit__(self, *exc):
        if self.p:
            self.p.terminate()
            try:
                self.p.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.p.kill()

    def summary(self):
        try:
            rows = [r.split(",") for r in open(self.f.name).read().strip().splitlines()]
        except OSError:
            rows = []
        os.unlink(self.f.name)
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in rows:
            if len(r) < 9:
                continue
            try:
                sm.append(float(r[1]))
                mx = float(r[2])
            except ValueError:
                continue
            for n, v in zip(names, r[5:9]):
                if v.strip() == "Active":
                    reasons.add(n)
        sm.sort()
        return {"sm_mhz": sm[len(sm) // 2] if sm else None, "sm_max_mhz": mx,
                "reasons": sorted(reasons), "samples": len(sm)}


def algorithmic_bytes(stats_list, nx, ny):
    """Sum over pairs, scales, warps of n_{s,w} * px_s * 60 B (inner iterations)."""
    tot = 0
    for st in stats_list:
        its = st["iterations"]
        for s in range(its.shape[0]):
            tot += int(its[s].sum()) * nx[s] * ny[s] * BYTES_PER_PX_ITER
    return tot


def level_sizes(ns, w=W, h=H):
    nx, ny = [w], [h]
    for _ in range(1, ns):
        nx.append(int(float(nx[-1]) * 0.5 + 0.5))
        ny.append(int(float(ny[-1]) * 0.5 + 0.5))
    return nx, ny


# ------------------------------------------------------------- CPU baseline
BENCH_SEED0 = 10_000  # rank r solves seeds BENCH_SEED0 + r*P ... (multigpu.rank_seeds)


def cpu_model():
    try:
        for line in open("/proc/cpuinfo"):
            if line.startswith("model name"):
                return line.split(":", 1)[1].strip()
    except OSError:
        pass
    return None


def cpu_runner(threads):
    """(kind, run(a, b)) for the reference's sequential TV-L1 (oracle/_ref,
    OpenMP over `threads` threads) or, without it, the oracle port (one
    thread)."""
    import numpy as np
    import oracle
    prm = oracle.TVL1Params(**PARAMS)
    if oracle.ref_available():
        return "reference", threads, lambda a, b: oracle.ref_tvl1(a, b, prm)
    return "port", 1, lambda a, b: oracle.tvl1(a.astype(np.float32), b.astype(np.float32), prm)


def cpu_worker(args):
    """Runs in a subprocess (OMP_NUM_THREADS set by the parent): the CPU
    implementation on the benchmark's own pairs (seeds BENCH_SEED0, +1, ...,
    the pairs rank 0 of the GPU arm solves), one after another, up to
    --cpu-pairs pairs or --cpu-seconds of work."""
    threads = int(os.environ.get("OMP_NUM_THREADS", "1"))
    kind, cores, run = cpu_runner(threads)
    pairs = make_pairs(min(args.cpu_pairs, args.batch), BENCH_SEED0)
    run(*pairs[0][:2])  # warm-up
    n, t0 = 0, time.perf_counter()
    times = []
    while n < args.cpu_pairs and (time.perf_counter() - t0) < args.cpu_seconds:
        a, b, _ = pairs[n % len(pairs)]
        t = time.perf_counter()
        run(a, b)
        times.append(time.perf_counter() - t)
        n += 1
    el = time.perf_counter() - t0
    print(json.dumps({"value": n / el, "unit": "pairs/s", "cores": cores, "kind": kind,
                      "sample": f"{n} pairs of the 1024x436 workload (generator seeds "
                                f"{BENCH_SEED0}..{BENCH_SEED0 + min(n, len(pairs)) - 1}, the "
                                f"GPU arm's first pairs), {el:.1f} s, median "
                                f"{1e3 * sorted(times)[len(times) // 2]:.0f} ms/pair"}))


def cpu_baseline(pairs=30, seconds=20.0, threads=None, batch=32):
    threads = threads or os.cpu_count() or 1
    env = dict(os.environ, OMP_NUM_THREADS=str(threads))
    cmd = [sys.executable, os.path.abspath(__file__), "--cpu-worker", "--cpu-pairs", str(pairs),
           "--cpu-seconds", str(seconds), "--batch", str(batch)]
    out = subprocess.run(cmd, env=env, capture_output=True, text=True, timeout=600)
    if out.returncode != 0:
        log(out.stderr[-2000:])
        return None
    return json.loads(out.stdout.strip().splitlines()[-1])


# ------------------------------------------------------------- reference arm
def reference_arm(args, rank):
    """The reference's sequential TV-L1 on all host threads.  Step k solves
    the benchmark pair k mod --batch (seeds BENCH_SEED0 ...): the same pairs,
    in the same order, that rank 0 of the GPU arm solves in every step."""
    if rank != 0:
        return 0
    threads = os.cpu_count() or 1
    os.environ["OMP_NUM_THREADS"] = str(threads)
    kind, threads, run = cpu_runner(threads)
    n_pairs = min(args.batch, max(args.steps, args.warmup, 1))
    pairs = make_pairs(n_pairs, BENCH_SEED0)
    for k in range(args.warmup):
        run(*pairs[k % n_pairs][:2])
    t0 = time.perf_counter()
    for k in range(args.steps):
        run(*pairs[k % n_pairs][:2])
    el = time.perf_counter() - t0
    v = args.steps / el
    sample = (f"{args.steps} pairs, one per step: generator seeds {BENCH_SEED0}.."
              f"{BENCH_SEED0 + min(args.steps, n_pairs) - 1} (the GPU arm's pairs)")
    line = {
        "impl": "reference", "metric": METRIC, "value": v, "unit": "pairs/s", "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * el / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic",
        "config": {"workload": "tvl1 1024x436, 5 scales x 5 warps x <=50 inner iterations, "
                               "1 uint8 pair per step", "solver": "reference sequential C++ "
                               "(src/tvl1/sequential, OpenMP)",
                   "pairs": f"seeds {BENCH_SEED0}+k mod {args.batch}, as the GPU arm"},
        "cpu_baseline": {"value": v, "unit": "pairs/s", "cores": threads, "kind": kind,
                         "sample": sample, "cpu_model": cpu_model()},
        "e2e": {"value": v, "unit": "pairs/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


# ------------------------------------------------------------- our arm
WARM_SCHEDULES = [
    # (name, warps per scale, iterations per scale), index 0 = finest scale
    ("2x20 uniform", [2, 2, 2, 2], [20, 20, 20, 20]),
    ("3x30 uniform", [3, 3, 3, 3], [30, 30, 30, 30]),
    ("finest 3x40, coarser 1x10", [3, 1, 1, 1], [40, 10, 10, 10]),
    ("finest 2x50, coarser 1x10", [2, 1, 1, 1], [50, 10, 10, 10]),
    ("finest 4x50, scale 1 2x20, coarser 1x10", [4, 2, 1, 1], [50, 20, 10, 10]),
    ("finest 5x50, coarser 1x10", [5, 1, 1, 1], [50, 10, 10, 10]),
    ("finest 5x50, scale 1 2x30, coarser 1x20", [5, 2, 1, 1], [50, 30, 20, 20]),
]


def warm_measure(oflow, synth, np, torch, pairs, d_in, prm, ctx, stream, args, P, world,
                 max_over_ranks, barrier, t_plain=None, schedules=None):
    """Warm-started TV-L1 on the same pairs: the network's flow initialises
    scale 3, then a per-scale schedule of warps x inner iterations.  Timed
    like the plain form; quality from one judged call (plain solve as judge:
    energy within 1 % and end-point difference from the plain flow within 1 %
    of its magnitude) and EPE against ground truth for both forms.  The
    judged throughput judges a sampled eighth of the pairs each step (the
    plain solve of those pairs runs beside the warm batch)."""
    from oflow import warmstart
    if not os.path.exists(warmstart.WEIGHTS):
        return None
    params, meta = warmstart.load()
    net = oflow.WarmNet(W, H, P, ctx)
    net.set_params(params)
    dev = d_in[0][0].device
    w_out = [(torch.empty((H, W), dtype=torch.float32, device=dev),
              torch.empty((H, W), dtype=torch.float32, device=dev)) for _ in range(P)]
    p_out = oflow.tvl1_batch(d_in, prm, ctx)
    epe_p = [synth.epe(p_out[i][0].cpu().numpy(), p_out[i][1].cpu().numpy(), pairs[i][2].u,
                       pairs[i][2].v, pairs[i][2].valid, 8) for i in range(P)]
    sample = d_in[::8]
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)

    def timed(fn):
        for _ in range(args.warmup):
            fn()
        torch.cuda.synchronize()
        barrier()
        e0.record(stream)
        for _ in range(args.steps):
            fn()
        e1.record(stream)
        torch.cuda.synchronize()
        return max_over_ranks(e0.elapsed_time(e1) / 1e3)

    rows = []
    if schedules is None:
        schedules = [("%dx%d uniform" % (args.warm_warps, args.warm_iters), [args.warm_warps] * 4,
                      [args.warm_iters] * 4)]
    for name, ws, its in schedules:
        wprm = oflow.TVL1Params(nscales=5, warps=max(ws), max_iterations=max(its))
        run = lambda: oflow.tvl1_warm(d_in, net, wprm, None, ctx, out=w_out, warps_per_scale=ws,
                                      iters_per_scale=its)
        t = timed(run)
        epe_w = [synth.epe(w_out[i][0].cpu().numpy(), w_out[i][1].cpu().numpy(), pairs[i][2].u,
                           pairs[i][2].v, pairs[i][2].valid, 8) for i in range(P)]
        t_j = timed(lambda: (run(), oflow.tvl1_batch(sample, prm, ctx)))
        _, info = oflow.tvl1_warm(d_in, net, wprm, prm, ctx, warps_per_scale=ws,
                                  iters_per_scale=its)
        ratio = info["energy_warm"] / info["energy_plain"]
        acc_e = ratio <= 1.01
        acc_x = info["epe_vs_plain"] <= 0.01
        row = {"schedule": name, "warps_per_scale": ws, "iters_per_scale": its,
               "value": world * P * args.steps / t, "unit": "pairs/s",
               "judged_sampled_value": world * P * args.steps / t_j,
               "accepted_fraction": float(np.mean(info["accepted"])),
               "accepted_energy_only": float(np.mean(acc_e)),
               "accepted_epe_only": float(np.mean(acc_x)),
               "energy_ratio_median": float(np.median(ratio)),
               "energy_ratio_max": float(ratio.max()),
               "epe_vs_plain_median": float(np.median(info["epe_vs_plain"])),
               "epe_warm": float(np.mean(epe_w)), "epe_plain": float(np.mean(epe_p)),
               "epe_rel_diff": float((np.mean(epe_w) - np.mean(epe_p)) / np.mean(epe_p))}
        if t_plain:
            row["speedup_vs_plain"] = row["value"] / t_plain
            row["judged_speedup_vs_plain"] = row["judged_sampled_value"] / t_plain
        rows.append(row)
    out = dict(rows[0])
    # one training step of the network (batch 16, the library's own forward
    # and backward kernels, Adam), timed over 10 steps
    tnet = oflow.WarmNet(W, H, 16, ctx)
    tnet.set_params(params)
    fr = torch.stack([torch.stack([d_in[i % P][0], d_in[i % P][1]]) for i in range(16)])
    tg = torch.zeros((16, tnet.out_h, tnet.out_w, 2), dtype=torch.float32, device=dev)
    for _ in range(3):
        tnet.train_step(fr, tg, 1e-6)
    torch.cuda.synchronize()
    t0 = time.time()
    for _ in range(10):
        tnet.train_step(fr, tg, 1e-6)
    torch.cuda.synchronize()
    out["training_step_ms"] = (time.time() - t0) * 100.0
    out["training_step_config"] = ("batch 16 pairs of 1024x436, forward + backward + Adam, "
                                   "host-timed per synchronous step")
    out["judge"] = ("plain 5x5x50 solve; energy <= 1.01 x plain and sum|warm-plain| <= 0.01 x "
                    "sum|plain|; judged throughput samples every 8th pair")
    out["training"] = meta
    if len(rows) > 1:
        out["frontier"] = rows
    return out


def solver_measure(oflow, synth, np, torch, ctx, stream, dev, peak):
    """Horn-Schunck on its 320x240 configuration (alpha 15, one level, one
    warp, 200 Jacobi sweeps; 64 pairs per call) and pyramidal Lucas-Kanade on
    its 640x480 configuration (3 levels x 3 refinements, 5x5 window; one pair
    per call), device-resident, with EPE against the generators' ground truth.
    Algorithmic bytes: HS 28 B/px per sweep plus 24 B/px for the warp and
    derivatives; pyramidal LK 24 B/px per level-refinement."""
    out = {}
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)

    def timed(fn, reps):
        for _ in range(3):
            fn()
        torch.cuda.synchronize()
        e0.record(stream)
        for _ in range(reps):
            fn()
        e1.record(stream)
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) / 1e3 / reps

    hp = oflow.HSParams(15.0, 1, 1, 200)
    gen = [synth.hs_pair(seed=40_000 + i) for i in range(64)]
    hs_in = [(torch.from_numpy(g.I0).to(dev), torch.from_numpy(g.I1).to(dev)) for g in gen]
    hs_out = [(torch.empty((240, 320), device=dev), torch.empty((240, 320), device=dev)) for _ in gen]
    t_fixed = timed(lambda: oflow.hs_batch(hs_in, hp, ctx, out=hs_out), 10)
    hs_cfg = oflow.hs_autotune(hs_in, hp, ctx)
    t = timed(lambda: oflow.hs_batch(hs_in, hp, ctx, out=hs_out), 10)
    per_pair = 320 * 240 * (200 * 28 + 24)
    epe = float(np.mean([synth.epe(o[0].cpu().numpy(), o[1].cpu().numpy(), g.u, g.v, g.valid, 8)
                         for o, g in zip(hs_out[:8], gen[:8])]))
    out["hs_320x240"] = {"pairs_per_s": 64 / t, "mpixels_per_s": 64 * 320 * 240 / t / 1e6,
                         "achieved_gbs": 64 * per_pair / t / 1e9,
                         "frac": 64 * per_pair / t / 1e9 / peak, "epe_vs_ground_truth": round(epe, 4),
                         "jacobi_config_per_level": hs_cfg,
                         "pairs_per_s_untuned": 64 / t_fixed,
                         "config": "alpha 15, 1 level, 1 warp, 200 sweeps, 64 pairs per call, autotuned"}
    lp = oflow.LKParams(3, 2, 5, 3, 3)
    g = synth.lk_pair(seed=41_000)
    a, b = torch.from_numpy(g.I0).to(dev), torch.from_numpy(g.I1).to(dev)
    lo = (torch.empty((480, 640), device=dev), torch.empty((480, 640), device=dev))
    t = timed(lambda: oflow.pyrlk(a, b, lp, ctx, out=lo), 50)
    per_pair = 3 * (640 * 480 + 320 * 240 + 160 * 120) * 24
    epe = synth.epe(lo[0].cpu().numpy(), lo[1].cpu().numpy(), g.u, g.v, g.valid, 8)
    out["pyrlk_640x480"] = {"pairs_per_s": 1 / t, "mpixels_per_s": 640 * 480 / t / 1e6,
                            "achieved_gbs": per_pair / t / 1e9,
                            "frac": per_pair / t / 1e9 / peak, "epe_vs_ground_truth": round(float(epe), 4),
                            "config": "3 levels x 3 refinements, 5x5 window, one pair per call"}
    # the same configuration, 64 pairs per call (oflow_pyrlk_batch)
    nb = 64
    gl = [synth.lk_pair(seed=41_000 + i) for i in range(nb)]
    lk_in = [(torch.from_numpy(q.I0).to(dev), torch.from_numpy(q.I1).to(dev)) for q in gl]
    lk_out = [(torch.empty((480, 640), device=dev), torch.empty((480, 640), device=dev)) for _ in gl]
    t = timed(lambda: oflow.pyrlk_batch(lk_in, lp, ctx, out=lk_out), 10)
    epe = float(np.mean([synth.epe(o[0].cpu().numpy(), o[1].cpu().numpy(), q.u, q.v, q.valid, 8)
                         for o, q in zip(lk_out[:8], gl[:8])]))
    out["pyrlk_640x480_batch"] = {"pairs_per_s": nb / t, "mpixels_per_s": nb * 640 * 480 / t / 1e6,
                                  "achieved_gbs": nb * per_pair / t / 1e9,
                                  "frac": nb * per_pair / t / 1e9 / peak,
                                  "epe_vs_ground_truth": round(epe, 4),
                                  "config": "3 levels x 3 refinements, 5x5 window, 64 pairs per call"}
    return out


def our_arm(args, rank, world, local_rank):
    import numpy as np
    import torch
    import torch.distributed as dist

    import oflow
    from oflow import multigpu, synth

    torch.cuda.set_device(local_rank)
    if world > 1:
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=180),
                                device_id=torch.device("cuda", local_rank))
    dev = torch.device("cuda", local_rank)
    P = args.batch
    log(f"[rank {rank}] generating {P} pairs ...")
    seeds = multigpu.rank_seeds(rank, world, P, base=BENCH_SEED0)
    pairs = make_pairs_seeds(seeds)
    prm = oflow.TVL1Params(**PARAMS)
    ctx = oflow.Context(local_rank)
    stream = torch.cuda.current_stream(dev)
    ctx.set_stream(stream.cuda_stream)

    d_in = [(torch.from_numpy(a).to(dev), torch.from_numpy(b).to(dev)) for a, b, _ in pairs]
    d_out = [(torch.empty((H, W), dtype=torch.float32, device=dev),
              torch.empty((H, W), dtype=torch.float32, device=dev)) for _ in range(P)]

    def barrier():
        if world > 1:
            dist.barrier()

    def max_over_ranks(x):
        return multigpu.max_over_ranks(x, dev)

    # --- tile shapes per scale from the autotuner (before warm-up, untimed)
    tuned = oflow.tvl1_autotune(d_in, prm, ctx) if not args.no_autotune else None
    # --- device-resident inputs (value)
    for _ in range(args.warmup):
        oflow.tvl1_batch(d_in, prm, ctx, out=d_out)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with Clocks(local_rank) as clk:
        barrier()
        torch.cuda.synchronize()
        e0.record(stream)
        for _ in range(args.steps):
            oflow.tvl1_batch(d_in, prm, ctx, out=d_out)
        e1.record(stream)
        torch.cuda.synchronize()
        barrier()
    t_dev = max_over_ranks(e0.elapsed_time(e1) / 1e3)
    clocks = clk.summary()

    # --- quality of the timed results, and the per-kernel profile
    (res, stats, prof) = oflow.tvl1_batch_profile(d_in, prm, ctx, out=d_out)
    torch.cuda.synchronize()
    u0 = d_out[0][0].cpu().numpy()
    v0 = d_out[0][1].cpu().numpy()
    g = pairs[0][2]
    epe = synth.epe(u0, v0, g.u, g.v, g.valid, 8)
    nx, ny = level_sizes(stats[0]["nscales"])
    alg_iter = algorithmic_bytes(stats, nx, ny)
    # dominant kernel: the blocked inner iterations at the finest scale
    alg0 = sum(int(s["iterations"][0].sum()) for s in stats) * nx[0] * ny[0] * BYTES_PER_PX_ITER
    ms0 = prof["iter_ms_scale"][0]
    iters_total = int(sum(int(s["iterations"].sum()) for s in stats))
    peak, peak_kind = measured_peak()
    achieved = alg0 / (ms0 / 1e3) / 1e9 if ms0 > 0 else None
    # the dominant launch: the persistent stage of the finest scale's first
    # warp (all pairs' iterations of that stage); its DRAM traffic from the
    # per-pair-iteration figure of the committed capture
    it00 = sum(int(s["iterations"][0][0]) for s in stats)
    traffic = ncu_traffic()
    if traffic is not None:
        traffic *= it00
    # the graph replays' launch count (inner iterations run as device-ended
    # while-loops, so it depends on the data); the timed steps replay the same
    # pairs, so each step launched the same kernels
    oflow.tvl1_batch(d_in, prm, ctx, out=d_out)
    launches_per_step = ctx.last_launches()

    # --- end to end through the public API: pinned host frames in, flow out
    h_in = []
    for a, b, _ in pairs:
        ta = torch.from_numpy(a).pin_memory()
        tb = torch.from_numpy(b).pin_memory()
        h_in.append((ta.numpy(), tb.numpy()))
    h_out = [(torch.empty((H, W), dtype=torch.float32).pin_memory().numpy(),
              torch.empty((H, W), dtype=torch.float32).pin_memory().numpy()) for _ in range(P)]
    for _ in range(max(1, args.warmup // 2)):
        oflow.tvl1_batch(h_in, prm, ctx, out=h_out)
    barrier()
    torch.cuda.synchronize()
    e0.record(stream)
    e2e_steps = max(3, args.steps // 2)
    for _ in range(e2e_steps):
        oflow.tvl1_batch(h_in, prm, ctx, out=h_out)
    e1.record(stream)
    torch.cuda.synchronize()
    barrier()
    t_e2e = max_over_ranks(e0.elapsed_time(e1) / 1e3)
    assert np.array_equal(h_out[0][0], u0), "end-to-end result differs from the device run"

    # --- learned warm start (scale 3 from the network, 2 warps x 20 iterations)
    warm = None
    if not args.no_warm:
        warm = warm_measure(oflow, synth, np, torch, pairs, d_in, prm, ctx, stream, args, P,
                            world, max_over_ranks, barrier, t_plain=world * P * args.steps / t_dev,
                            schedules=WARM_SCHEDULES if args.warm_frontier else None)

    # --- flowToColor of the step's flows (device in, device out); the argument
    # arrays are built once so that the loop times the C call and the kernel
    import ctypes
    from oflow.capi import BgrImage, Flow, lib as oflow_lib
    imgs = [torch.empty((H, W, 3), dtype=torch.uint8, device=dev) for _ in range(P)]
    first = oflow.flow_to_color_batch(d_out, ctx, out=imgs)
    fl = (Flow * P)(*[Flow(ctypes.cast(ctypes.c_void_p(u.data_ptr()), ctypes.POINTER(ctypes.c_float)),
                           ctypes.cast(ctypes.c_void_p(v.data_ptr()), ctypes.POINTER(ctypes.c_float)),
                           W, 1) for u, v in d_out])
    im = (BgrImage * P)(*[BgrImage(t.data_ptr(), 3 * W, 1) for t in imgs])
    for _ in range(3):
        oflow_lib().oflow_flow_to_color(ctx.handle, P, W, H, fl, im)
    torch.cuda.synchronize()
    reps = 50
    e0.record(stream)
    for _ in range(reps):
        oflow_lib().oflow_flow_to_color(ctx.handle, P, W, H, fl, im)
    e1.record(stream)
    torch.cuda.synchronize()
    t_col = e0.elapsed_time(e1) / 1e3 / reps
    col_gbs = P * W * H * 11 / t_col / 1e9
    assert first[0].shape == (H, W, 3)
    color = {"flows_per_s": P / t_col, "ms_per_batch": 1e3 * t_col, "achieved_gbs": col_gbs,
             "frac": col_gbs / measured_peak()[0],
             "bytes_basis": "8 B in (u, v) + 3 B out (B, G, R) per pixel", "batch": P}

    # --- the other two solvers on their configurations (device-resident)
    solvers = solver_measure(oflow, synth, np, torch, ctx, stream, dev, measured_peak()[0])

    # --- the mixed batch workload (256 pairs, HS and TV-L1, five sizes)
    mixed = None
    if not args.no_mixed:
        mixed = batch_measure(ctx, dev, stream, args.mixed_steps, 3, args.batch_pairs, rank,
                              max_over_ranks, barrier, measured_peak()[0])
        mixed["value"] *= world
        mixed["e2e"]["value"] *= world

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cpu = cpu_baseline(args.cpu_pairs, args.cpu_seconds, batch=P)
        if cpu:
            one = cpu_baseline(8, args.cpu_seconds / 2, threads=1, batch=P)
            cpu["cpu_model"] = cpu_model()
            cpu["single_thread"] = one and {"value": one["value"], "unit": one["unit"],
                                            "cores": 1, "sample": one["sample"]}

    if world > 1:
        dist.destroy_process_group()
    if rank != 0:
        return 0
    value = world * P * args.steps / t_dev
    line = {
        "metric": METRIC, "value": value, "unit": "pairs/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * t_dev / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic",
        "config": {"workload": f"tvl1 1024x436, 5 scales x 5 warps x <=50 inner iterations, "
                               f"{P} uint8 pairs per GPU per step (plain TV-L1)",
                   "batch_pairs_per_gpu": P, "parallelism": f"independent pairs x{world}",
                   "l2": f"inputs larger than L2 (finest-level u, p, warp data and coefficients "
                         f"~{P * W * H * 136 / 1e9:.1f} GB)",
                   "inner_iterations_per_step": iters_total,
                   "tile_config_per_scale": tuned,
                   "epe_vs_ground_truth": round(epe, 5)},
        "e2e": {"value": world * P * e2e_steps / t_e2e, "unit": "pairs/s",
                "h2d_bytes_per_step": P * 2 * W * H, "d2h_bytes_per_step": P * 2 * W * H * 4},
        "gpu_launches": args.steps * launches_per_step,
        # frame-pair pixels solved per second (whole job), the Mpixel/s form of value
        "mpixels_per_s": value * W * H / 1e6,
        "roofline": {"bound": "hbm", "kernel": "k_tvl1_q (inner iterations, finest scale)",
                     "achieved": achieved, "peak": peak, "unit": "GB/s",
                     "frac": (achieved / peak) if achieved else None,
                     "traffic": traffic, "peak_source": peak_kind,
                     "bytes_basis": "algorithmic 60 B/px per inner iteration; traffic = DRAM "
                                    "bytes of the finest scale's first-warp stage launch (ncu "
                                    "bytes per pair-iteration x that stage's iterations)",
                     "traffic_algorithmic_same_launch": it00 * nx[0] * ny[0] * BYTES_PER_PX_ITER,
                     "finest_scale_ms": round(ms0, 3),
                     "all_scales_achieved": alg_iter / (prof["iter_ms"] / 1e3) / 1e9
                     if prof["iter_ms"] > 0 else None,
                     "iter_share_of_step": prof["iter_ms"] / prof["total_ms"]
                     if prof["total_ms"] else None,
                     "iter_ms_per_scale": [round(x, 3) for x in
                                           prof["iter_ms_scale"][:stats[0]["nscales"]]],
                     "profile_total_ms": round(prof["total_ms"], 3),
                     "warp_ms": round(prof["warp_ms"], 3)},
        "clocks": clocks,
    }
    if cpu:
        line["cpu_baseline"] = cpu
    if warm:
        warm["speedup_vs_plain"] = warm["value"] / value
        line["warm_start"] = warm
    line["flow_to_color"] = color
    line["solvers"] = solvers
    if mixed:
        line["mixed_batch"] = dict(mixed, metric=METRIC_BATCH)
    print(json.dumps(line), flush=True)
    return 0


def once_other(args):
    """Profiling cases of the other kernels (--once-solver): hs: --batch pairs
    of the 320x240 HS configuration (alpha 15, 200 sweeps); pyrlk: --batch
    pairs of the 640x480 pyramidal LK configuration; color: flowToColor of
    --batch 1024x436 flows; conv: the warm-start network's forward pass on
    --batch 1024x436 pairs; train: one training step of the network (forward,
    backward, Adam) on --batch pairs, after two untimed ones."""
    import numpy as np
    import torch
    import oflow
    from oflow import synth
    dev = torch.device("cuda", 0)
    ctx = oflow.Context(0)
    n = args.batch
    if args.once_solver == "hs":
        gen = [synth.hs_pair(seed=40_000 + i) for i in range(n)]
        d = [(torch.from_numpy(g.I0).to(dev), torch.from_numpy(g.I1).to(dev)) for g in gen]
        oflow.hs_batch(d, oflow.HSParams(15.0, 1, 1, 200), ctx)
    elif args.once_solver == "pyrlk":
        gen = [synth.lk_pair(seed=41_000 + i) for i in range(n)]
        d = [(torch.from_numpy(g.I0).to(dev), torch.from_numpy(g.I1).to(dev)) for g in gen]
        oflow.pyrlk_batch(d, oflow.LKParams(3, 2, 5, 3, 3), ctx)
    elif args.once_solver == "color":
        rng = np.random.default_rng(5)
        flows = [(torch.from_numpy(rng.normal(0, 4, (H, W)).astype(np.float32)).to(dev),
                  torch.from_numpy(rng.normal(0, 4, (H, W)).astype(np.float32)).to(dev))
                 for _ in range(n)]
        oflow.flow_to_color_batch(flows, ctx)
    else:
        from oflow import warmstart
        params, _ = warmstart.load()
        net = oflow.WarmNet(W, H, n, ctx)
        net.set_params(params)
        pairs = make_pairs(n, 0)
        fr = torch.from_numpy(np.stack([np.stack([a, b]) for a, b, _ in pairs])).to(dev)
        if args.once_solver == "conv":
            net.predict(fr)
        else:
            tg = torch.zeros((n, net.out_h, net.out_w, 2), dtype=torch.float32, device=dev)
            for _ in range(3):
                net.train_step(fr, tg, 1e-6)
    torch.cuda.synchronize()
    log("done:", args.once_solver, n)
    return 0


def once(args):
    """Profiling case: one solve of --batch pairs with --nscales / --iters."""
    if args.once_solver != "tvl1":
        return once_other(args)
    import torch
    import oflow
    pairs = make_pairs(args.batch, 0)
    dev = torch.device("cuda", 0)
    d_in = [(torch.from_numpy(a).to(dev), torch.from_numpy(b).to(dev)) for a, b, _ in pairs]
    prm = oflow.TVL1Params(nscales=args.nscales, max_iterations=args.iters)
    ctx = oflow.Context(0)
    if args.tuning:
        # the bench's tile choice without the autotuner's launches: tune and
        # save when the table is missing, else load it
        if os.path.exists(args.tuning):
            ctx.load_tuning(args.tuning)
        else:
            oflow.tvl1_autotune(d_in, prm, ctx)
            ctx.save_tuning(args.tuning)
    res, st = oflow.tvl1_batch(d_in, prm, ctx, stats=True)
    torch.cuda.synchronize()
    log("iterations per pair:", [int(s["iterations"].sum()) for s in st])
    return 0


METRIC_BATCH = "mixed batch pairs/s: 256 pairs, half HS half TV-L1, 5 sizes up to 1920x1080"
HS_SWEEP_BYTES = 28  # per px per Jacobi sweep: read du, dv, Ix, Iy, Iz; write du, dv
HS_WARP_BYTES = 24   # per px per warp: warp + derivatives
TV_WARP_BYTES = 32   # per px per warp stage: warp of I1, I1x, I1y + rho_c / grad
TV_LEVEL_BYTES = 40  # per px per level: pyramid, gradients, zoom of the flow


def batch_measure(ctx, dev, stream, steps, warmup, n_pairs, seed, max_over_ranks, barrier,
                  peak):
    """The batched uneven workload: n_pairs pairs with sizes uniform over
    {320x240, 640x480, 1024x436, 1280x720, 1920x1080}, half Horn-Schunck
    (alpha 15, 200 sweeps) and half TV-L1 (5 scales x 5 warps x <= 50),
    solved as one oflow_batch schedule (one graph, a branch per group).
    Returns the measurement: pairs/s device-resident and end to end, and the
    whole step's algorithmic bytes against the HBM peak."""
    import torch
    import oflow
    from oflow import synth, synth_gpu

    specs = synth.batch_specs(n_pairs, seed=seed)
    tp = oflow.TVL1Params(nscales=5, max_iterations=50)
    hp = oflow.HSParams(15.0, 1, 1, 200)
    groups = {}
    for i, (solver, w, h, _) in enumerate(specs):
        groups.setdefault((solver, w, h), []).append(i)
    frames = [None] * len(specs)
    for (solver, w, h), idx in groups.items():
        gen = synth_gpu.tvl1_pairs if solver == "tvl1" else synth_gpu.hs_pairs
        a, b, *_ = gen(len(idx), w, h, seed=(seed * 7919 + w * 31 + h) & 0xffff, device=dev)
        for k, i in enumerate(idx):
            frames[i] = (a[k].contiguous(), b[k].contiguous())
    jobs = [(solver, frames[i][0], frames[i][1], tp if solver == "tvl1" else hp)
            for i, (solver, w, h, _) in enumerate(specs)]
    outs = [(torch.empty((h, w), dtype=torch.float32, device=dev),
             torch.empty((h, w), dtype=torch.float32, device=dev)) for (_, w, h, _) in specs]
    # tile shapes per group (untimed), and the TV-L1 iteration counts that
    # set the algorithmic bytes (same kernels and inputs as the timed batch)
    alg = 0
    for (solver, w, h), idx in groups.items():
        grp = [frames[i] for i in idx]
        if solver == "tvl1":
            oflow.tvl1_autotune(grp, tp, ctx)
            _, st = oflow.tvl1_batch(grp, tp, ctx, stats=True)
            nx, ny = level_sizes(st[0]["nscales"], w, h)
            for sti in st:
                its = sti["iterations"]
                for sc in range(its.shape[0]):
                    px = nx[sc] * ny[sc]
                    alg += px * (int(its[sc].sum()) * BYTES_PER_PX_ITER
                                 + its.shape[1] * TV_WARP_BYTES + TV_LEVEL_BYTES)
        else:
            oflow.hs_autotune(grp, hp, ctx)
            alg += len(idx) * w * h * (hp.nsolver * HS_SWEEP_BYTES + HS_WARP_BYTES)
    for _ in range(warmup):
        oflow.batch(jobs, ctx, out=outs)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    barrier()
    e0.record(stream)
    for _ in range(steps):
        oflow.batch(jobs, ctx, out=outs)
    e1.record(stream)
    torch.cuda.synchronize()
    t = max_over_ranks(e0.elapsed_time(e1) / 1e3)
    # end to end: pinned host frames in, host flows out
    h_jobs = [(s_, f0.cpu().pin_memory().numpy(), f1.cpu().pin_memory().numpy(), p_)
              for (s_, f0, f1, p_) in jobs]
    h_outs = [(torch.empty(o[0].shape).pin_memory().numpy(),
               torch.empty(o[0].shape).pin_memory().numpy()) for o in outs]
    oflow.batch(h_jobs, ctx, out=h_outs)
    torch.cuda.synchronize()
    barrier()
    e0.record(stream)
    e2e_steps = max(2, steps // 2)
    for _ in range(e2e_steps):
        oflow.batch(h_jobs, ctx, out=h_outs)
    e1.record(stream)
    torch.cuda.synchronize()
    t_e2e = max_over_ranks(e0.elapsed_time(e1) / 1e3)
    n = len(specs)
    px = sum(w * h for (_, w, h, _) in specs)
    ach = alg * steps / t / 1e9
    return {"value": n * steps / t, "unit": "pairs/s", "ms_per_step": 1e3 * t / steps,
            "mpixels_per_s": px * steps / t / 1e6,
            "steps": steps,
            "config": {"workload": "mixed batch (HS alpha 15, 1 level, 1 warp, 200 sweeps; "
                                   "TV-L1 5 scales x 5 warps x <=50)",
                       "pairs": n, "groups": len(groups), "megapixels_per_step": px / 1e6,
                       "tvl1_pairs": sum(1 for sp in specs if sp[0] == "tvl1"),
                       "l2": "inputs larger than L2"},
            "e2e": {"value": n * e2e_steps / t_e2e, "unit": "pairs/s",
                    "h2d_bytes_per_step": sum(f0.nbytes + f1.nbytes for (_, f0, f1, _) in h_jobs),
                    "d2h_bytes_per_step": 2 * 4 * px},
            "roofline": {"bound": "hbm", "achieved": ach, "peak": peak, "unit": "GB/s",
                         "frac": ach / peak, "algorithmic_bytes_per_step": alg,
                         "bytes_basis": "whole step: TV-L1 per px 60 B x inner iterations + "
                                        "32 B per warp stage + 40 B per level; HS per px "
                                        "28 B x sweeps + 24 B per warp"}}


def batch_arm(args, rank, world, local_rank):
    """--workload batch: the mixed workload alone, as its own JSON line."""
    import torch
    import torch.distributed as dist
    import oflow
    from oflow import multigpu

    torch.cuda.set_device(local_rank)
    if world > 1:
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=180),
                                device_id=torch.device("cuda", local_rank))
    dev = torch.device("cuda", local_rank)
    ctx = oflow.Context(local_rank)
    stream = torch.cuda.current_stream(dev)
    ctx.set_stream(stream.cuda_stream)
    with Clocks(local_rank) as clk:
        m = batch_measure(ctx, dev, stream, args.steps, args.warmup, args.batch_pairs, rank,
                          lambda x: multigpu.max_over_ranks(x, dev),
                          (lambda: dist.barrier()) if world > 1 else (lambda: None),
                          measured_peak()[0])
    if world > 1:
        dist.destroy_process_group()
    if rank != 0:
        return 0
    line = {"metric": METRIC_BATCH, "value": world * m["value"], "unit": "pairs/s",
            "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": m["ms_per_step"], "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic", "config": m["config"],
            "e2e": dict(m["e2e"], value=world * m["e2e"]["value"]),
            "roofline": m["roofline"], "clocks": clk.summary()}
    print(json.dumps(line), flush=True)
    return 0


def main():
    ap = argparse.ArgumentParser(description=__doc__.split("\n")[0])
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--batch", type=int, default=32, help="pairs per GPU per step")
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-autotune", action="store_true")
    ap.add_argument("--no-warm", action="store_true", help="skip the warm-start measurement")
    ap.add_argument("--warm-warps", type=int, default=2)
    ap.add_argument("--warm-iters", type=int, default=20)
    ap.add_argument("--warm-frontier", action="store_true",
                    help="time and judge every schedule of WARM_SCHEDULES")
    ap.add_argument("--workload", choices=["tvl1", "batch"], default="tvl1",
                    help="tvl1: the 1024x436 TV-L1 workload (default); batch: the 256-pair "
                         "mixed HS/TV-L1 workload")
    ap.add_argument("--batch-pairs", type=int, default=256)
    ap.add_argument("--no-mixed", action="store_true",
                    help="skip the mixed batch workload in the default run")
    ap.add_argument("--mixed-steps", type=int, default=5,
                    help="timed steps of the mixed batch workload in the default run")
    ap.add_argument("--cpu-pairs", type=int, default=30)
    ap.add_argument("--cpu-seconds", type=float, default=20.0)
    ap.add_argument("--cpu-worker", action="store_true", help=argparse.SUPPRESS)
    ap.add_argument("--once", action="store_true",
                    help="one solve of --batch device-resident pairs and exit (profiling case)")
    ap.add_argument("--once-solver", choices=["tvl1", "hs", "pyrlk", "color", "conv", "train"],
                    default="tvl1", help="kernel family of the --once profiling case")
    ap.add_argument("--nscales", type=int, default=PARAMS["nscales"])
    ap.add_argument("--iters", type=int, default=PARAMS["max_iterations"])
    ap.add_argument("--tuning", default=None,
                    help="with --once: tuning table to load (autotuned and saved if missing)")
    args = ap.parse_args()
    if args.cpu_worker:
        return cpu_worker(args)
    if args.warmup < 3 and args.impl == "ours":
        log("warm-up raised to 3 steps")
        args.warmup = 3
    rank = int(os.environ.get("RANK", 0))
    world = int(os.environ.get("WORLD_SIZE", 1))
    local_rank = int(os.environ.get("LOCAL_RANK", 0))
    if args.impl == "reference":
        return reference_arm(args, rank)
    if args.once:
        return once(args)
    if args.workload == "batch":
        return batch_arm(args, rank, world, local_rank)
    return our_arm(args, rank, world, local_rank)


if __name__ == "__main__":
    sys.exit(main() or 0)
