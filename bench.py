#!/usr/bin/env python
"""Benchmark of the B200 SGM stereo path.

Workload (default): the batched mixed-size workload - 64 seeded synthetic
rectified pairs, resolution drawn from {320x240, 640x480, 1242x375, 1280x720},
D from {64, 128, 192}, 8 paths, 5x5 census, P1=10, P2=120, subpixel, LR check
(tolerance 1). One step = one batched pass (census, all 8 paths of all pairs,
WTA + LR) over the 64 pairs with the images already in device memory.

Metric: Gpixel-disparities/s (sum of W*H*D over pairs / seconds), whole job.
Also reported: the plain per-pair path on the same pairs (one synchronous
compute_disparity call per pair, like the reference) with p50/p99 latency per
pair, the end-to-end rate through the C ABI with host buffers (H2D of the
images and D2H of the disparity maps inside the timed region), the served
path (continuous batching of Poisson arrivals of mixed requests under the 40 GB
device budget, at a moderate rate and past saturation, and past saturation
again under 80 GB), the roofline of the aggregation kernel, and the CPU oracle
on a bounded sample.

Multi-GPU (torchrun): replicas only - every rank runs its own 64 pairs
(different seeds), no data-path collective; value = all ranks' pixel-
disparities / the slowest rank's time.

--impl reference: the reference algorithm on the host cores (the CPU
restatement in oracle/, since the reference's Metal GPU path cannot run here),
same metric and workload, each step a bounded sample of the pairs.
"""
import argparse
import json
import os
import sys
import time

import numpy as np

REPO = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(REPO, "vx-rs_b200"))

METRIC = "SGM Gpixel-disparities/s (batched, mixed sizes, 8 paths)"
UNIT = "Gpd/s"
SIZES = [(320, 240), (640, 480), (1242, 375), (1280, 720)]
DISPARITIES = [64, 128, 192]
NUM_PAIRS = 64


def workload(rank: int, name: str = "mixed"):
    """(w, h, D, seed) tuples; seeds differ per rank (replicas). "mixed" is the 64-pair
    mixed-size workload; "profile" is a small case for profiler captures (2 pairs of
    1242x375, D=128: 1.9 GB of path slabs, larger than L2) and "profile-mix" a
    medium one that fills the GPU with all three D (32 pairs of 320x240);
    "profile-many" has enough aggregation units (3840) to keep every warp of a
    three-warpgroup launch busy in a small memory footprint."""
    if name == "profile":
        return [(1242, 375, 128, 1_000_003 * (rank + 1) + i) for i in range(2)]
    if name == "profile-mix":  # 32 pairs of 320x240, D cycling 64/128/192: 5 GB of slabs
        return [(320, 240, DISPARITIES[i % 3], 1_000_003 * (rank + 1) + i) for i in range(32)]
    if name == "profile-wide":  # 8 pairs of 1280x720, D=64: few border (x < D) pixels
        return [(1280, 720, 64, 1_000_003 * (rank + 1) + i) for i in range(8)]
    if name == "profile-hd":  # 2 pairs of 1280x720, D=192: a 354 MB cost volume (> L2), 3.6 GB with --sync
        return [(1280, 720, 192, 1_000_003 * (rank + 1) + i) for i in range(2)]
    if name == "profile-many":  # 128 pairs of 160x120, D cycling 64/128/192: 3840 aggregation units, 2.5 GB
        return [(160, 120, DISPARITIES[i % 3], 1_000_003 * (rank + 1) + i) for i in range(128)]
    rng = np.random.default_rng(20261203 + 7919 * rank)
    items = []
    for i in range(NUM_PAIRS):
        w, h = SIZES[int(rng.integers(len(SIZES)))]
        d = int(DISPARITIES[int(rng.integers(len(DISPARITIES)))])
        items.append((w, h, d, 1_000_003 * (rank + 1) + i))
    return items


def sgm_config(vx_sgm, d):
    return vx_sgm.SGMStereoConfig(num_disparities=d, p1=10.0, p2=120.0, census_radius_x=2,
                                  census_radius_y=2, num_paths=8, subpixel=True, lr_check=True,
                                  lr_tolerance=1, invalid_value=-1.0)


def make_pairs(vx_sgm, items):
    pairs = []
    for (w, h, d, seed) in items:
        L, R, _ = vx_sgm.synth_pair(vx_sgm.SCENE_PLANES, w, h, 4, int(0.9 * d), seed)
        pairs.append((L, R))
    return pairs


class ClockSampler:
    """SM clock, power and clock-event (throttle) reasons of the bench's GPU, read
    through NVML every 10 ms on a background thread while the timed region runs
    (plus one reading at its start and one at its end). Read-only."""

    REASONS = {0x8: "hw_slowdown", 0x40: "hw_thermal_slowdown", 0x20: "sw_thermal_slowdown",
               0x4: "sw_power_cap"}

    def __init__(self, device: int):
        self.device = device
        self.rows = []
        self.err = None
        self.stop = None

    def _handle(self, nv):
        try:
            import torch
            uuid = str(torch.cuda.get_device_properties(self.device).uuid)
            return nv.nvmlDeviceGetHandleByUUID(uuid if uuid.startswith("GPU-") else "GPU-" + uuid)
        except Exception:
            return nv.nvmlDeviceGetHandleByIndex(self.device)

    def _sample(self):
        nv, h = self.nv, self.h
        reasons = nv.nvmlDeviceGetCurrentClocksEventReasons(h)
        self.rows.append((float(nv.nvmlDeviceGetClockInfo(h, nv.NVML_CLOCK_SM)),
                          float(nv.nvmlDeviceGetMaxClockInfo(h, nv.NVML_CLOCK_SM)),
                          nv.nvmlDeviceGetPowerUsage(h) / 1000.0, int(reasons)))

    def __enter__(self):
        import threading
        try:
            import pynvml as nv
            nv.nvmlInit()
            self.nv, self.h = nv, self._handle(nv)
            self._sample()
        except Exception as e:  # no NVML: report it instead of clocks
            self.err = f"nvml unavailable: {type(e).__name__}"
            return self
        self.stop = threading.Event()

        def loop():
            while not self.stop.wait(0.01):
                try:
                    self._sample()
                except Exception:
                    pass
        self.thread = threading.Thread(target=loop, daemon=True)
        self.thread.start()
        return self

    def __exit__(self, *exc):
        if self.stop is not None:
            self.stop.set()
            self.thread.join(timeout=5)
            try:
                self._sample()
            except Exception:
                pass

    def summary(self):
        if self.err or not self.rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": [self.err or "no samples"]}
        reasons = sorted({name for r in self.rows for bit, name in self.REASONS.items() if r[3] & bit})
        return {"sm_mhz": float(np.median([r[0] for r in self.rows])),
                "sm_max_mhz": max(r[1] for r in self.rows),
                "power_w_max": max(r[2] for r in self.rows),
                "samples": len(self.rows), "source": "nvml", "reasons": reasons}


def oracle_config(oracle, d):
    return oracle.config(num_disparities=d, p1=10, p2=120, census_radius_x=2, census_radius_y=2,
                         num_paths=8, subpixel=True, lr_check=True)


def strata(items):
    """Indices of the workload's pairs grouped by (W, H, D): pairs of one stratum are the
    same amount of work (seeded scenes of one generator)."""
    groups = {}
    for i, (w, h, d, _) in enumerate(items):
        groups.setdefault((w, h, d), []).append(i)
    return groups


def cpu_stratified(items, get_pair, threads, rounds, first_round=0, keep_outputs=False):
    """The oracle (CPU restatement of the reference algorithm) on a size-stratified
    sample of the workload: round r runs the r-th pair (cycling) of every (W, H, D)
    stratum. The whole workload's CPU time is estimated as the sum over strata of
    (pairs in the stratum) x (mean time of its sampled pairs), so the rate refers to
    the same 64-pair workload as the GPU numbers. Returns (rate Gpd/s, sampled pairs,
    sampled pd, sampled seconds, {index: oracle outputs} when keep_outputs)."""
    sys.path.insert(0, os.path.join(REPO, "oracle"))
    import oracle
    groups = strata(items)
    times = {k: [] for k in groups}
    outputs = {}
    n = pd = 0
    secs = 0.0
    for r in range(first_round, first_round + rounds):
        for key, idx in groups.items():
            i = idx[r % len(idx)]
            w, h, d, _ = items[i]
            L, R = get_pair(i)
            t0 = time.perf_counter()
            out = oracle.sgm(L, R, oracle_config(oracle, d), nthreads=threads)
            dt = time.perf_counter() - t0
            times[key].append(dt)
            secs += dt
            n += 1
            pd += w * h * d
            if keep_outputs:
                outputs[i] = out
    est = sum(len(groups[k]) * float(np.mean(v)) for k, v in times.items())
    total_pd = sum(w * h * d for (w, h, d, _) in items)
    return total_pd / est / 1e9, n, pd, secs, outputs


def stratified_sample_text(items, n, pd, secs, threads):
    return (f"{n} pairs: one of each of the {len(strata(items))} (W, H, D) strata of the {len(items)}-pair "
            f"workload per round ({pd / 1e6:.0f} M pd, {secs:.1f} s, oracle on {threads} threads); "
            f"workload time = sum over strata of pairs x the stratum's sampled time")


def barrier(dist):
    """All ranks meet (no-op on one process)."""
    if dist is not None:
        dist.barrier()


def max_over_ranks(dist, v, device="cuda"):
    """The largest of every rank's value (the job's time is its slowest rank's)."""
    if dist is None:
        return v
    import torch
    t = torch.tensor([v], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def sum_over_ranks(dist, v, device="cuda"):
    """The sum of every rank's value (each replica's pairs differ, and so does its work)."""
    if dist is None:
        return v
    import torch
    t = torch.tensor([v], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.SUM)
    return float(t.item())


def job_rate(job_pd, ms_per_step):
    """Whole-job Gpd/s: all ranks' pixel-disparities of a step over the slowest rank's step time."""
    return job_pd / (ms_per_step * 1e-3) / 1e9


# DRAM bytes (read + write) per path-pixel-disparity of one aggregation launch in
# the scanline-pair form with three warpgroups a CTA (the shape the autotuner
# picks for the 64-pair batch), measured on a small case of the same workload
# and scaled by path-pd: the first 8 pairs of the mixed workload (3.741 G
# path-pd, 3.74 GB of byte slabs), the autotuner's two three-warpgroup launches
# (the 5th and 6th aggregation launches) of
#   VX_SGM_AGG_FORM=pairs ncu --metrics dram__bytes_read.sum,dram__bytes_write.sum,
#       gpu__time_duration.sum --clock-control none -k regex:aggregate_kernel
#       python bench.py --workload mixed --pairs 8 --kernels-only --steps 2 --warmup 3
# read 2.520 / 2.462 GB (cost-volume reads that missed L2) + write 3.703 GB
# (slabs and escaped vectors' shadow) = 6.19 GB a launch. One warpgroup a CTA
# moves 5.84 GB (fewer pairs in flight share L2 better); the 1280x720 D=192
# pair case moves 0.77 of its algorithmic bytes, as here (0.83).
AGG_DRAM_BYTES_PER_PATH_PD = (0.5 * (2.520e9 + 2.462e9) + 3.703e9) / 3740620800
AGG_TRAFFIC_SAMPLE = ("first 8 pairs of the mixed workload (3.741 G path-pd), the autotuner's "
                      "three-warpgroup scanline-pair launches: ncu dram__bytes_read.sum 2.49 GB + "
                      "dram__bytes_write.sum 3.70 GB per launch, scaled by path-pd")

FORM_NAMES = {64: "scanline pairs, 64-scanline units", 32: "single scanline, 32-scanline units",
              1: "across-lanes scan, one lane segment a scanline"}

# Device bytes the server may hold for in-flight requests: the served workload's
# 40 GB admission cap. A served batch lasts at least as long as its longest scanline
# chain (a 1920-wide D = 192 request: ~10 ms), so the budget sets how many requests
# share that time; the saturated point is also measured with SERVE_BUDGET_LARGE
# (batches of ~21 requests instead of ~13) and reported apart.
SERVE_BUDGET = 40 << 30
SERVE_BUDGET_LARGE = 80 << 30


SERVED_KEYS = ("rate_per_s", "requests", "completed", "latency_ms_p50", "latency_ms_p99",
               "throughput_gpd_s", "achieved_rate_per_s", "mean_batch", "max_batches_in_flight")


def served(vx_sgm, ctx, sgm, rates, max_batch=32, slots=2, budget=SERVE_BUDGET):
    """Served SGM: open-loop Poisson arrivals, mixed sizes and D, `budget` device bytes.
    rates: (requests per second, number of requests) per point; a fresh server per
    point so that each point's counters are its own."""
    import loadgen
    reqs = loadgen.make_requests(48)
    out = []
    for r, num_requests in rates:
        srv = vx_sgm.Server(sgm, ctx, memory_budget_bytes=budget, max_batch=max_batch,
                            max_inflight_batches=slots)
        loadgen.run_poisson(srv, reqs, 100.0, 16)  # warm the pool and the planner
        before = srv.stats()
        res = loadgen.run_poisson(srv, reqs, r, num_requests)
        after = srv.stats()
        srv.close()
        res["server"] = after
        batches = after["batches"] - before["batches"]
        res["mean_batch"] = (after["completed"] - before["completed"]) / batches if batches else None
        res["max_batches_in_flight"] = after["max_batches_in_flight"]
        res["max_batch"], res["slots"], res["budget_bytes"] = max_batch, slots, budget
        out.append(res)
    return out


def run_serve_sweep(args, local_rank):
    import vx_sgm
    ctx = vx_sgm.Context(local_rank)
    sgm = vx_sgm.SGMStereo(ctx)
    rates = [float(x) for x in args.serve_sweep.split(",") if x]
    for res in served(vx_sgm, ctx, sgm, [(r, args.serve_requests) for r in rates], args.serve_max_batch,
                      args.serve_slots, int(args.serve_budget_gb * (1 << 30))):
        print(json.dumps({"metric": "served SGM", "unit": UNIT,
                          "workload": "Poisson arrivals, sizes {640x480,1242x375,1280x720,1920x1080} "
                                      "x D{64,128,192}, 8 paths", **res}), flush=True)


# The single-pair and high-resolution configurations of the metric (besides the
# 64-pair batch): (name, pairs, w, h, D, paths, scene, d_lo, d_hi, description).
CONFIG_TABLE = [
    ("c0", 1, 640, 480, 64, 4, "planes", 4, 60, "640x480 D=64, 4 paths, LR tol 1, 5x5 census"),
    ("c1", 1, 1242, 375, 128, 8, "slanted", 0, 120, "1242x375 D=128, 8 paths, subpixel, LR, 5x5 census"),
    ("c3", 16, 2048, 1536, 256, 8, "surface", 0, 230,
     "16 x 2048x1536 D=256, 8 paths, planes + sinusoid + 10% textureless, staged batches"),
]


def run_config_table(args, local_rank):
    """One JSON line per configuration: the plain per-pair path (one synchronous call per
    pair, device-resident images, CUDA events; p50/p99 over repeats), the batched path
    for the multi-pair configuration, and the CPU oracle on one pair of it."""
    import torch

    import vx_sgm
    sys.path.insert(0, os.path.join(REPO, "oracle"))
    import oracle
    torch.cuda.set_device(local_rank)
    ctx = vx_sgm.Context(local_rank)
    sgm = vx_sgm.SGMStereo(ctx)
    stream = torch.cuda.ExternalStream(ctx.stream)
    scenes = {"planes": vx_sgm.SCENE_PLANES, "slanted": vx_sgm.SCENE_SLANTED, "surface": vx_sgm.SCENE_SURFACE}
    threads = os.cpu_count() or 1
    for (name, n, w, h, d, paths, scene, lo, hi, desc) in CONFIG_TABLE:
        cfg = vx_sgm.SGMStereoConfig(num_disparities=d, p1=10.0, p2=120.0, census_radius_x=2,
                                     census_radius_y=2, num_paths=paths, subpixel=True,
                                     lr_check=True, lr_tolerance=1, invalid_value=-1.0)
        pairs = [vx_sgm.synth_pair(scenes[scene], w, h, lo, hi, 4242 + i)[:2] for i in range(n)]
        tl = [ctx.texture_gray8(L, w, h) for L, _ in pairs]
        tr = [ctx.texture_gray8(R, w, h) for _, R in pairs]
        of = [ctx.texture_output_r32float(w, h) for _ in pairs]
        oi = [ctx.texture_output_i16(w, h) for _ in pairs]
        pd = w * h * d
        # plain: one synchronous call per pair (the reference's call pattern)
        reps = max(3, 40 // n)
        for i in range(min(n, 3)):
            sgm.compute_disparity(ctx, tl[i], tr[i], of[i], cfg, output_i16=oi[i])
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        lat = []
        for r in range(reps):
            i = r % n
            e0.record(stream)
            sgm.compute_disparity(ctx, tl[i], tr[i], of[i], cfg, output_i16=oi[i])
            e1.record(stream)
            e1.synchronize()
            lat.append(e0.elapsed_time(e1))
        line = {"config": name, "workload": desc, "pairs": n, "pd_per_pair": pd,
                "plain": {"value": pd / (float(np.mean(lat)) * 1e-3) / 1e9, "unit": UNIT,
                          "latency_ms_p50": float(np.percentile(lat, 50)),
                          "latency_ms_p99": float(np.percentile(lat, 99)), "calls": reps}}
        if n > 1:
            cfgs = [cfg] * n

            def timed_batches(stream_arg, steps=3):
                for _ in range(2):
                    sgm.compute_batch(ctx, tl, tr, of, cfgs, outputs_i16=oi, stream=stream_arg)
                ctx.synchronize()
                e0.record(stream)
                for _ in range(steps):
                    sgm.compute_batch(ctx, tl, tr, of, cfgs, outputs_i16=oi, stream=stream_arg)
                e1.record(stream)
                e1.synchronize()
                return e0.elapsed_time(e1) / steps

            # Synchronous batch calls keep escaped path vectors in a 1/16 shadow pool
            # (a third of the workspace), so the 16 pairs fit fewer sub-batches;
            # asynchronous ones (on a stream) reserve the full shadow.
            ms = timed_batches(None)
            ms_async = timed_batches(ctx.stream)
            line["batched"] = {"value": n * pd / (ms * 1e-3) / 1e9, "unit": UNIT, "ms_per_step": ms,
                               "call": "synchronous compute_batch (shadow pool, sub-batches under the "
                                       "workspace limit)",
                               "workspace_per_pair_bytes_full_shadow": vx_sgm.workspace_bytes(w, h, cfg)}
            line["batched_async"] = {"value": n * pd / (ms_async * 1e-3) / 1e9, "unit": UNIT,
                                     "ms_per_step": ms_async,
                                     "call": "compute_batch on a stream (full shadow, staged sub-batches)"}
        ocfg = oracle.config(num_disparities=d, p1=10, p2=120, census_radius_x=2, census_radius_y=2,
                             num_paths=paths, subpixel=True, lr_check=True)
        t0 = time.perf_counter()
        oracle.sgm(pairs[0][0], pairs[0][1], ocfg, nthreads=threads)
        secs = time.perf_counter() - t0
        line["cpu_baseline"] = {"value": pd / secs / 1e9, "unit": UNIT, "cores": threads, "kind": "port",
                                "sample": f"one pair ({pd / 1e6:.1f} M pd, {secs:.2f} s)"}
        print(json.dumps(line), flush=True)
        del tl, tr, of, oi

    # Post-filters of the depth chain (DepthFilter) on a 1920x1080 disparity map
    # (25 % invalid = -1): per-call device time over 50 calls, and bytes moved
    # per pixel (4 read + 4 written) against the HBM peak.
    w, h = 1920, 1080
    rng = np.random.default_rng(5)
    d = (rng.random((h, w)) * 120).astype(np.float32)
    d[rng.random((h, w)) < 0.25] = -1.0
    tin = ctx.texture_r32float(d, w, h)
    tout = ctx.texture_output_r32float(w, h)
    filt = vx_sgm.DepthFilter(ctx)
    peak = float(json.load(open(os.path.join(REPO, "MEASURED_PEAKS.json")))["hbm_gbs"]) \
        if os.path.exists(os.path.join(REPO, "MEASURED_PEAKS.json")) else 6650.0
    for name, run in (("median r=1", lambda: filt.apply_median(ctx, tin, tout, vx_sgm.DepthMedianConfig(1),
                                                               stream=ctx.stream)),
                      ("median r=2", lambda: filt.apply_median(ctx, tin, tout, vx_sgm.DepthMedianConfig(2),
                                                               stream=ctx.stream)),
                      ("bilateral r=3", lambda: filt.apply_bilateral(ctx, tin, tout, vx_sgm.DepthFilterConfig(),
                                                                     stream=ctx.stream))):
        for _ in range(5):
            run()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(50):
            run()
        e1.record(stream)
        e1.synchronize()
        ms = e0.elapsed_time(e1) / 50
        gbs = 8 * w * h / (ms * 1e-3) / 1e9
        print(json.dumps({"config": "post-filter", "filter": name, "map": f"{w}x{h} f32, 25% invalid",
                          "ms_per_call": ms, "gpx_per_s": w * h / (ms * 1e-3) / 1e9,
                          "hbm_gbs": gbs, "hbm_frac": gbs / peak}), flush=True)
    filt.close()

    # The depth chain's ends: RGBA -> gray ingest (5 bytes a pixel) and depth map ->
    # point cloud (4 bytes a pixel read, 36 bytes a point written), 1920x1080,
    # 50 back-to-back calls each (the device-buffer form for the cloud).
    rgba = rng.integers(0, 256, (h, w, 4), dtype=np.uint8)
    tin, tgray = ctx.texture_rgba8(rgba, w, h), ctx.texture_output_gray8(w, h)
    conv = vx_sgm.ColorConvert(ctx)
    depth = rng.uniform(0.0, 13.3, (h, w)).astype(np.float32)     # ~75 % inside [0.1, 10]
    tdep = ctx.texture_r32float(depth, w, h)
    d2c = vx_sgm.DepthToCloud(ctx)
    cfg = vx_sgm.DepthToCloudConfig()
    pts = torch.empty(w * h * 9, dtype=torch.int32, device=torch.device("cuda", local_rank))
    cnt = torch.zeros(1, dtype=torch.int32, device=torch.device("cuda", local_rank))
    for name, run, nbytes in (
            ("rgba_to_gray", lambda: conv.rgba_to_gray(ctx, tin, tgray, stream=ctx.stream), lambda: 5 * w * h),
            ("depth_to_cloud", lambda: d2c.compute_device(ctx, tdep, None, 1000.0, 1000.0, 960.0, 540.0, cfg,
                                                          pts.data_ptr(), w * h, cnt.data_ptr(), stream=ctx.stream),
             lambda: 4 * w * h + 36 * int(cnt.item()))):
        for _ in range(5):
            run()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(50):
            run()
        e1.record(stream)
        e1.synchronize()
        ms = e0.elapsed_time(e1) / 50
        gbs = nbytes() / (ms * 1e-3) / 1e9
        print(json.dumps({"config": "depth-chain", "kernel": name, "image": f"{w}x{h}", "ms_per_call": ms,
                          "gpx_per_s": w * h / (ms * 1e-3) / 1e9, "hbm_gbs": gbs, "hbm_frac": gbs / peak,
                          **({"points": int(cnt.item())} if name == "depth_to_cloud" else {})}), flush=True)
    d2c.close()


# Sparse ORB stereo matching (StereoMatcher): the reference example's size
# (examples/orb_stereo_benchmark.rs: <= 512 keypoints per side, EuRoC
# intrinsics), a SLAM front end's 2048, and 16384 per side as a throughput case.
STEREO_WORKLOADS = [
    ("euroc-512", 512, 512, dict(fx=458.654, fy=457.296, cx=367.215, cy=248.375, baseline=0.110),
     "512 x 512 ORB keypoints, 752x480 frame, EuRoC intrinsics (the reference example's configuration)"),
    ("slam-2048", 2048, 2048, {}, "2048 x 2048 ORB keypoints, 752x480 frame, StereoConfig::default"),
    ("dense-16384", 16384, 16384, {}, "16384 x 16384 ORB keypoints, 752x480 frame, StereoConfig::default"),
]


def run_stereo_match(args, local_rank):
    """One JSON line per workload: keypoint pairs (n_left x n_right, the
    reference's distance-matrix size) per second through the host-buffer entry
    point (end to end, host copies inside), through the device-buffer entry
    point (kernels only, CUDA events), and on the CPU (the oracle on every host
    thread; the reference shader compiled as C++, one thread, where built)."""
    import torch

    import vx_sgm
    sys.path.insert(0, os.path.join(REPO, "oracle"))
    import oracle
    torch.cuda.set_device(local_rank)
    ctx = vx_sgm.Context(local_rank)
    matcher = vx_sgm.StereoMatcher(ctx)
    stream = torch.cuda.ExternalStream(ctx.stream)
    threads = os.cpu_count() or 1
    dev = torch.device("cuda", local_rank)
    for (name, nl, nr, cfgd, desc) in STEREO_WORKLOADS:
        if args.stereo_only and name != args.stereo_only:
            continue
        lk, rk, ld, rd = vx_sgm.synth_orb_stereo(nl, nr, 9000 + nl)
        cfg = vx_sgm.StereoConfig(**cfgd)
        pairs = nl * nr
        # end to end: the reference's call (host slices in, Vec of matches out)
        for _ in range(args.warmup):
            n_match = len(matcher.run(ctx, lk, rk, ld, rd, cfg).matches)
        lat = []
        for _ in range(max(args.steps, 50)):
            t0 = time.perf_counter()
            matcher.run(ctx, lk, rk, ld, rd, cfg)
            lat.append(time.perf_counter() - t0)
        # device resident: the kernels alone
        t_lk = torch.from_numpy(lk.view(np.float32).reshape(-1, 4).copy()).to(dev)
        t_rk = torch.from_numpy(rk.view(np.float32).reshape(-1, 4).copy()).to(dev)
        t_ld = torch.from_numpy(ld["desc"].view(np.int32).copy()).to(dev)
        t_rd = torch.from_numpy(rd["desc"].view(np.int32).copy()).to(dev)
        t_out = torch.empty((nl, 7), dtype=torch.int32, device=dev)
        t_cnt = torch.empty((1,), dtype=torch.int32, device=dev)
        torch.cuda.synchronize()

        def call():
            matcher.run_device(ctx, t_lk.data_ptr(), nl, t_rk.data_ptr(), nr, t_ld.data_ptr(), t_rd.data_ptr(),
                               cfg, t_out.data_ptr(), t_cnt.data_ptr(), stream=ctx.stream)

        def time_device(form):
            if form:
                os.environ["VX_STEREO_FORM"] = form
            try:
                for _ in range(args.warmup):
                    call()
                reps = max(args.steps, 200)
                launches0 = vx_sgm.kernel_launch_count()
                e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                e0.record(stream)
                for _ in range(reps):
                    call()
                e1.record(stream)
                e1.synchronize()
                assert int(t_cnt.item()) == n_match
                return e0.elapsed_time(e1) / reps, (vx_sgm.kernel_launch_count() - launches0) / reps
            finally:
                os.environ.pop("VX_STEREO_FORM", None)
        # the form the library picks: banded from 2^24 pairs (0 <= max_epipolar < 2^20)
        form = "banded" if pairs >= (1 << 24) and 0.0 <= cfg.max_epipolar < 2.0 ** 20 else "brute"
        dev_ms, launches = time_device(None)
        other = "brute" if form == "banded" else "banded"
        other_ms, _ = time_device(other)
        # CPU: the oracle on every host thread (median of 3), the reference shader on one
        secs = []
        for _ in range(3):
            t0 = time.perf_counter()
            oracle.stereo_match(lk, rk, ld["desc"], rd["desc"], dict(oracle.STEREO_DEFAULTS, **cfgd),
                                nthreads=threads)
            secs.append(time.perf_counter() - t0)
        cpu = pairs / float(np.median(secs)) / 1e9
        line = {"config": "stereo-match", "workload": name, "desc": desc, "n_left": nl, "n_right": nr,
                "matches": n_match, "metric": "keypoint pairs/s", "unit": "G pairs/s",
                "form": form,
                "device": {"value": pairs / (dev_ms * 1e-3) / 1e9, "ms_per_call": dev_ms,
                           "gpu_launches_per_call": launches},
                f"device_{other}": {"value": pairs / (other_ms * 1e-3) / 1e9, "ms_per_call": other_ms},
                "e2e": {"value": pairs / float(np.mean(lat)) / 1e9, "latency_ms_p50": 1e3 * float(np.percentile(lat, 50)),
                        "latency_ms_p99": 1e3 * float(np.percentile(lat, 99)),
                        "h2d_bytes_per_call": 48 * (nl + nr), "d2h_bytes_per_call": 16 + 28 * nl},
                "cpu_baseline": {"value": cpu, "unit": "G pairs/s", "cores": threads, "kind": "port",
                                 "sample": f"the whole workload, median of 3 ({float(np.median(secs)) * 1e3:.2f} ms)"},
                "inputs": "device-resident and L2-sized (48 B per keypoint); the kernels are issue- or launch-bound"}
        if oracle.ref_stereo_available() and pairs <= 2048 * 2048:
            t0 = time.perf_counter()
            oracle.ref_stereo_match(lk, rk, ld["desc"], rd["desc"], dict(oracle.STEREO_DEFAULTS, **cfgd))
            rs = time.perf_counter() - t0
            line["cpu_reference"] = {"value": pairs / rs / 1e9, "unit": "G pairs/s", "cores": 1,
                                     "kind": "reference", "sample": f"the whole workload once ({rs * 1e3:.1f} ms)"}
        print(json.dumps(line), flush=True)

    # Frames: 64 frames of the example's size in one launch, against 64 calls.
    if not args.stereo_only or args.stereo_only == "frames-64x512":
        nf, n = 64, 512
        cfg = vx_sgm.StereoConfig(**STEREO_WORKLOADS[0][3])
        frames = [vx_sgm.synth_orb_stereo(n, n, 5000 + i) for i in range(nf)]
        lo = np.arange(nf + 1, dtype=np.uint32) * n
        ro = lo.copy()
        cat = lambda i: np.concatenate([f[i] for f in frames])  # noqa: E731
        lk, rk, ld, rd = cat(0), cat(1), cat(2), cat(3)
        t_lk = torch.from_numpy(lk.view(np.float32).reshape(-1, 4).copy()).to(dev)
        t_rk = torch.from_numpy(rk.view(np.float32).reshape(-1, 4).copy()).to(dev)
        t_ld = torch.from_numpy(ld["desc"].view(np.int32).copy()).to(dev)
        t_rd = torch.from_numpy(rd["desc"].view(np.int32).copy()).to(dev)
        t_out = torch.empty((nf * n, 7), dtype=torch.int32, device=dev)
        t_cnt = torch.empty((nf,), dtype=torch.int32, device=dev)
        torch.cuda.synchronize()

        def frames_call():
            matcher.run_frames_device(ctx, lo, ro, t_lk.data_ptr(), t_rk.data_ptr(), t_ld.data_ptr(),
                                      t_rd.data_ptr(), cfg, t_out.data_ptr(), t_cnt.data_ptr(), stream=ctx.stream)
        for _ in range(args.warmup):
            frames_call()
        reps = max(args.steps, 100)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(reps):
            frames_call()
        e1.record(stream)
        e1.synchronize()
        ms = e0.elapsed_time(e1) / reps
        pairs = nf * n * n
        print(json.dumps({"config": "stereo-match", "workload": "frames-64x512",
                          "desc": f"{nf} frames of {n} x {n} ORB keypoints in one launch, EuRoC intrinsics",
                          "metric": "keypoint pairs/s", "unit": "G pairs/s",
                          "device": {"value": pairs / (ms * 1e-3) / 1e9, "ms_per_call": ms,
                                     "us_per_frame": 1e3 * ms / nf, "gpu_launches_per_call": 1},
                          "matches": int(t_cnt.sum().item())}), flush=True)
    matcher.close()


def run_single_pair(args, local_rank):
    """The plain path for one pair size: synchronous compute_disparity calls on one
    seeded slanted-plane pair (W x H, D disparities, P paths), device-resident images;
    per-call latency (CUDA events) and per-stage device times."""
    import torch

    import vx_sgm
    parts = [int(v) for v in args.pair.lower().split("x")]
    w, h, d = parts[:3]
    paths = parts[3] if len(parts) > 3 else 8
    torch.cuda.set_device(local_rank)
    ctx = vx_sgm.Context(local_rank)
    sgm = vx_sgm.SGMStereo(ctx)
    stream = torch.cuda.ExternalStream(ctx.stream)
    cfg = vx_sgm.SGMStereoConfig(num_disparities=d, p1=10.0, p2=120.0, census_radius_x=2, census_radius_y=2,
                                 num_paths=paths, subpixel=True, lr_check=True, lr_tolerance=1,
                                 invalid_value=-1.0)
    L, R, _ = vx_sgm.synth_pair(vx_sgm.SCENE_SLANTED, w, h, 0, max(d - 8, 1), 3)
    tl, tr = ctx.texture_gray8(L, w, h), ctx.texture_gray8(R, w, h)
    of, oi = ctx.texture_output_r32float(w, h), ctx.texture_output_i16(w, h)
    for _ in range(args.warmup):
        sgm.compute_disparity(ctx, tl, tr, of, cfg, output_i16=oi)
    ctx.enable_stage_timing(True)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    lat = []
    for _ in range(args.steps):
        e0.record(stream)
        sgm.compute_disparity(ctx, tl, tr, of, cfg, output_i16=oi)
        e1.record(stream)
        e1.synchronize()
        lat.append(e0.elapsed_time(e1))
    census_ms, costs_ms, agg_ms, wta_ms = ctx.stage_times_detail()
    ctx.enable_stage_timing(False)
    pd = w * h * d
    print(json.dumps({"config": "single pair", "pair": f"{w}x{h} D={d}, {paths} paths", "calls": args.steps,
                      "value": pd / (float(np.mean(lat)) * 1e-3) / 1e9, "unit": UNIT,
                      "latency_ms_p50": float(np.percentile(lat, 50)),
                      "latency_ms_p99": float(np.percentile(lat, 99)),
                      "stages_ms": {"census": census_ms, "costs": costs_ms, "aggregate": agg_ms,
                                    "wta": wta_ms}}), flush=True)


WORKLOAD_DESC = ("c2: 64 mixed pairs {320x240,640x480,1242x375,1280x720} x D{64,128,192}, "
                 "8 paths, 5x5 census, P1=10 P2=120, subpixel, LR tol 1")


def run_reference(args, rank, world):
    """The reference algorithm on the host cores: the oracle restatement (the reference's
    own path is Metal and cannot run here) on every host thread, same workload and
    metric as the GPU arm. Each step is a size-stratified sample: one pair of every
    (W, H, D) stratum, a different pair of each stratum every step. Loads the pair
    generator alone (vx_synth), no CUDA code."""
    if rank != 0:
        return
    import vx_synth
    items = workload(0)
    threads = os.cpu_count() or 1
    cache = {}

    def get_pair(i):
        if i not in cache:
            cache[i] = make_pairs(vx_synth, [items[i]])[0]
        return cache[i]
    rates, n, pd, secs = [], 0, 0, 0.0
    for step in range(args.warmup + args.steps):
        rate, n1, pd1, secs1, _ = cpu_stratified(items, get_pair, threads, 1, first_round=step)
        if step >= args.warmup:
            rates.append(rate)
            n, pd, secs = n + n1, pd + pd1, secs + secs1
    value = float(np.mean(rates))
    total_pd = sum(w * h * d for (w, h, d, _) in items)
    sample = stratified_sample_text(items, n // max(args.steps, 1), pd // max(args.steps, 1),
                                    secs / max(args.steps, 1), threads) + f", {args.steps} rounds"
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "impl": "reference",
        "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": 1e3 * total_pd / 1e9 / value, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "u16", "data": "synthetic",
        "config": {"workload": WORKLOAD_DESC, "pairs_per_rank": NUM_PAIRS, "pd_per_rank": total_pd,
                   "parallelism": f"replicas x{world}"},
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": threads, "kind": "port", "sample": sample},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--plain-steps", type=int, default=1)
    ap.add_argument("--workload", default="mixed",
                    choices=["mixed", "profile", "profile-mix", "profile-wide", "profile-hd", "profile-many"])
    ap.add_argument("--sync", action="store_true",
                    help="with --kernels-only: synchronous batch calls (escape pools, no graph), for "
                         "profiler captures that must stay small")
    ap.add_argument("--serve-rate", type=float, default=200.0,
                    help="Poisson arrival rate of the served measurement (requests/s)")
    ap.add_argument("--serve-requests", type=int, default=300)
    ap.add_argument("--serve-sat-rate", type=float, default=1500.0,
                    help="arrival rate of the saturated served point (requests/s)")
    ap.add_argument("--serve-sat-requests", type=int, default=1000)
    ap.add_argument("--cpu-rounds", type=int, default=2,
                    help="stratified CPU-baseline rounds (one pair of every (W, H, D) stratum each)")
    ap.add_argument("--serve-max-batch", type=int, default=32, help="server: requests per batch at most")
    ap.add_argument("--serve-slots", type=int, default=2, help="server: batches in flight at most")
    ap.add_argument("--serve-budget-gb", type=float, default=SERVE_BUDGET / (1 << 30),
                    help="server: device budget of the served sweep (GiB)")
    ap.add_argument("--serve-sweep", default="",
                    help="comma-separated arrival rates: run the served sweep and print one JSON "
                         "line per rate instead of the benchmark")
    ap.add_argument("--pairs", type=int, default=0,
                    help="keep only the first N pairs of the workload (small profiler cases)")
    ap.add_argument("--config-table", action="store_true",
                    help="print one JSON line per single-pair / high-resolution configuration "
                         "(plain latency, batched throughput, CPU oracle) instead of the benchmark")
    ap.add_argument("--stereo-match", action="store_true",
                    help="print one JSON line per sparse ORB stereo workload (device, end to end, "
                         "CPU) instead of the benchmark")
    ap.add_argument("--stereo-only", default="",
                    choices=[""] + [w[0] for w in STEREO_WORKLOADS] + ["frames-64x512"],
                    help="with --stereo-match: run this workload only (profiler runs)")
    ap.add_argument("--pair", default="", metavar="WxHxD[xP]",
                    help="time synchronous calls on one pair of this size (the plain path) instead of "
                         "the benchmark")
    ap.add_argument("--kernels-only", action="store_true",
                    help="time the device-resident batched steps only (profiler runs)")
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3)

    rank = int(os.environ.get("RANK", 0))
    world = int(os.environ.get("WORLD_SIZE", 1))
    local_rank = int(os.environ.get("LOCAL_RANK", 0))

    if args.impl == "reference":
        run_reference(args, rank, world)
        return

    import torch
    torch.cuda.set_device(local_rank)
    dist = None
    if world > 1:
        import datetime

        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                device_id=torch.device("cuda", local_rank))

    import vx_sgm
    if args.config_table:
        run_config_table(args, local_rank)
        return
    if args.serve_sweep:
        run_serve_sweep(args, local_rank)
        return
    if args.stereo_match:
        run_stereo_match(args, local_rank)
        return
    if args.pair:
        run_single_pair(args, local_rank)
        return
    items = workload(rank, args.workload)
    if args.pairs:
        items = items[:args.pairs]
    pairs = make_pairs(vx_sgm, items)
    cfgs = [sgm_config(vx_sgm, d) for (_, _, d, _) in items]
    total_pd = sum(w * h * d for (w, h, d, _) in items)
    total_px = sum(w * h for (w, h, _, _) in items)

    ctx = vx_sgm.Context(local_rank)
    sgm = vx_sgm.SGMStereo(ctx)          # batched path: autotuned, CUDA graph per bucket
    plain_sgm = vx_sgm.SGMStereo(ctx)    # per-pair path, like the reference's call
    stream = torch.cuda.ExternalStream(ctx.stream)
    tl = [ctx.texture_gray8(L, L.shape[1], L.shape[0]) for (L, _) in pairs]
    tr = [ctx.texture_gray8(R, R.shape[1], R.shape[0]) for (_, R) in pairs]
    of = [ctx.texture_output_r32float(w, h) for (w, h, _, _) in items]
    oi = [ctx.texture_output_i16(w, h) for (w, h, _, _) in items]

    def batch():
        if args.sync:
            sgm.compute_batch(ctx, tl, tr, of, cfgs, outputs_i16=oi)
        else:
            sgm.compute_batch(ctx, tl, tr, of, cfgs, outputs_i16=oi, stream=ctx.stream)

    # ---- autotune the aggregation launch shape on this batch, then graph it ----
    if args.sync:   # a profiler case: no autotuning runs, no graph (the planner's shape)
        tuned_wg, tuned_ms, tuned_unit = 0, 0.0, 0
    else:
        tuned_wg, tuned_ms, tuned_unit = sgm.autotune_batch(ctx, tl, tr, of, cfgs, oi, iterations=1)
        sgm.set_graph_cache(2)

    # ---- device-resident batched steps (headline value) ----
    for _ in range(args.warmup):
        batch()
    ctx.synchronize()
    barrier(dist)
    torch.cuda.synchronize()
    ctx.enable_stage_timing(True)
    launches0 = vx_sgm.kernel_launch_count()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(local_rank) as clocks:
        e0.record(stream)
        for _ in range(args.steps):
            batch()
        e1.record(stream)
        e1.synchronize()
    launches = vx_sgm.kernel_launch_count() - launches0
    census_ms, costs_ms, agg_ms, wta_ms = ctx.stage_times_detail()
    ctx.enable_stage_timing(False)
    torch.cuda.synchronize()
    barrier(dist)
    ms = max_over_ranks(dist, e0.elapsed_time(e1)) / args.steps
    job_pd = sum_over_ranks(dist, float(total_pd))
    value = job_rate(job_pd, ms)
    # The timed batch's own results, kept for the parity check against the oracle.
    batch_out = [(f.read_r32float(), i.download()) for f, i in zip(of, oi)]
    if args.kernels_only:
        if rank == 0:
            print(json.dumps({"metric": METRIC, "value": value, "unit": UNIT, "ms_per_step": ms,
                              "workload": args.workload, "stages_ms": {
                                  "census": census_ms, "costs": costs_ms, "aggregate": agg_ms, "wta": wta_ms},
                              "autotuned_warpgroups": tuned_wg, "autotune_aggregate_ms": tuned_ms,
                              "autotuned_unit_scanlines": tuned_unit,
                              "gpu_launches": launches, "clocks": clocks.summary()}), flush=True)
        if dist is not None:
            dist.destroy_process_group()
        return

    # ---- end to end through the C ABI with host buffers ----
    pin = lambda n, dt: torch.empty(n, dtype=dt, pin_memory=True).numpy()
    hl = [pin(L.size, torch.uint8).reshape(L.shape) for (L, _) in pairs]
    hr = [pin(R.size, torch.uint8).reshape(R.shape) for (_, R) in pairs]
    ho = [pin(w * h, torch.float32).reshape(h, w) for (w, h, _, _) in items]
    for (L, R), a, b in zip(pairs, hl, hr):
        a[...] = L
        b[...] = R
    h2d = sum(a.nbytes + b.nbytes for a, b in zip(hl, hr))
    d2h = sum(o.nbytes for o in ho)

    # Double-buffered: two sets of device images and outputs; step k+1's uploads
    # (one copy stream) and step k's downloads (another) overlap step k's batch
    # on the context's stream. Every step still copies its own inputs in and its
    # disparities out; events order each set's upload -> batch -> download and
    # keep a set from being refilled before its batch and download are done.
    sets = [(tl, tr, of, oi),
            ([ctx.texture_gray8(L, L.shape[1], L.shape[0]) for (L, _) in pairs],
             [ctx.texture_gray8(R, R.shape[1], R.shape[0]) for (_, R) in pairs],
             [ctx.texture_output_r32float(w, h) for (w, h, _, _) in items],
             [ctx.texture_output_i16(w, h) for (w, h, _, _) in items])]
    h2d_s, d2h_s = torch.cuda.Stream(), torch.cuda.Stream()
    ev_in = [torch.cuda.Event(), torch.cuda.Event()]
    ev_done = [torch.cuda.Event(), torch.cuda.Event()]
    ev_out = [torch.cuda.Event(), torch.cuda.Event()]

    def upload(k):
        st = sets[k % 2]
        h2d_s.wait_event(ev_done[k % 2])   # its previous batch has read the inputs
        for t, a in zip(st[0], hl):
            t.upload(a, stream=h2d_s.cuda_stream)
        for t, b in zip(st[1], hr):
            t.upload(b, stream=h2d_s.cuda_stream)
        ev_in[k % 2].record(h2d_s)

    def compute(k):
        st = sets[k % 2]
        stream.wait_event(ev_in[k % 2])
        stream.wait_event(ev_out[k % 2])   # its previous outputs are downloaded
        sgm.compute_batch(ctx, st[0], st[1], st[2], cfgs, outputs_i16=st[3], stream=ctx.stream)
        ev_done[k % 2].record(stream)

    def download(k):
        st = sets[k % 2]
        d2h_s.wait_event(ev_done[k % 2])
        for t, o in zip(st[2], ho):
            t.download(o, stream=d2h_s.cuda_stream)
        ev_out[k % 2].record(d2h_s)

    def e2e_run(n):
        upload(0)
        for k in range(n):
            compute(k)
            if k + 1 < n:
                upload(k + 1)
            download(k)

    e2e_run(3)
    torch.cuda.synchronize()
    barrier(dist)
    e0.record(h2d_s)
    e2e_run(args.steps)
    stream.wait_stream(d2h_s)
    e1.record(stream)
    e1.synchronize()
    e2e_ms = max_over_ranks(dist, e0.elapsed_time(e1)) / args.steps
    e2e_value = job_rate(job_pd, e2e_ms)

    # ---- plain per-pair path (synchronous call per pair, like the reference) ----
    lat = []
    pe0, pe1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    plain_sgm.compute_disparity(ctx, tl[0], tr[0], of[0], cfgs[0], output_i16=oi[0])
    barrier(dist)
    plain_ms = 0.0
    for _ in range(args.plain_steps):
        for i in range(len(items)):
            pe0.record(stream)
            plain_sgm.compute_disparity(ctx, tl[i], tr[i], of[i], cfgs[i], output_i16=oi[i])
            pe1.record(stream)
            pe1.synchronize()
            t = pe0.elapsed_time(pe1)
            lat.append(t)
            plain_ms += t
    plain_ms = max_over_ranks(dist, plain_ms / args.plain_steps)
    plain_value = job_rate(job_pd, plain_ms)

    # ---- served: continuous batching under SERVE_BUDGET, Poisson arrivals ----
    # One point at a moderate rate and one past saturation (arrivals faster than the
    # service rate: the queue grows, batches fill and several run at once), and the
    # saturated point again with the larger budget. The batched steps are done: their
    # graph's workspace (~94 GB with full u16 shadows) goes back to the pool first, so
    # that the server's arena fits beside the rest on every rank.
    sgm.set_graph_cache(0)
    ctx.synchronize()
    serve, serve_sat = served(vx_sgm, ctx, sgm, [(args.serve_rate, args.serve_requests),
                                                 (args.serve_sat_rate, args.serve_sat_requests)])
    try:   # an extra point: a device without room for the larger arena reports why instead
        serve_sat_large, = served(vx_sgm, ctx, sgm, [(args.serve_sat_rate, args.serve_sat_requests)],
                                  budget=SERVE_BUDGET_LARGE)
        serve_sat_large = {**{k: serve_sat_large[k] for k in SERVED_KEYS}, "budget_bytes": SERVE_BUDGET_LARGE}
    except vx_sgm.VxError as e:
        serve_sat_large = {"budget_bytes": SERVE_BUDGET_LARGE, "unavailable": str(e)}

    # ---- roofline of the dominant kernel (path aggregation) ----
    peaks_path = os.path.join(REPO, "MEASURED_PEAKS.json")
    if os.path.exists(peaks_path):
        peak = float(json.load(open(peaks_path))["hbm_gbs"])
        peak_src = "measured"
    else:
        peak, peak_src = 6650.0, "fallback"
    # Algorithmic bytes (P2 = 120: byte path slabs, Dv = D rounded up to 16).
    # Scanline-pair and scan forms: the cost kernel reads the left and right
    # census and writes the cost volume (one byte per pixel-disparity); the
    # aggregation reads the volume once per path and writes one byte per path-pd.
    # Single-scanline form: the aggregation reads the census words once per path
    # instead. The pipeline adds the census pass (images in, row-major and banded
    # planes out) and the WTA (slabs in, f32 + i16 disparities out).
    census_bytes = 4  # 5x5 census: one u32 word per pixel
    dv = lambda d: (d + 15) // 16 * 16
    if tuned_unit in (64, 1):
        agg_bytes = sum(8 * 2 * w * h * dv(d) for (w, h, d, _) in items)
        costs_bytes = sum(w * h * dv(d) + 2 * w * h * census_bytes for (w, h, d, _) in items)
    else:
        agg_bytes = sum(8 * (w * h * dv(d) + 2 * w * h * census_bytes) for (w, h, d, _) in items)
        costs_bytes = 0
    agg_gbs = agg_bytes / (agg_ms * 1e-3) / 1e9
    pipeline_bytes = agg_bytes + costs_bytes + sum(8 * w * h * dv(d) + 6 * w * h + 2 * w * h + 4 * w * h * census_bytes
                                                   for (w, h, d, _) in items)
    slab_bytes = sum(8 * w * h * dv(d) for (w, h, d, _) in items)

    result = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "u16", "data": "synthetic",
        "config": {"workload": WORKLOAD_DESC,
                   "pairs_per_rank": NUM_PAIRS, "pd_per_rank": total_pd, "pixels_per_rank": total_px,
                   "parallelism": f"replicas x{world}",
                   "l2": "working set larger than L2 (byte path slabs %.1f GB per step)" % (
                       slab_bytes / 1e9)},
        "plain": {"value": plain_value, "unit": UNIT, "ms_per_pass": plain_ms,
                  "latency_ms_p50": float(np.percentile(lat, 50)),
                  "latency_ms_p99": float(np.percentile(lat, 99)),
                  "batched_over_plain": value / plain_value},
        "served": {**{k: serve[k] for k in SERVED_KEYS}, "budget_bytes": SERVE_BUDGET},
        "served_saturated": {**{k: serve_sat[k] for k in SERVED_KEYS}, "budget_bytes": SERVE_BUDGET},
        "served_saturated_80gb": serve_sat_large,
        "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": h2d,
                "d2h_bytes_per_step": d2h, "ms_per_step": e2e_ms,
                "copies": "pinned host buffers, every step; double-buffered on two copy streams, "
                          "overlapping the neighbouring steps' batches"},
        "stages_ms": {"census": census_ms, "costs": costs_ms, "aggregate": agg_ms, "wta": wta_ms},
        "roofline": {"bound": "hbm", "kernel": "path aggregation (all pairs, all paths)",
                     "achieved": agg_gbs, "peak": peak, "unit": "GB/s", "frac": agg_gbs / peak,
                     "peak_source": peak_src,
                     "traffic": AGG_DRAM_BYTES_PER_PATH_PD * 8 * total_pd if tuned_unit == 64 else None,
                     "traffic_source": AGG_TRAFFIC_SAMPLE if tuned_unit == 64 else
                     "not measured for this form (the capture is of the scanline-pair form)",
                     "algorithmic_bytes_per_launch": agg_bytes,
                     "bound_note": "the recurrence is bound by L1 requests and latency, not HBM: each "
                                   "lane reads its own scanline's cost row (a 16-byte load of a warp "
                                   "touches ~27 sectors) and each pixel's chain is serial over d; "
                                   "tensor memory holds three warpgroups' state a CTA"},
        "pipeline_roofline": {"bytes_per_step": pipeline_bytes,
                              "achieved_gbs": pipeline_bytes / (ms * 1e-3) / 1e9,
                              "frac": pipeline_bytes / (ms * 1e-3) / 1e9 / peak},
        "gpu_launches": launches,
        "batching": {"persistent_aggregation_launch": True, "cuda_graph_per_bucket": True,
                     "autotuned_warpgroups_per_cta": tuned_wg, "autotune_aggregate_ms": tuned_ms,
                     "autotuned_form": FORM_NAMES.get(tuned_unit, str(tuned_unit))},
        "clocks": clocks.summary(),
    }

    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        threads = os.cpu_count() or 1
        rate, n, pd, secs, outs = cpu_stratified(items, lambda i: pairs[i], threads, args.cpu_rounds,
                                                 keep_outputs=True)
        result["cpu_baseline"] = {"value": rate, "unit": UNIT, "cores": threads, "kind": "port",
                                  "sample": stratified_sample_text(items, n, pd, secs, threads)}
        # Parity of the timed batch: the sampled pairs' oracle results against the
        # batched run's (integer disparity exact, subpixel within 1e-4 px).
        int_ok, sub = True, 0.0
        for i, (d, di, _) in outs.items():
            gf, gi = batch_out[i]
            int_ok &= bool(np.array_equal(gi, di))
            sub = max(sub, float(np.abs(gf.astype(np.float64) - d.astype(np.float64)).max()))
        result["parity"] = {"pairs_checked": len(outs), "of": len(items), "against": "oracle",
                            "integer_exact": int_ok, "subpixel_max_abs_diff_px": sub,
                            "subpixel_tolerance_px": 1e-4, "ok": int_ok and sub <= 1e-4}
    if rank == 0:
        print(json.dumps(result), flush=True)
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
