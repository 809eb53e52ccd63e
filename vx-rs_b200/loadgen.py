"""Open-loop Poisson load generator for the SGM server (vx_sgm.Server).

Requests arrive with exponential inter-arrival times at a given rate whatever
the server's state (open loop); each is submitted from a producer thread and
collected by a consumer thread that records the submit-to-completion latency
measured by the server. ctypes releases the GIL during the library calls, so
submission and collection overlap with the GPU work.
"""
from __future__ import annotations

import threading
import time

import numpy as np

import vx_sgm

# Resolutions and disparity ranges of the served workload.
SERVED_SIZES = [(640, 480), (1242, 375), (1280, 720), (1920, 1080)]
SERVED_DISPARITIES = [64, 128, 192]


def make_requests(count: int, seed: int = 7, paths: int = 8):
    """Seeded synthetic requests: (left, right, config), sizes and D drawn uniformly,
    piecewise-planar scenes with a per-request seed."""
    rng = np.random.default_rng(seed)
    out = []
    for i in range(count):
        w, h = SERVED_SIZES[int(rng.integers(len(SERVED_SIZES)))]
        d = int(SERVED_DISPARITIES[int(rng.integers(len(SERVED_DISPARITIES)))])
        L, R, _ = vx_sgm.synth_pair(vx_sgm.SCENE_PLANES, w, h, 4, int(0.9 * d), 90_000 + seed * 1000 + i)
        cfg = vx_sgm.SGMStereoConfig(num_disparities=d, census_radius_x=2, census_radius_y=2,
                                     num_paths=paths, lr_check=True)
        out.append((L, R, cfg))
    return out


def run_poisson(server: "vx_sgm.Server", requests, rate_per_s: float, num_requests: int,
                seed: int = 11, timeout_ms: int = 120000) -> dict:
    """Submits num_requests (cycling through `requests`) at Poisson arrivals of the
    given rate and waits for all. Returns latency percentiles and throughput."""
    rng = np.random.default_rng(seed)
    gaps = rng.exponential(1.0 / rate_per_s, size=num_requests)
    ids: list = [None] * num_requests
    lat = np.zeros(num_requests)
    pds = np.zeros(num_requests)
    submitted = threading.Semaphore(0)
    errors = []

    def produce():
        t_next = time.perf_counter()
        for i in range(num_requests):
            t_next += gaps[i]
            delay = t_next - time.perf_counter()
            if delay > 0:
                time.sleep(delay)
            L, R, cfg = requests[i % len(requests)]
            try:
                ids[i] = server.submit(L, R, cfg, want_i16=False)
            except vx_sgm.VxError as e:  # rejected: counted, not waited for
                errors.append(str(e))
            pds[i] = L.size * cfg.num_disparities
            submitted.release()

    def consume():
        for i in range(num_requests):
            submitted.acquire()
            if ids[i] is None:
                continue
            _, _, lat[i] = server.wait(ids[i], timeout_ms)

    t0 = time.perf_counter()
    threads = [threading.Thread(target=produce), threading.Thread(target=consume)]
    for t in threads:
        t.start()
    for t in threads:
        t.join()
    wall = time.perf_counter() - t0
    done = np.array([i is not None for i in ids])
    return {
        "rate_per_s": rate_per_s,
        "requests": int(num_requests),
        "completed": int(done.sum()),
        "rejected": len(errors),
        "latency_ms_p50": float(np.percentile(lat[done], 50)) if done.any() else None,
        "latency_ms_p99": float(np.percentile(lat[done], 99)) if done.any() else None,
        "latency_ms_mean": float(lat[done].mean()) if done.any() else None,
        "throughput_gpd_s": float(pds[done].sum() / wall / 1e9),
        "achieved_rate_per_s": float(done.sum() / wall),
        "wall_s": wall,
    }
