"""Host logic of the multi-GPU run (replicas only), on CPU with gloo, world size 2:
every rank gets its own pairs, no data-path collective, and the reported time is the
maximum over ranks, through bench.py's own barrier / max_over_ranks / job_rate."""
import os
import socket

import pytest
import torch.distributed as dist
import torch.multiprocessing as mp

import bench


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _worker(rank, world, port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    import torch
    items = bench.workload(rank)
    seeds = torch.tensor([it[3] for it in items], dtype=torch.int64)
    gathered = [torch.zeros_like(seeds) for _ in range(world)]
    dist.all_gather(gathered, seeds)
    # bench.py's own barrier and max-over-ranks (on the CPU: gloo), with a
    # different step time per rank; the job's time is the slowest rank's.
    bench.barrier(dist)
    ms = bench.max_over_ranks(dist, 10.0 + rank, device="cpu")
    pd = sum(w * h * d for (w, h, d, _) in items)
    job_pd = bench.sum_over_ranks(dist, float(pd), device="cpu")
    rate = bench.job_rate(job_pd, ms)
    bench.barrier(dist)
    q.put((rank, [g.tolist() for g in gathered], ms, pd, rate))
    dist.destroy_process_group()


@pytest.mark.timeout(120)
def test_replicas_get_distinct_pairs_and_max_time():
    world = 2
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    out = [q.get(timeout=90) for _ in range(world)]
    for p in procs:
        p.join(timeout=30)
        assert p.exitcode == 0
    out.sort()
    seeds0, seeds1 = out[0][1]
    assert len(seeds0) == len(seeds1) == bench.NUM_PAIRS
    assert not set(seeds0) & set(seeds1)          # replicas process different pairs
    assert out[0][2] == out[1][2] == 11.0         # max over ranks
    assert out[0][3] > 1e9 and out[1][3] > 1e9    # every rank carries a full workload
    # whole-job rate: all ranks' work over the slowest rank's time, the same on every rank
    assert out[0][4] == out[1][4] == pytest.approx((out[0][3] + out[1][3]) / 11.0e-3 / 1e9)


def test_single_process_helpers_need_no_process_group():
    assert bench.max_over_ranks(None, 3.5) == 3.5
    bench.barrier(None)
    assert bench.sum_over_ranks(None, 7.0) == 7.0
    assert bench.job_rate(2e9, 1000.0) == pytest.approx(2.0)


def test_stratified_cpu_sample_covers_every_stratum():
    groups = bench.strata(bench.workload(0))
    assert sum(len(v) for v in groups.values()) == bench.NUM_PAIRS
    assert {(w, h) for (w, h, _) in groups} <= set(bench.SIZES)


def test_workload_is_deterministic():
    assert bench.workload(0) == bench.workload(0)
    assert bench.workload(0) != bench.workload(1)
    sizes = {(w, h) for (w, h, _, _) in bench.workload(0)}
    assert sizes <= set(bench.SIZES)
    assert {d for (_, _, d, _) in bench.workload(0)} <= set(bench.DISPARITIES)
