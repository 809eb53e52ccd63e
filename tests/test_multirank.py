"""Host logic of the multi-GPU run (replicas only), on CPU with gloo, world size 2:
every rank gets its own pairs, no data-path collective, and the reported time is the
maximum over ranks."""
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
    # each rank's simulated step time; the job's time is the slowest rank's
    t = torch.tensor([10.0 + rank], dtype=torch.float64)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    pd = sum(w * h * d for (w, h, d, _) in items)
    q.put((rank, [g.tolist() for g in gathered], float(t.item()), pd))
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


def test_workload_is_deterministic():
    assert bench.workload(0) == bench.workload(0)
    assert bench.workload(0) != bench.workload(1)
    sizes = {(w, h) for (w, h, _, _) in bench.workload(0)}
    assert sizes <= set(bench.SIZES)
    assert {d for (_, _, d, _) in bench.workload(0)} <= set(bench.DISPARITIES)
