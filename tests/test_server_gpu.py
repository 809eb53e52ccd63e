"""Serving loop on the GPU: continuous batching under a memory budget. Each served
result equals the same pair computed alone; oversize requests are rejected;
queued requests can be cancelled."""
import numpy as np
import pytest

import vx_sgm
from gpu_helpers import assert_disparity_equal, run_pair

pytestmark = pytest.mark.gpu

SIZES = [(160, 120), (320, 240), (211, 97), (400, 150)]


def _request(i):
    w, h = SIZES[i % len(SIZES)]
    nd = [32, 64, 128][i % 3]
    L, R, _ = vx_sgm.synth_pair(vx_sgm.SCENE_PLANES, w, h, 2, nd - 4, 500 + i)
    cfg = vx_sgm.SGMStereoConfig(num_disparities=nd, census_radius_x=2, census_radius_y=2,
                                 num_paths=8, lr_check=True)
    return L, R, cfg


def test_served_results_equal_solo(gpu_ctx, sgm):
    reqs = [_request(i) for i in range(14)]
    biggest = max(vx_sgm.workspace_bytes(L.shape[1], L.shape[0], c) for L, _, c in reqs)
    # Budget for about three requests at a time: requests queue and batches form.
    srv = vx_sgm.Server(sgm, gpu_ctx, memory_budget_bytes=3 * biggest, max_batch=4,
                        max_inflight_batches=2)
    ids = [srv.submit(L, R, c) for L, R, c in reqs]
    results = [srv.wait(i) for i in ids]
    st = srv.stats()
    srv.close()
    assert st["completed"] == len(reqs) and st["batches"] >= 2 and st["failed"] == 0
    assert st["completed_pixel_disparities"] == sum(L.size * c.num_disparities for L, _, c in reqs)
    for (L, R, c), (d, di, lat) in zip(reqs, results):
        assert lat > 0
        assert_disparity_equal((d, di), run_pair(gpu_ctx, sgm, L, R, c), tol=0.0, what="served vs solo")


def test_batches_overlap_on_the_device(gpu_ctx, sgm):
    """Continuous batching: with memory for two batches and two stream slots, a batch is
    launched while the previous one is still running on the GPU (the server counts the
    unfinished batches at every launch), and every result still equals the solo result."""
    reqs = [_request(i) for i in range(3, 3 + 16)]
    biggest = max(vx_sgm.workspace_bytes(L.shape[1], L.shape[0], c) for L, _, c in reqs)
    srv = vx_sgm.Server(sgm, gpu_ctx, memory_budget_bytes=10 * biggest, max_batch=4,
                        max_inflight_batches=2)
    ids = [srv.submit(L, R, c) for L, R, c in reqs]
    results = [srv.wait(i) for i in ids]
    st = srv.stats()
    srv.close()
    assert st["completed"] == len(reqs) and st["failed"] == 0 and st["batches"] >= 4
    assert st["max_batches_in_flight"] == 2, st
    for (L, R, c), (d, di, _) in zip(reqs, results):
        assert_disparity_equal((d, di), run_pair(gpu_ctx, sgm, L, R, c), tol=0.0, what="overlapped vs solo")


@pytest.mark.parametrize("pool", [None, "1"])
def test_escape_pool_and_reruns(gpu_ctx, sgm, monkeypatch, pool):
    """Served requests keep their escaped path vectors in a pool of 1/16 of their
    vectors. With the default pool nothing overflows and every result equals the
    solo (full-shadow) result; with a pool of one vector every pair with two or
    more escapes overflows, is recomputed with a full shadow, and still equals it."""
    if pool:
        monkeypatch.setenv("VX_SGM_SHADOW_POOL", pool)
    reqs = [_request(i) for i in range(10)]
    biggest = max(vx_sgm.workspace_bytes(L.shape[1], L.shape[0], c) for L, _, c in reqs)
    srv = vx_sgm.Server(sgm, gpu_ctx, memory_budget_bytes=3 * biggest, max_batch=6,
                        max_inflight_batches=2)
    ids = [srv.submit(L, R, c) for L, R, c in reqs]
    results = [srv.wait(i) for i in ids]
    st = srv.stats()
    srv.close()
    monkeypatch.delenv("VX_SGM_SHADOW_POOL", raising=False)
    assert st["completed"] == len(reqs) and st["failed"] == 0
    if pool:
        assert st["shadow_reruns"] > 0
    else:
        assert st["shadow_reruns"] == 0
    for (L, R, c), (d, di, _) in zip(reqs, results):
        assert_disparity_equal((d, di), run_pair(gpu_ctx, sgm, L, R, c), tol=0.0, what="served vs solo")


def test_escape_pool_with_wide_slab_requests(gpu_ctx, sgm, monkeypatch):
    """Batches that mix wide-slab requests (P2 = 300: every vector in u16, no pool)
    with pooled byte-slab requests run the pool-aware kernels with wide tiles; with
    a one-vector pool the byte-slab requests overflow, are recomputed, and every
    result equals its solo result."""
    monkeypatch.setenv("VX_SGM_SHADOW_POOL", "1")
    reqs = []
    for i in range(8):
        L, R, c = _request(i)
        if i % 2:
            c = vx_sgm.SGMStereoConfig(num_disparities=c.num_disparities, census_radius_x=2, census_radius_y=2,
                                       num_paths=8, p1=15.0, p2=300.0, lr_check=True)
        reqs.append((L, R, c))
    biggest = max(vx_sgm.workspace_bytes(L.shape[1], L.shape[0], c) for L, _, c in reqs)
    srv = vx_sgm.Server(sgm, gpu_ctx, memory_budget_bytes=4 * biggest, max_batch=8, max_inflight_batches=1)
    ids = [srv.submit(L, R, c) for L, R, c in reqs]
    results = [srv.wait(i) for i in ids]
    st = srv.stats()
    srv.close()
    monkeypatch.delenv("VX_SGM_SHADOW_POOL", raising=False)
    assert st["completed"] == len(reqs) and st["failed"] == 0 and st["shadow_reruns"] > 0
    for (L, R, c), (d, di, _) in zip(reqs, results):
        assert_disparity_equal((d, di), run_pair(gpu_ctx, sgm, L, R, c), tol=0.0, what="served vs solo")


def test_serving_allocates_nothing_after_start(gpu_ctx, sgm):
    """The device arena and the pinned staging arena are taken at creation; serving a
    stream of mixed requests grows neither the context's pool nor the pinned memory."""
    reqs = [_request(i) for i in range(24)]
    biggest = max(vx_sgm.workspace_bytes(L.shape[1], L.shape[0], c) for L, _, c in reqs)
    srv = vx_sgm.Server(sgm, gpu_ctx, memory_budget_bytes=4 * biggest, max_batch=4,
                        max_inflight_batches=2)
    st0 = srv.stats()
    ids = [srv.submit(L, R, c) for L, R, c in reqs]
    for i in ids:
        srv.wait(i)
    st = srv.stats()
    srv.close()
    assert st["completed"] == len(reqs) and st["failed"] == 0
    assert st["pool_reserved_bytes"] == st0["pool_reserved_bytes"]
    assert st["pinned_bytes"] == st0["pinned_bytes"] and st["staging_overflows"] == 0
    assert st["inflight_bytes"] == 0


def test_staging_overflow_still_serves(gpu_ctx, sgm):
    """A staging arena too small for the queued requests: the excess requests get
    their own pinned buffers and the results are unchanged."""
    reqs = [_request(i) for i in range(8)]
    biggest = max(vx_sgm.workspace_bytes(L.shape[1], L.shape[0], c) for L, _, c in reqs)
    srv = vx_sgm.Server(sgm, gpu_ctx, memory_budget_bytes=3 * biggest, max_batch=4,
                        max_inflight_batches=2, host_staging_bytes=1 << 18)
    ids = [srv.submit(L, R, c) for L, R, c in reqs]
    results = [srv.wait(i) for i in ids]
    st = srv.stats()
    srv.close()
    assert st["completed"] == len(reqs) and st["staging_overflows"] > 0
    for (L, R, c), (d, di, _) in zip(reqs, results):
        assert_disparity_equal((d, di), run_pair(gpu_ctx, sgm, L, R, c), tol=0.0, what="overflow staging")


def test_oversize_request_is_rejected(gpu_ctx, sgm):
    srv = vx_sgm.Server(sgm, gpu_ctx, memory_budget_bytes=1 << 20, max_batch=4)
    L, R, c = _request(1)
    with pytest.raises(vx_sgm.VxError) as e:
        srv.submit(L, R, c)
    assert e.value.status == 8  # VX_ERR_BUDGET
    assert srv.stats()["rejected"] == 1
    srv.close()


def test_cancel_queued_request(gpu_ctx, sgm):
    reqs = [_request(i) for i in range(6)]
    need = max(vx_sgm.workspace_bytes(L.shape[1], L.shape[0], c) for L, _, c in reqs)
    srv = vx_sgm.Server(sgm, gpu_ctx, memory_budget_bytes=int(need * 1.5), max_batch=1,
                        max_inflight_batches=1)
    ids = [srv.submit(L, R, c) for L, R, c in reqs]
    cancelled = None
    for rid in reversed(ids):  # the last ones are still queued behind the first
        try:
            srv.cancel(rid)
            cancelled = rid
            break
        except vx_sgm.VxError:
            continue
    assert cancelled is not None
    for rid in ids:
        if rid == cancelled:
            with pytest.raises(vx_sgm.VxError) as e:
                srv.wait(rid)
            assert e.value.status == 12  # VX_ERR_CANCELLED
        else:
            d, di, _ = srv.wait(rid)
            assert d.shape == di.shape
    assert srv.stats()["cancelled"] == 1
    srv.close()


def test_server_rejects_bad_config(gpu_ctx, sgm):
    srv = vx_sgm.Server(sgm, gpu_ctx, memory_budget_bytes=1 << 30)
    L, R, _ = _request(0)
    with pytest.raises(vx_sgm.VxError) as e:
        srv.submit(L, R, vx_sgm.SGMStereoConfig(num_disparities=300))
    assert e.value.status == 6
    srv.close()
