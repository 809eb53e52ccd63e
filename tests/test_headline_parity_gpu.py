"""Parity at the benchmarked scale: the benchmark's own workloads, run the way the
benchmark runs them, against the oracle pair by pair (integer disparity exact,
subpixel within 1e-4 px). The semantics are those of
vx-vision/shaders/SGMStereo.metal:120-214 plus the 8-path and LR extensions.

* The 64-pair mixed batch (sizes {320x240, 640x480, 1242x375, 1280x720}, D in
  {64, 128, 192}, 8 paths, LR check): autotuned, then through the CUDA-graph
  cache, two batched calls of which the second is a graph replay.
* The high-resolution configuration (2048x1536, D = 256, planes + sinusoid +
  textureless patches) as a staged batch: three pairs under a workspace limit
  that splits them into sub-batches of two and one.
"""
import os

import numpy as np
import pytest

import bench
import oracle
import vx_sgm
from gpu_helpers import SUBPIXEL_TOL, assert_disparity_equal

pytestmark = pytest.mark.gpu

THREADS = os.cpu_count() or 1


def _textures(ctx, pairs):
    tl = [ctx.texture_gray8(L, L.shape[1], L.shape[0]) for L, _ in pairs]
    tr = [ctx.texture_gray8(R, R.shape[1], R.shape[0]) for _, R in pairs]
    of = [ctx.texture_output_r32float(L.shape[1], L.shape[0]) for L, _ in pairs]
    oi = [ctx.texture_output_i16(L.shape[1], L.shape[0]) for L, _ in pairs]
    return tl, tr, of, oi


@pytest.mark.timeout(900)
def test_benchmark_batch_matches_oracle(gpu_ctx):
    items = bench.workload(0)
    pairs = bench.make_pairs(vx_sgm, items)
    cfgs = [bench.sgm_config(vx_sgm, d) for (_, _, d, _) in items]
    tl, tr, of, oi = _textures(gpu_ctx, pairs)
    sgm = vx_sgm.SGMStereo(gpu_ctx)
    sgm.autotune_batch(gpu_ctx, tl, tr, of, cfgs, oi, iterations=1)
    sgm.set_graph_cache(2)
    launches = vx_sgm.kernel_launch_count()
    for call in range(2):                      # capture, then a replay of the captured graph
        sgm.compute_batch(gpu_ctx, tl, tr, of, cfgs, outputs_i16=oi, stream=gpu_ctx.stream)
        gpu_ctx.synchronize()
    assert vx_sgm.kernel_launch_count() - launches >= 2 * 4
    got = [(f.read_r32float(), i.download()) for f, i in zip(of, oi)]
    sgm.set_graph_cache(0)
    sgm.close()
    worst = 0.0
    for k, ((w, h, d, seed), (L, R), g) in enumerate(zip(items, pairs, got)):
        want_f, want_i, _ = oracle.sgm(L, R, bench.oracle_config(oracle, d), nthreads=THREADS)
        assert_disparity_equal(g, (want_f, want_i), what=f"pair {k} ({w}x{h} D={d} seed {seed})")
        worst = max(worst, float(np.abs(g[0].astype(np.float64) - want_f).max()))
    assert worst <= SUBPIXEL_TOL


@pytest.mark.timeout(900)
def test_staged_high_resolution_batch_matches_oracle(gpu_ctx):
    w, h, d = 2048, 1536, 256
    cfg = vx_sgm.SGMStereoConfig(num_disparities=d, p1=10.0, p2=120.0, census_radius_x=2,
                                 census_radius_y=2, num_paths=8, subpixel=True, lr_check=True,
                                 lr_tolerance=1, invalid_value=-1.0)
    pairs = [vx_sgm.synth_pair(vx_sgm.SCENE_SURFACE, w, h, 0, 230, 4242 + i)[:2] for i in range(3)]
    per_pair = vx_sgm.workspace_bytes(w, h, cfg)
    ctx = vx_sgm.Context(0)
    # Room for two pairs' workspaces but not three: sub-batches of two and one.
    ctx.set_workspace_limit(int(2.5 * per_pair))
    sgm = vx_sgm.SGMStereo(ctx)
    tl, tr, of, oi = _textures(ctx, pairs)
    sgm.compute_batch(ctx, tl, tr, of, [cfg] * 3, outputs_i16=oi)
    got = [(f.read_r32float(), i.download()) for f, i in zip(of, oi)]
    del tl, tr, of, oi
    sgm.close()
    ctx.close()
    ocfg = oracle.config(num_disparities=d, p1=10, p2=120, census_radius_x=2, census_radius_y=2,
                         num_paths=8, subpixel=True, lr_check=True)
    for k, ((L, R), g) in enumerate(zip(pairs, got)):
        want_f, want_i, _ = oracle.sgm(L, R, ocfg, nthreads=THREADS)
        assert (want_i >= 0).mean() > 0.5, "the scene should be mostly matchable"
        assert_disparity_equal(g, (want_f, want_i), what=f"staged pair {k}")
