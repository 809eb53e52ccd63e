"""Batched path on the GPU: CUDA graphs per shape bucket and the autotuner give
the same results as the plain batched call (bit for bit)."""
import os

import numpy as np
import pytest

import vx_sgm
from gpu_helpers import assert_disparity_equal, run_batch

pytestmark = pytest.mark.gpu


def _pairs(n, seed):
    rng = np.random.default_rng(seed)
    pairs, cfgs = [], []
    for i in range(n):
        w, h = int(rng.choice([96, 160, 211])), int(rng.choice([64, 90, 120]))
        nd = int(rng.choice([32, 64, 128]))
        L, R, _ = vx_sgm.synth_pair(i % 3, w, h, 2, nd - 4, seed * 100 + i)
        pairs.append((L, R))
        cfgs.append(vx_sgm.SGMStereoConfig(num_disparities=nd, census_radius_x=2, census_radius_y=2,
                                           num_paths=8, lr_check=True))
    return pairs, cfgs


def _textures(ctx, pairs):
    tl = [ctx.texture_gray8(L, L.shape[1], L.shape[0]) for L, _ in pairs]
    tr = [ctx.texture_gray8(R, R.shape[1], R.shape[0]) for _, R in pairs]
    of = [ctx.texture_output_r32float(L.shape[1], L.shape[0]) for L, _ in pairs]
    oi = [ctx.texture_output_i16(L.shape[1], L.shape[0]) for L, _ in pairs]
    return tl, tr, of, oi


def test_graph_cache_matches_plain_batch(gpu_ctx):
    pairs, cfgs = _pairs(6, 7)
    plain_sgm = vx_sgm.SGMStereo(gpu_ctx)
    want = run_batch(gpu_ctx, plain_sgm, pairs, cfgs)
    sgm = vx_sgm.SGMStereo(gpu_ctx)
    sgm.set_graph_cache(2)
    tl, tr, of, oi = _textures(gpu_ctx, pairs)
    for _ in range(3):  # capture, then replays
        sgm.compute_batch(gpu_ctx, tl, tr, of, cfgs, outputs_i16=oi)
        for (f, i), w in zip([(f.read_r32float(), i.download()) for f, i in zip(of, oi)], want):
            assert_disparity_equal((f, i), w, tol=0.0, what="graph replay")
    # same bucket, new images and outputs: the pair table is rebound
    pairs2, _ = _pairs(6, 7)
    pairs2 = [(np.ascontiguousarray(R), np.ascontiguousarray(L)) for L, R in pairs2]  # other content
    want2 = run_batch(gpu_ctx, plain_sgm, pairs2, cfgs)
    tl2, tr2, of2, oi2 = _textures(gpu_ctx, pairs2)
    sgm.compute_batch(gpu_ctx, tl2, tr2, of2, cfgs, outputs_i16=oi2)
    for f, i, w in zip(of2, oi2, want2):
        assert_disparity_equal((f.read_r32float(), i.download()), w, tol=0.0, what="graph rebind")
    # other buckets evict the least recently used one; results stay exact
    for seed in (8, 9):
        p, c = _pairs(3, seed)
        t = _textures(gpu_ctx, p)
        sgm.compute_batch(gpu_ctx, t[0], t[1], t[2], c, outputs_i16=t[3])
        w = run_batch(gpu_ctx, plain_sgm, p, c)
        for f, i, ww in zip(t[2], t[3], w):
            assert_disparity_equal((f.read_r32float(), i.download()), ww, tol=0.0, what="evict")
    sgm.set_graph_cache(0)
    sgm.close()
    plain_sgm.close()


def test_autotune_and_tuning_file(gpu_ctx, tmp_path):
    pairs, cfgs = _pairs(5, 11)
    sgm = vx_sgm.SGMStereo(gpu_ctx)
    want = run_batch(gpu_ctx, sgm, pairs, cfgs)
    tl, tr, of, oi = _textures(gpu_ctx, pairs)
    w, ms, unit = sgm.autotune_batch(gpu_ctx, tl, tr, of, cfgs, oi, iterations=1)
    assert w >= 1 and ms > 0 and unit in (1, 32, 64)
    for f, i, ww in zip(of, oi, want):
        assert_disparity_equal((f.read_r32float(), i.download()), ww, tol=0.0, what="autotune run")
    sgm.compute_batch(gpu_ctx, tl, tr, of, cfgs, outputs_i16=oi)  # uses the tuned shape
    for f, i, ww in zip(of, oi, want):
        assert_disparity_equal((f.read_r32float(), i.download()), ww, tol=0.0, what="tuned batch")
    path = os.path.join(tmp_path, "tuning.json")
    sgm.tuning_save(path)
    text = open(path).read()
    assert f'"warpgroups": {w}' in text and f'"unit_scanlines": {unit}' in text
    other = vx_sgm.SGMStereo(gpu_ctx)
    other.tuning_load(path)
    other.compute_batch(gpu_ctx, tl, tr, of, cfgs, outputs_i16=oi)
    for f, i, ww in zip(of, oi, want):
        assert_disparity_equal((f.read_r32float(), i.download()), ww, tol=0.0, what="loaded tuning")
    with pytest.raises(vx_sgm.VxError):
        other.tuning_load(os.path.join(tmp_path, "missing.json"))
    other.close()
    sgm.close()


@pytest.mark.parametrize("form", ["pairs", "single", "scan"])
def test_stage_times_through_graphs(gpu_ctx, monkeypatch, form):
    """Stage timing of graph-launched batches: every stage's events are recorded;
    the cost-volume stage exists in the scanline-pair form only, and the launch
    counter counts its kernel."""
    monkeypatch.setenv("VX_SGM_AGG_FORM", form)
    pairs, cfgs = _pairs(4, 13)
    plain = vx_sgm.SGMStereo(gpu_ctx)
    want = run_batch(gpu_ctx, plain, pairs, cfgs)
    plain.close()
    sgm = vx_sgm.SGMStereo(gpu_ctx)
    sgm.set_graph_cache(2)
    tl, tr, of, oi = _textures(gpu_ctx, pairs)
    sgm.compute_batch(gpu_ctx, tl, tr, of, cfgs, outputs_i16=oi)   # captures the bucket's graph
    gpu_ctx.enable_stage_timing(True)
    before = vx_sgm.kernel_launch_count()
    for _ in range(2):
        sgm.compute_batch(gpu_ctx, tl, tr, of, cfgs, outputs_i16=oi)
    launches = vx_sgm.kernel_launch_count() - before
    census, costs, agg, wta = gpu_ctx.stage_times_detail()
    gpu_ctx.enable_stage_timing(False)
    assert census > 0 and agg > 0 and wta > 0
    if form in ("pairs", "scan"):
        assert costs > 0 and launches == 2 * 4
    else:
        assert costs < 0.01 and launches == 2 * 3
    for f, i, ww in zip(of, oi, want):
        assert_disparity_equal((f.read_r32float(), i.download()), ww, tol=0.0, what=f"graph {form}")
    sgm.set_graph_cache(0)
    sgm.close()


@pytest.mark.parametrize("warpgroups", [1, 2, 3, 4])
def test_queue_classes_match_the_oracle(gpu_ctx, monkeypatch, warpgroups):
    """The scanline-pair kernel on a batch mixing D = 192, 128 and 64 with every CTA
    size: from 3 warpgroups up the warpgroups get TMEM budgets of different disparity
    classes (e.g. 192 + 192 + 128 columns) and the units come from one queue per
    class, so warps of a smaller budget never run a unit of a larger D. Every pair
    equals the oracle."""
    import oracle
    from gpu_helpers import cfg_pair
    monkeypatch.setenv("VX_SGM_AGG_FORM", "pairs")
    monkeypatch.setenv("VX_SGM_AGG_WARPGROUPS", str(warpgroups))
    rng = np.random.default_rng(21)
    pairs, cfgs, ocfgs = [], [], []
    for i in range(12):
        w, h = int(rng.choice([97, 160, 233])), int(rng.choice([40, 75, 130]))
        nd = [192, 128, 64, 100][i % 4]
        L, R, _ = vx_sgm.synth_pair(i % 3, w, h, 0, nd - 8, 700 + i)
        pairs.append((L, R))
        c, o = cfg_pair(num_disparities=nd, census_radius_x=2, census_radius_y=2, num_paths=8, lr_check=True)
        cfgs.append(c)
        ocfgs.append(o)
    sgm = vx_sgm.SGMStereo(gpu_ctx)
    got = run_batch(gpu_ctx, sgm, pairs, cfgs)
    sgm.close()
    for k, ((L, R), o, g) in enumerate(zip(pairs, ocfgs, got)):
        d, di, _ = oracle.sgm(L, R, o)
        assert_disparity_equal(g, (d, di), what=f"pair {k} D={o.num_disparities} with {warpgroups} warpgroups")


@pytest.mark.parametrize("pool", [None, "1"])
def test_synchronous_batch_escape_pools(gpu_ctx, monkeypatch, pool):
    """Synchronous batch calls keep escaped path vectors in a pool of 1/16 of each pair's
    vectors; with a pool of one vector (VX_SGM_SHADOW_POOL=1) every pair with two or
    more escapes overflows and is recomputed with a full shadow. Both equal the oracle,
    for every aggregation form."""
    import oracle
    from gpu_helpers import cfg_pair
    if pool:
        monkeypatch.setenv("VX_SGM_SHADOW_POOL", pool)
    rng = np.random.default_rng(5)
    pairs, cfgs, ocfgs = [], [], []
    for i in range(6):
        w, h = int(rng.choice([120, 203])), int(rng.choice([70, 101]))
        nd = [64, 128, 96, 192, 160, 48][i]     # both WTA lane forms (16 a lane; 8 at 129..192)
        L, R, _ = vx_sgm.synth_pair(2, w, h, 0, nd - 6, 900 + i)
        c, o = cfg_pair(num_disparities=nd, census_radius_x=2, census_radius_y=2, num_paths=8, lr_check=True,
                        p1=float(rng.choice([2, 10])), p2=float(rng.choice([60, 120])))
        pairs.append((L, R))
        cfgs.append(c)
        ocfgs.append(o)
    for form in ("pairs", "single", "scan"):
        monkeypatch.setenv("VX_SGM_AGG_FORM", form)
        sgm = vx_sgm.SGMStereo(gpu_ctx)
        got = run_batch(gpu_ctx, sgm, pairs, cfgs)
        sgm.close()
        for k, ((L, R), o, g) in enumerate(zip(pairs, ocfgs, got)):
            d, di, _ = oracle.sgm(L, R, o)
            assert_disparity_equal(g, (d, di), what=f"{form} pool={pool} pair {k}")


def test_plan_cache_rebinds_and_revalidates(gpu_ctx):
    """Calls whose pairs have the shapes of an earlier call reuse its plan: the pair table's
    image and output pointers are refreshed (two pairs of one shape, alternated, each equal
    to the oracle) and the pairs are validated again (an output of the wrong size is still
    rejected on a cached shape)."""
    import oracle
    from gpu_helpers import cfg_pair, run_pair
    w, h, nd = 211, 97, 64
    cfg, ocfg = cfg_pair(num_disparities=nd, census_radius_x=2, census_radius_y=2, num_paths=8, lr_check=True)
    pairs = [vx_sgm.synth_pair(k, w, h, 0, nd - 4, 500 + k)[:2] for k in range(2)]
    want = [oracle.sgm(L, R, ocfg)[:2] for (L, R) in pairs]
    sgm = vx_sgm.SGMStereo(gpu_ctx)
    for k in (0, 1, 0, 1):
        L, R = pairs[k]
        assert_disparity_equal(run_pair(gpu_ctx, sgm, L, R, cfg), want[k], what=f"call of pair {k}")
    L, R = pairs[0]
    tl, tr = gpu_ctx.texture_gray8(L, w, h), gpu_ctx.texture_gray8(R, w, h)
    small, oi = gpu_ctx.texture_output_r32float(w - 1, h), gpu_ctx.texture_output_i16(w, h)
    with pytest.raises(vx_sgm.VxError) as e:      # the same key as the calls above: a cache hit
        sgm.compute_disparity(gpu_ctx, tl, tr, small, cfg, output_i16=oi)
    assert e.value.status == 5   # VX_ERR_SIZE_MISMATCH
    sgm.close()
