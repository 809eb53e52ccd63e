"""SGMStereo::compute -> DepthMap, the depth epilogue, batches staged under a
workspace limit, and one full pair of the high-resolution configuration
(2048x1536, D=256, 8 paths) against the oracle."""
import numpy as np
import pytest

import oracle
import vx_sgm
from gpu_helpers import assert_disparity_equal, cfg_pair, run_batch, run_pair

pytestmark = pytest.mark.gpu


def test_compute_returns_depth_map_like_reference(gpu_ctx, sgm):
    w, h = 200, 120
    L, R, _ = vx_sgm.synth_pair(vx_sgm.SCENE_PLANES, w, h, 4, 40, 77)
    cfg = vx_sgm.SGMStereoConfig(num_disparities=64, census_radius_x=2, census_radius_y=2,
                                 num_paths=4, lr_check=True)
    intr = vx_sgm.CameraIntrinsics(fx=700.0, fy=700.0, cx=w / 2, cy=h / 2, width=w, height=h)
    tl, tr = gpu_ctx.texture_gray8(L, w, h), gpu_ctx.texture_gray8(R, w, h)
    depth = gpu_ctx.texture_output_r32float(w, h)
    dm = sgm.compute(gpu_ctx, tl, tr, cfg, intr, 0.12, depth_out=depth)
    # sgm.rs:278-287: the DepthMap wraps the disparity texture, range [0, f32::MAX]
    assert dm.min_depth == 0.0 and dm.max_depth == np.finfo(np.float32).max
    assert dm.intrinsics == intr
    disp = dm.texture.read_r32float()
    want_f, want_i = run_pair(gpu_ctx, sgm, L, R, cfg)
    assert np.array_equal(disp.view(np.uint32), want_f.view(np.uint32))
    z = depth.read_r32float()
    valid = (want_i >= 0) & (want_f > 0)
    expect = np.where(valid, np.float32(700.0 * 0.12) / np.where(valid, want_f, 1).astype(np.float32), 0)
    assert np.array_equal(z, expect.astype(np.float32))
    dm.texture.close()


def test_batch_over_workspace_limit_is_staged(gpu_ctx, sgm):
    pairs, cfgs = [], []
    for i in range(5):
        w, h = 240 + 16 * i, 100 + 8 * i
        nd = [64, 128, 48][i % 3]
        L, R, _ = vx_sgm.synth_pair(i % 3, w, h, 2, nd - 4, 300 + i)
        pairs.append((L, R))
        cfgs.append(vx_sgm.SGMStereoConfig(num_disparities=nd, census_radius_x=2, census_radius_y=2,
                                           num_paths=8, lr_check=True))
    want = [run_pair(gpu_ctx, sgm, L, R, c) for (L, R), c in zip(pairs, cfgs)]
    biggest = max(vx_sgm.workspace_bytes(L.shape[1], L.shape[0], c) for (L, _), c in zip(pairs, cfgs))
    ctx = vx_sgm.Context(0)
    s2 = vx_sgm.SGMStereo(ctx)
    ctx.set_workspace_limit(int(biggest * 1.5))  # at most one or two pairs per sub-batch
    got = run_batch(ctx, s2, pairs, cfgs)
    for g, w_ in zip(got, want):
        assert_disparity_equal(g, w_, tol=0.0, what="staged batch")
    s2.close()
    ctx.close()


@pytest.mark.timeout(600)
def test_high_resolution_pair_matches_oracle(gpu_ctx, sgm):
    """One pair of the 16 x 2048x1536 configuration (planes + sinusoidal surface + 10%
    textureless patches, D=256, 8 paths, LR): integer disparity bit-exact, subpixel
    within 1e-4 px."""
    w, h = 2048, 1536
    L, R, _ = vx_sgm.synth_pair(vx_sgm.SCENE_SURFACE, w, h, 0, 250, 2048)
    cfg, ocfg = cfg_pair(num_disparities=256, census_radius_x=2, census_radius_y=2, num_paths=8,
                         lr_check=True)
    got = run_pair(gpu_ctx, sgm, L, R, cfg)
    d, di, _ = oracle.sgm(L, R, ocfg)
    assert_disparity_equal(got, (d, di), what="2048x1536 D=256")
