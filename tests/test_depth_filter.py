"""Depth-map post-filters (vx-vision DepthFilter: median, bilateral).

CPU: the oracle restatement (oracle/depth_oracle.cpp) equals the reference
shader's own outputs (tests/golden/depth_filter_cases.npz, made by
tests/golden/make_depth_golden.py from shaders/DepthFilter.metal compiled as
C++); the reference's own test assertions hold on the oracle.
GPU: the CUDA filters through the C ABI against the same fixtures — the median
bit-exact, the bilateral within 1e-5 relative (its range weights come from CUDA's
__expf intrinsic, the fixtures' from the host's expf) — and against the oracle on SGM
disparity maps."""
import json
import os

import numpy as np
import pytest

import oracle
import vx_sgm

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "depth_filter_cases.npz")
BILATERAL_RTOL = 1e-5


def _cases():
    z = np.load(GOLDEN)
    meta = json.loads(bytes(z["meta"]).decode())
    maps = {k.split("/", 1)[1]: z[k] for k in z.files if k.startswith("map/")}
    return [(m, maps[m["map"]], z[f"out/{m['id']}"]) for m in meta]


def _run_oracle(m, depth):
    if m["kind"] == "median":
        return oracle.depth_median(depth, m["radius"])
    return oracle.depth_bilateral(depth, m["radius"], m["sigma_spatial"], m["sigma_depth"])


def _same_bits(a, b):
    return np.array_equal(np.asarray(a, np.float32).view(np.uint32), np.asarray(b, np.float32).view(np.uint32))


def test_oracle_equals_reference_fixtures():
    cases = _cases()
    assert len(cases) >= 60
    for m, depth, want in cases:
        got = _run_oracle(m, depth)
        assert _same_bits(got, want), m


def test_reference_assertions_on_oracle():
    """vx-vision/tests/test_kernels.rs:840-901, on the oracle."""
    w = h = 32
    edge = np.where(np.arange(w * h).reshape(h, w) % w < w // 2, 1.0, 5.0).astype(np.float32)
    r = oracle.depth_bilateral(edge, 2, 3.0, 0.1)
    assert abs(r[h // 2, w // 4] - 1.0) < 0.5 and abs(r[h // 2, 3 * w // 4] - 5.0) < 0.5
    noisy = np.full((h, w), 2.0, np.float32)
    noisy.flat[100] = 99.0
    noisy.flat[200] = 0.5
    assert abs(oracle.depth_median(noisy, 1).flat[100] - 2.0) < 1.0


def test_median_excludes_invalid_and_takes_upper_middle():
    d = np.array([[-1, 3, 1], [2, -1, 4], [-1, -1, 5]], np.float32)
    # centre window (r = 1, clamped) holds the valid values 3 1 2 4 5 -> sorted 1 2 3 4 5 -> index 2
    assert oracle.depth_median(d, 1)[1, 1] == 3.0
    d2 = np.array([[1, 2], [3, 4]], np.float32)
    # r = 1 window of (0, 0), clamped: 1 1 2 1 1 2 3 3 4 -> count 9, index 4 -> 2
    assert oracle.depth_median(d2, 1)[0, 0] == 2.0
    assert oracle.depth_median(np.full((3, 3), -1, np.float32), 1).max() == 0.0


@pytest.mark.gpu
def test_cuda_filters_match_reference_fixtures(gpu_ctx):
    filt = vx_sgm.DepthFilter(gpu_ctx)
    for m, depth, want in _cases():
        h, w = depth.shape
        tin = gpu_ctx.texture_r32float(depth, w, h)
        tout = gpu_ctx.texture_output_r32float(w, h)
        if m["kind"] == "median":
            filt.apply_median(gpu_ctx, tin, tout, vx_sgm.DepthMedianConfig(m["radius"]))
            assert _same_bits(tout.read_r32float(), want), m
        else:
            filt.apply_bilateral(gpu_ctx, tin, tout, vx_sgm.DepthFilterConfig(
                m["radius"], m["sigma_spatial"], m["sigma_depth"]))
            got = tout.read_r32float()
            np.testing.assert_allclose(got, want, rtol=BILATERAL_RTOL, atol=0, err_msg=str(m))
    filt.close()


@pytest.mark.gpu
def test_cuda_median_on_sgm_output_large(gpu_ctx, sgm):
    """The demo chain: SGM with the LR check (invalid = -1), then the median filter; the
    filtered map equals the oracle's median of the same map, bit for bit."""
    w, h = 640, 480
    L, R, _ = vx_sgm.synth_pair(vx_sgm.SCENE_PLANES, w, h, 4, 60, 77)
    cfg = vx_sgm.SGMStereoConfig(num_disparities=64, census_radius_x=2, census_radius_y=2,
                                 num_paths=4, lr_check=True)
    tl, tr = gpu_ctx.texture_gray8(L, w, h), gpu_ctx.texture_gray8(R, w, h)
    disp = gpu_ctx.texture_output_r32float(w, h)
    sgm.compute_disparity(gpu_ctx, tl, tr, disp, cfg)
    d = disp.read_r32float()
    assert (d < 0).any()
    filt = vx_sgm.DepthFilter(gpu_ctx)
    out = gpu_ctx.texture_output_r32float(w, h)
    for r in (1, 2, 3):
        filt.apply_median(gpu_ctx, disp, out, vx_sgm.DepthMedianConfig(r))
        assert _same_bits(out.read_r32float(), oracle.depth_median(d, r)), r
    filt.apply_bilateral(gpu_ctx, disp, out, vx_sgm.DepthFilterConfig())
    np.testing.assert_allclose(out.read_r32float(), oracle.depth_bilateral(d, 3, 5.0, 0.05),
                               rtol=BILATERAL_RTOL, atol=0)
    filt.close()


@pytest.mark.gpu
def test_cuda_filter_argument_checks(gpu_ctx):
    filt = vx_sgm.DepthFilter(gpu_ctx)
    a = gpu_ctx.texture_output_r32float(16, 8)
    b = gpu_ctx.texture_output_r32float(16, 9)
    with pytest.raises(vx_sgm.VxError) as e:
        filt.apply_median(gpu_ctx, a, b)
    assert e.value.status == 5  # size mismatch
    c = gpu_ctx.texture_output_r32float(16, 8)
    for bad in (-1, 6):
        with pytest.raises(vx_sgm.VxError) as e:
            filt.apply_median(gpu_ctx, a, c, vx_sgm.DepthMedianConfig(bad))
        assert e.value.status == 6
    with pytest.raises(vx_sgm.VxError):
        filt.apply_bilateral(gpu_ctx, a, c, vx_sgm.DepthFilterConfig(3, 0.0, 0.05))
    with pytest.raises(vx_sgm.VxError):
        filt.apply_median(gpu_ctx, a, a)  # in place
    filt.close()
