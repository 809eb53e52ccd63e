"""The depth chain's ends around SGM: RGBA -> gray ingest
(vx-vision/shaders/ColorConvert.metal:21-32) and depth map -> point cloud
(vx-vision/shaders/DepthToCloud.metal:30-70).

CPU: the oracle restatement equals the fixtures made by the reference shaders
compiled as C++ (tests/golden/make_cloud_golden.py). GPU: the CUDA kernels equal
the fixtures (gray bytes exact; points field for field, NaN = NaN) and the
oracle on larger maps, through the host-buffer and the device-buffer entry
points, and the whole chain (colour pair -> gray -> SGM with its depth output ->
point cloud) equals the oracle applied step by step."""
import json
import os

import numpy as np
import pytest

import oracle
import vx_sgm

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.fixture(scope="module")
def cases():
    z = np.load(os.path.join(REPO, "tests", "golden", "cloud_cases.npz"))
    meta = json.loads(bytes(z["meta"]).decode())
    out = []
    for m in meta:
        c = dict(m)
        for k in ("rgba", "gray", "depth", "color", "points"):
            key = f"{m['name']}/{k}"
            c[k] = z[key] if key in z else None
        out.append(c)
    return out


def assert_points_equal(got, want, what):
    assert len(got) == len(want), f"{what}: {len(got)} points, want {len(want)}"
    for f in ("position", "normal"):
        g, w = got[f].astype(np.float64), want[f].astype(np.float64)
        assert np.array_equal(g, w, equal_nan=True), f"{what}: {f} differs at {np.argwhere(~((g == w) | (np.isnan(g) & np.isnan(w))))[:3]}"
    assert np.array_equal(got["color"], want["color"]), f"{what}: colour differs"


def test_oracle_matches_reference_fixtures(cases):
    for c in cases:
        if c["kind"] == "gray":
            assert np.array_equal(oracle.rgba_to_gray(c["rgba"]), c["gray"]), c["name"]
        else:
            pts, n = oracle.depth_to_cloud(c["depth"], c["color"], **c["params"])
            assert n == c["count"], c["name"]
            assert_points_equal(pts, c["points"], c["name"])


def test_reference_unprojection_test_case(cases):
    """vx-vision/tests/test_kernels.rs:948-982: every pixel of a flat map at 2.0 gives a
    point with Z = 2 (the fixture, checked here as the reference test states it)."""
    c = next(c for c in cases if c["name"] == "cloud_reference_test")
    assert c["count"] == 32 * 32 and np.all(np.abs(c["points"]["position"][:, 2] - 2.0) < 0.01)


def _cloud_gpu(ctx, dc, depth, color, params, device_form=False):
    h, w = depth.shape
    td = ctx.texture_r32float(depth, w, h)
    tc = None
    if color is not None:
        tc = ctx.texture_rgba8(color, w, h) if color.ndim == 3 else ctx.texture_gray8(color, color.shape[1],
                                                                                       color.shape[0])
    cfg = vx_sgm.DepthToCloudConfig(params["min_depth"], params["max_depth"], params["depth_scale"],
                                    params["max_points"])
    if not device_form:
        return dc.compute_raw(ctx, td, tc, params["fx"], params["fy"], params["cx"], params["cy"], cfg).points
    import torch
    cap = min(cfg.max_points, w * h)
    buf = torch.zeros(max(cap, 1) * 9, dtype=torch.int32, device="cuda")
    cnt = torch.zeros(1, dtype=torch.int32, device="cuda")
    dc.compute_device(ctx, td, tc, params["fx"], params["fy"], params["cx"], params["cy"], cfg, buf.data_ptr(), cap,
                      cnt.data_ptr())
    n = min(int(cnt.item()), cap)
    return np.frombuffer(buf.cpu().numpy().tobytes(), vx_sgm.POINT3D)[:n]


@pytest.mark.gpu
@pytest.mark.parametrize("device_form", [False, True])
def test_gpu_matches_reference_fixtures(gpu_ctx, cases, device_form):
    dc = vx_sgm.DepthToCloud(gpu_ctx)
    conv = vx_sgm.ColorConvert(gpu_ctx)
    for c in cases:
        if c["kind"] == "gray":
            h, w, _ = c["rgba"].shape
            tin, tout = gpu_ctx.texture_rgba8(c["rgba"], w, h), gpu_ctx.texture_output_gray8(w, h)
            conv.rgba_to_gray(gpu_ctx, tin, tout)
            assert np.array_equal(tout.download(), c["gray"]), c["name"]
        else:
            got = _cloud_gpu(gpu_ctx, dc, c["depth"], c["color"], c["params"], device_form)
            assert_points_equal(got, c["points"], c["name"])
    dc.close()


@pytest.mark.gpu
def test_gpu_large_maps_match_the_oracle(gpu_ctx):
    """1920x1080 (2 025 tiles of 1024 pixels: offsets across many CTAs), colour, NaN,
    and max_points cutting inside a tile."""
    rng = np.random.default_rng(77)
    w, h = 1920, 1080
    depth = rng.uniform(-2.0, 14.0, (h, w)).astype(np.float32)
    depth[rng.random((h, w)) < 0.01] = np.nan
    color = rng.integers(0, 256, (h, w, 4), dtype=np.uint8)
    dc = vx_sgm.DepthToCloud(gpu_ctx)
    for extra in (dict(), dict(max_points=777_777), dict(depth_scale=0.5, min_depth=0.0, max_depth=np.inf)):
        params = dict(oracle.CLOUD_DEFAULTS, fx=1000.0, fy=1001.0, cx=960.5, cy=539.5)
        params.update(extra)
        want, n = oracle.depth_to_cloud(depth, color, **params)
        got = _cloud_gpu(gpu_ctx, dc, depth, color, params)
        assert_points_equal(got, want, str(extra))
        got_d = _cloud_gpu(gpu_ctx, dc, depth, color, params, device_form=True)
        assert_points_equal(got_d, want, f"device {extra}")
    dc.close()
    conv = vx_sgm.ColorConvert(gpu_ctx)
    tin, tout = gpu_ctx.texture_rgba8(color, w, h), gpu_ctx.texture_output_gray8(w, h)
    conv.rgba_to_gray(gpu_ctx, tin, tout)
    assert np.array_equal(tout.download(), oracle.rgba_to_gray(color))


@pytest.mark.gpu
def test_colour_pair_to_point_cloud_chain(gpu_ctx, sgm):
    """The demo chain (examples/depth_to_cloud_demo.rs:44-92) on the GPU: a colour pair is
    converted to gray, matched by SGM whose WTA also writes depth = fx * B / d, and the
    depth map is unprojected with its intrinsics; every step equals the oracle's."""
    w, h, nd = 160, 96, 64
    L, R, _ = vx_sgm.synth_pair(vx_sgm.SCENE_PLANES, w, h, 4, 50, 99)
    rng = np.random.default_rng(3)
    tint = rng.integers(0, 2, 3)
    rgba_l = np.stack([L, L // 2 + 60 * tint[0], L, np.full_like(L, 255)], axis=2).astype(np.uint8)
    rgba_r = np.stack([R, R // 2 + 60 * tint[0], R, np.full_like(R, 255)], axis=2).astype(np.uint8)
    conv = vx_sgm.ColorConvert(gpu_ctx)
    gl, gr = gpu_ctx.texture_output_gray8(w, h), gpu_ctx.texture_output_gray8(w, h)
    conv.rgba_to_gray(gpu_ctx, gpu_ctx.texture_rgba8(rgba_l, w, h), gl)
    conv.rgba_to_gray(gpu_ctx, gpu_ctx.texture_rgba8(rgba_r, w, h), gr)
    ol, orr = oracle.rgba_to_gray(rgba_l), oracle.rgba_to_gray(rgba_r)
    assert np.array_equal(gl.download(), ol) and np.array_equal(gr.download(), orr)
    cfg = vx_sgm.SGMStereoConfig(num_disparities=nd, census_radius_x=2, census_radius_y=2, num_paths=8,
                                 lr_check=True)
    intr = vx_sgm.CameraIntrinsics(fx=200.0, fy=200.0, cx=80.0, cy=48.0, width=w, height=h)
    depth_tex = gpu_ctx.texture_output_r32float(w, h)
    dmap = sgm.compute(gpu_ctx, gl, gr, cfg, intr, 0.12, depth_out=depth_tex)
    depth = depth_tex.download()
    ocfg = oracle.config(num_disparities=nd, census_radius_x=2, census_radius_y=2, num_paths=8, lr_check=True)
    disp, _, _ = oracle.sgm(ol, orr, ocfg)
    scale = np.float32(np.float32(200.0) * np.float32(0.12))
    want_depth = np.where(disp > 0, scale / np.where(disp > 0, disp, 1), 0).astype(np.float32)
    assert np.allclose(depth, want_depth, rtol=1e-6, atol=0)
    dc = vx_sgm.DepthToCloud(gpu_ctx)
    cloud = dc.compute(gpu_ctx, vx_sgm.DepthMap(depth_tex, intr, 0.0, 3.4e38), gpu_ctx.texture_rgba8(rgba_l, w, h),
                       vx_sgm.DepthToCloudConfig.new(0.1, 10.0))
    want, n = oracle.depth_to_cloud(depth, rgba_l, fx=200.0, fy=200.0, cx=80.0, cy=48.0, min_depth=0.1, max_depth=10.0)
    assert len(cloud) == n > 1000
    assert_points_equal(cloud.points, want, "chain")
    dc.close()
    del dmap


def test_invalid_arguments_are_rejected_before_any_launch():
    """Format and size checks of the C entry points (no GPU needed: the checks come first)."""
    import ctypes
    lib = ctypes.CDLL(vx_sgm.LIB_PATH)
    lib.vx_color_rgba_to_gray.restype = ctypes.c_int
    assert lib.vx_color_rgba_to_gray(None, None, None, None) == 10
    lib.vx_depth_to_cloud_compute_raw.restype = ctypes.c_int
    assert lib.vx_depth_to_cloud_compute_raw(None, None, None, None, ctypes.c_float(1), ctypes.c_float(1),
                                             ctypes.c_float(0), ctypes.c_float(0), None, None, ctypes.c_size_t(0),
                                             None) == 10
