"""Generates tests/golden/cloud_cases.npz from the reference itself.

The reference colour conversion and depth unprojection
(vx-vision/shaders/ColorConvert.metal: rgba_to_gray, and
vx-vision/shaders/DepthToCloud.metal: depth_to_cloud) are compiled unmodified as
C++ by oracle/Makefile into oracle/_ref/libcloud_ref.so, which only builds where
the reference sources are mounted. This script runs them (one pixel at a time,
row-major, so the shader's atomic point counter hands out slots in pixel order)
and stores inputs, parameters and outputs as fixtures, so that the oracle
restatement and the CUDA path can be pinned against the reference anywhere.

Inputs: the reference's own unprojection test (vx-vision/tests/test_kernels.rs:
948-982: a 32x32 depth map of 2.0, fx = fy = 100, cx = cy = 16, range
[0.1, 10]), the depth chain of examples/depth_to_cloud_demo.rs:78-92 (an SGM
disparity map used as depth, intrinsics from_focal_length(W, W, H), range
[1, max disparity]) with its LR-invalid pixels, seeded maps with NaN, +-inf and
negative depths, a depth scale, U8 and RGBA8 colour images, a colour image one
pixel wide (ignored by the shader), max_points below the number of valid
pixels; RGBA images of odd sizes, every gray level, saturated colours.

Usage: python tests/golden/make_cloud_golden.py
"""
import json
import os
import sys

import numpy as np

REPO = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, os.path.join(REPO, "oracle"))
sys.path.insert(0, os.path.join(REPO, "vx-rs_b200"))
import oracle  # noqa: E402
import vx_synth  # noqa: E402  (synthetic pairs only)


def sgm_disparity(w, h, nd, seed):
    L, R, _ = vx_synth.synth_pair(vx_synth.SCENE_SLANTED, w, h, 2, nd - 4, seed)
    cfg = oracle.config(num_disparities=nd, census_radius_x=2, census_radius_y=2, num_paths=4,
                        subpixel=True, lr_check=True, lr_tolerance=1, invalid_value=-1.0)
    d, _, _ = oracle.sgm(L, R, cfg)
    return d, L


def main():
    if not oracle.ref_cloud_available():
        sys.exit("oracle/_ref/libcloud_ref.so is missing: run make -C oracle where the reference is mounted")
    rng = np.random.default_rng(2024)
    arrays, meta = {}, []

    # ---- rgba_to_gray ----
    grays = {
        "gray_random_64x48": rng.integers(0, 256, (48, 64, 4), dtype=np.uint8),
        "gray_odd_333x7": rng.integers(0, 256, (7, 333, 4), dtype=np.uint8),
        "gray_1x1": np.array([[[12, 200, 77, 3]]], np.uint8),
        "gray_levels": np.repeat(np.arange(256, dtype=np.uint8)[None, :, None], 4, axis=2),
        "gray_saturated": np.array([[[255, 0, 0, 255], [0, 255, 0, 255], [0, 0, 255, 255], [255, 255, 255, 0],
                                     [0, 0, 0, 255], [255, 255, 0, 9], [0, 255, 255, 9], [255, 0, 255, 9]]],
                                   np.uint8),
    }
    for name, im in grays.items():
        arrays[f"{name}/rgba"] = im
        arrays[f"{name}/gray"] = oracle.rgba_to_gray(im, ref=True)
        meta.append({"name": name, "kind": "gray"})

    # ---- depth_to_cloud ----
    clouds = []
    clouds.append(("cloud_reference_test", np.full((32, 32), 2.0, np.float32), None,
                   dict(fx=100.0, fy=100.0, cx=16.0, cy=16.0, min_depth=0.1, max_depth=10.0)))
    disp, L = sgm_disparity(96, 64, 48, 7)
    valid = disp[disp > 0]
    clouds.append(("cloud_sgm_demo_chain", disp, None,
                   dict(fx=96.0, fy=96.0, cx=48.0, cy=32.0, min_depth=1.0, max_depth=float(max(valid.max(), 1.0)))))
    clouds.append(("cloud_sgm_gray_color", disp, L,
                   dict(fx=96.0, fy=96.0, cx=48.0, cy=32.0, min_depth=1.0, max_depth=float(max(valid.max(), 1.0)))))
    d = rng.uniform(-1.0, 12.0, (41, 57)).astype(np.float32)
    d[rng.random(d.shape) < 0.05] = np.nan
    d[0, :3] = [np.inf, -np.inf, 0.1]
    d[1, :2] = [10.0, np.float32(10.0) * 1.0000001]
    color = rng.integers(0, 256, (41, 57, 4), dtype=np.uint8)
    clouds.append(("cloud_random_rgba", d, color, dict(fx=311.5, fy=298.25, cx=28.3, cy=20.1)))
    clouds.append(("cloud_random_max_points", d, color, dict(fx=311.5, fy=298.25, cx=28.3, cy=20.1,
                                                               max_points=500)))
    mm = rng.uniform(0.0, 12000.0, (23, 19)).astype(np.float32)
    clouds.append(("cloud_millimetres", mm, None, dict(fx=50.0, fy=52.0, cx=9.0, cy=11.0, depth_scale=0.001)))
    clouds.append(("cloud_color_one_wide", np.full((5, 1), 3.0, np.float32), np.full((5, 1), 80, np.uint8),
                   dict(fx=10.0, fy=10.0, cx=0.0, cy=2.0)))
    clouds.append(("cloud_one_row", rng.uniform(0, 5, (1, 300)).astype(np.float32), None,
                   dict(fx=400.0, fy=400.0, cx=150.0, cy=0.0)))
    clouds.append(("cloud_none_valid", np.full((8, 8), 50.0, np.float32), None, dict(fx=1.0, fy=1.0)))
    for name, depth, col, kw in clouds:
        params = dict(oracle.CLOUD_DEFAULTS, fx=500.0, fy=500.0, cx=0.0, cy=0.0)
        params.update(kw)
        pts, n = oracle.depth_to_cloud(depth, col, ref=True, **params)
        arrays[f"{name}/depth"] = depth
        if col is not None:
            arrays[f"{name}/color"] = col
        arrays[f"{name}/points"] = pts
        meta.append({"name": name, "kind": "cloud", "params": params, "count": n, "color": col is not None})

    arrays["meta"] = np.frombuffer(json.dumps(meta).encode(), np.uint8)
    out = os.path.join(REPO, "tests", "golden", "cloud_cases.npz")
    np.savez_compressed(out, **arrays)
    print(f"wrote {out}: {len(meta)} cases")


if __name__ == "__main__":
    main()
