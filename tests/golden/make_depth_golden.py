"""Generates tests/golden/depth_filter_cases.npz from the reference itself.

The reference depth filters (vx-vision/shaders/DepthFilter.metal: depth_median,
depth_bilateral) are compiled unmodified as C++ by oracle/Makefile into
oracle/_ref/libdepth_ref.so, which only builds where the reference sources are
mounted. This script runs them on small maps and stores inputs, parameters and
outputs as fixtures, so that the oracle restatement and the CUDA path can be
pinned against the reference anywhere.

Inputs: the reference's own depth-filter test maps (vx-vision/tests/
test_kernels.rs:843-851, a 32x32 step edge 1.0 | 5.0, and :883-887, a 32x32
map of 2.0 with two noisy pixels), and disparity maps produced by the SGM
oracle on seeded synthetic pairs with the LR check on (invalid pixels = -1),
with every median radius 0..5 and several bilateral settings; plus edge maps
(W = 1, H = 1, all invalid, +inf and NaN values for the median).

Usage: python tests/golden/make_depth_golden.py
"""
import json
import os
import sys

import numpy as np

REPO = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, os.path.join(REPO, "oracle"))
sys.path.insert(0, os.path.join(REPO, "vx-rs_b200"))
import oracle  # noqa: E402
import vx_sgm  # noqa: E402  (synthetic pairs only)


def sgm_disparity(w, h, nd, seed):
    L, R, _ = vx_sgm.synth_pair(vx_sgm.SCENE_SLANTED, w, h, 2, nd - 4, seed)
    cfg = oracle.config(num_disparities=nd, census_radius_x=2, census_radius_y=2, num_paths=4,
                        subpixel=True, lr_check=True, lr_tolerance=1, invalid_value=-1.0)
    d, _, _ = oracle.sgm(L, R, cfg)
    return d


def main():
    if not oracle.ref_depth_available():
        sys.exit("oracle/_ref/libdepth_ref.so is missing: run make -C oracle where the reference is mounted")
    maps = {}
    w = h = 32
    maps["ref_edge"] = np.where(np.arange(w * h).reshape(h, w) % w < w // 2, 1.0, 5.0).astype(np.float32)
    noisy = np.full((h, w), 2.0, np.float32)
    noisy.flat[100] = 99.0
    noisy.flat[200] = 0.5
    maps["ref_noise"] = noisy
    maps["sgm_96x64"] = sgm_disparity(96, 64, 32, 11)
    maps["sgm_131x47"] = sgm_disparity(131, 47, 48, 12)
    maps["row_1x40"] = sgm_disparity(40, 8, 16, 13)[3:4, :].copy()
    maps["col_37x1"] = sgm_disparity(37, 20, 16, 14)[:, 5:6].copy()
    maps["invalid"] = np.full((9, 7), -1.0, np.float32)
    special = sgm_disparity(45, 30, 32, 15)
    special[3, 4] = np.inf
    special[10, 10] = np.nan
    special[20, 40] = 0.0
    maps["special"] = special

    cases = []
    for name, m in maps.items():
        for r in range(0, 6):
            if name == "ref_edge" and r > 1:
                continue
            cases.append(("median", name, {"radius": r}))
        if name == "special":
            continue  # bilateral of inf/NaN is NaN in any implementation: not a parity case
        for (r, ss, sd) in ([(2, 3.0, 0.1)] if name.startswith("ref") else
                            [(3, 5.0, 0.05), (1, 1.0, 0.5), (2, 3.0, 2.0), (5, 2.0, 1.0)]):
            cases.append(("bilateral", name, {"radius": r, "sigma_spatial": ss, "sigma_depth": sd}))
    out, meta = {}, []
    for name, m in maps.items():
        out[f"map/{name}"] = m
    for i, (kind, name, p) in enumerate(cases):
        m = maps[name]
        if kind == "median":
            res = oracle.ref_depth_median(m, p["radius"])
        else:
            res = oracle.ref_depth_bilateral(m, p["radius"], p["sigma_spatial"], p["sigma_depth"])
        out[f"out/{i}"] = res
        meta.append({"id": i, "kind": kind, "map": name, **p})
    out["meta"] = np.frombuffer(json.dumps(meta).encode(), np.uint8)
    path = os.path.join(os.path.dirname(os.path.abspath(__file__)), "depth_filter_cases.npz")
    np.savez_compressed(path, **out)
    print(f"wrote {len(cases)} cases to {path}")


if __name__ == "__main__":
    main()
