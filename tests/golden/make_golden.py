"""Generates tests/golden/reference_cases.npz from the reference itself.

The reference SGM shader (vx-vision/shaders/SGMStereo.metal) is compiled
unmodified as C++ by oracle/Makefile into oracle/_ref/libsgm_ref.so, which only
builds where the reference sources are mounted. This script runs it on small
inputs and stores inputs, parameters and outputs (census words, the u16 cost
volume S, the f32 disparity) as fixtures, so that the oracle restatement and
the CUDA path can be pinned against the reference anywhere.

Inputs: the reference's own SGM test pattern (vx-vision/tests/test_kernels.rs:
787-812: 64x64 checkerboard, right image built with its shift of 5), the bench
image of vx-vision/benches/kernel_benchmarks.rs:14-24 shifted by 8 px as in
:199-208, and seeded synthetic pairs that cover odd sizes, W < D, W = 1, H = 1,
empty and 62-bit census windows, and extreme penalties.

Usage: python tests/golden/make_golden.py
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


def checkerboard_case():
    w = h = 64
    shift = 5
    x = np.arange(w)[None, :].repeat(h, 0)
    y = np.arange(h)[:, None].repeat(w, 1)
    left = np.where(((x // 4) + (y // 4)) % 2 == 0, 200, 50).astype(np.uint8)
    sx = np.where(x >= shift, x - shift, 0)
    right = np.where(((sx // 4) + (y // 4)) % 2 == 0, 200, 50).astype(np.uint8)
    return left, right


def bench_image_case(w=320, h=240, shift=8):
    x = np.arange(w, dtype=np.uint32)[None, :].repeat(h, 0)
    y = np.arange(h, dtype=np.uint32)[:, None].repeat(w, 1)
    grad = ((x.astype(np.float32) / np.float32(w)) * np.float32(255.0)).astype(np.uint8)
    noise = (((x * 17) ^ (y * 31)) % 64).astype(np.uint8)
    left = (grad.astype(np.uint16) + noise).astype(np.uint8)  # wrapping_add
    right = left.copy()
    right[:, shift:] = left[:, :-shift]
    return left, right


CASES = [
    # name, inputs, nd, p1, p2, rx, ry, store_S
    ("reference_test_checkerboard", checkerboard_case, 32, 10.0, 120.0, 4, 3, True),
    ("reference_bench_320x240_d64", bench_image_case, 64, 10.0, 120.0, 4, 3, False),
    ("planes_40x24_d16_r2", (0, 40, 24, 2, 14, 11), 16, 10.0, 120.0, 2, 2, True),
    ("planes_33x17_d7_r1_odd", (0, 33, 17, 1, 6, 12), 7, 3.0, 40.0, 1, 1, True),
    ("planes_12x20_d24_w_lt_d", (0, 12, 20, 1, 10, 13), 24, 10.0, 120.0, 4, 3, True),
    ("planes_1x9_d5_w1", (0, 1, 9, 0, 0, 14), 5, 10.0, 120.0, 1, 1, True),
    ("planes_17x1_d8_h1", (0, 17, 1, 1, 6, 15), 8, 10.0, 120.0, 2, 2, True),
    ("planes_24x16_d12_r0", (0, 24, 16, 1, 10, 16), 12, 10.0, 120.0, 0, 0, True),
    ("planes_30x12_d16_r31x0", (0, 30, 12, 1, 12, 17), 16, 10.0, 120.0, 31, 0, True),
    ("planes_32x16_d16_p1_gt_p2", (0, 32, 16, 1, 12, 18), 16, 200.0, 100.0, 2, 2, True),
    ("planes_32x16_d16_p0", (0, 32, 16, 1, 12, 19), 16, 0.0, 0.0, 2, 2, True),
    ("planes_32x16_d16_p2_5000", (0, 32, 16, 1, 12, 20), 16, 10.0, 5000.0, 2, 2, True),
    ("planes_32x16_d16_p_60000", (0, 32, 16, 1, 12, 21), 16, 60000.0, 60000.5, 2, 2, True),
    ("planes_48x32_d256", (0, 48, 32, 1, 30, 22), 256, 10.0, 120.0, 2, 2, True),
    ("slanted_64x48_d64_r4x3", (1, 64, 48, 2, 50, 23), 64, 10.0, 120.0, 4, 3, True),
    ("surface_96x64_d128_r2", (2, 96, 64, 2, 90, 24), 128, 7.5, 95.9, 2, 2, False),
]


def main():
    oracle.build()
    assert oracle.ref_available(), "reference shader not built (mount the reference, run make -C oracle)"
    out = {}
    meta = []
    for name, src, nd, p1, p2, rx, ry, store_S in CASES:
        if callable(src):
            left, right = src()
        else:
            scene, w, h, lo, hi, seed = src
            left, right, _ = vx_sgm.synth_pair(scene, w, h, lo, hi, seed)
        cl, cr, S, disp = oracle.reference_sgm(left, right, nd, p1, p2, rx, ry)
        out[f"{name}/left"] = left
        out[f"{name}/right"] = right
        out[f"{name}/census_l"] = cl
        out[f"{name}/census_r"] = cr
        out[f"{name}/disparity"] = disp
        if store_S:
            out[f"{name}/S"] = S
        out[f"{name}/S_sum"] = np.array([int(S.astype(np.uint64).sum())], np.uint64)
        meta.append(dict(name=name, nd=nd, p1=p1, p2=p2, rx=rx, ry=ry, store_S=store_S))
    out["meta"] = np.frombuffer(json.dumps(meta).encode(), dtype=np.uint8)
    path = os.path.join(os.path.dirname(os.path.abspath(__file__)), "reference_cases.npz")
    np.savez_compressed(path, **out)
    print(f"wrote {path} ({os.path.getsize(path)} bytes, {len(meta)} cases)")


if __name__ == "__main__":
    main()
