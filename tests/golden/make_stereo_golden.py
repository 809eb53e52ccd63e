"""Generates tests/golden/stereo_match_cases.npz from the reference itself.

The reference sparse matcher (vx-vision/shaders/StereoMatch.metal:
stereo_hamming + stereo_extract, as StereoMatcher::run in
vx-vision/src/kernels/stereomatch.rs:115-249 drives them) is compiled unmodified
as C++ by oracle/Makefile into oracle/_ref/libstereo_ref.so, which only builds
where the reference sources are mounted. This script runs it on seeded
keypoint sets and stores inputs, configurations and the matches as fixtures,
so that the oracle restatement and the CUDA path are pinned against the
reference anywhere. The reference has no test of its own for this kernel; its
example (examples/orb_stereo_benchmark.rs:22-94: at most 512 keypoints per
side, EuRoC intrinsics) gives the first case's sizes and configuration.

Cases: synthetic pairs at the example's sizes and configuration and at the
default StereoConfig; empty sides; one keypoint; ties (duplicate descriptors,
equal distances); the max_hamming boundary; max_hamming 0xFFFF (keypoints
without a candidate match right index 0) and a max_hamming above 16 bits
(the shader's ushort cast); NaN and infinite positions; tests hitting the
epipolar and disparity bounds exactly; a negative epipolar tolerance; an
empty disparity range; zero disparity (infinite depth); every keypoint on a
few rows; a larger random case.

Usage: python tests/golden/make_stereo_golden.py
"""
import os
import sys

import numpy as np

REPO = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, os.path.join(REPO, "oracle"))
sys.path.insert(0, os.path.join(REPO, "vx-rs_b200"))
import oracle  # noqa: E402
import vx_sgm  # noqa: E402  (synthetic keypoints only)

CFG_KEYS = ["max_epipolar", "min_disparity", "max_disparity", "max_hamming", "ratio_thresh", "fx", "fy",
            "cx", "cy", "baseline"]
EUROC = dict(max_epipolar=2.0, min_disparity=1.0, max_disparity=120.0, max_hamming=50, ratio_thresh=0.8,
             fx=458.654, fy=457.296, cx=367.215, cy=248.375, baseline=0.110)


def kp(xy, level=0):
    xy = np.asarray(xy, np.float32).reshape(-1, 2)
    k = np.zeros(len(xy), vx_sgm.CORNER_POINT)
    k["position"] = xy
    k["response"] = 1.0
    k["pyramid_level"] = level
    return k


def words(rng, n):
    return rng.integers(0, 2 ** 32, (n, 8), dtype=np.uint64).astype(np.uint32)


def with_bits(base, nbits, rng):
    out = base.copy()
    for b in rng.choice(256, nbits, replace=False):
        out[b >> 5] ^= np.uint32(1) << np.uint32(b & 31)
    return out


def synth(n_left, n_right, seed, **kw):
    lk, rk, ld, rd = vx_sgm.synth_orb_stereo(n_left, n_right, seed, **kw)
    return lk, rk, ld["desc"].copy(), rd["desc"].copy()


def main():
    if not oracle.ref_stereo_available():
        sys.exit("oracle/_ref/libstereo_ref.so is missing: run make -C oracle where the reference is mounted")
    rng = np.random.default_rng(20240601)
    cases = {}

    cases["euroc_512"] = (*synth(512, 512, 1), EUROC)
    cases["euroc_300x450"] = (*synth(300, 450, 2), EUROC)
    cases["default_1000x1200"] = (*synth(1000, 1200, 3, width=640), {})
    cases["empty_left"] = (kp(np.zeros((0, 2))), kp([[10, 10]]), words(rng, 0), words(rng, 1), {})
    cases["empty_right"] = (kp([[10, 10]]), kp(np.zeros((0, 2))), words(rng, 1), words(rng, 0), {})
    d = words(rng, 1)
    cases["single"] = (kp([[100, 50]]), kp([[60, 50.5]]), d, with_bits(d[0], 7, rng)[None], {})
    cases["single_none"] = (kp([[100, 50]]), kp([[160, 50]]), d, d.copy(), {})

    # Ties: identical descriptors at several right indices, and different ones at
    # the same distance; the first right index must win.
    base = words(rng, 1)[0]
    l_xy = [[200, 100], [300, 150], [400, 200]]
    r_xy, r_w = [], []
    for (x, y) in l_xy:
        for j in range(6):
            r_xy.append([x - 10 - 7 * j, y + (j % 3) - 1])
            r_w.append(with_bits(base, 12 if j % 2 else 9, rng) if j < 4 else base.copy())
    lw = np.stack([with_bits(base, 3, rng), base.copy(), with_bits(base, 20, rng)])
    order = rng.permutation(len(r_xy))
    cases["ties"] = (kp(l_xy), kp(np.asarray(r_xy)[order]), lw, np.stack(r_w)[order], {})

    # max_hamming boundary: distances exactly 49, 50, 51 against max_hamming 50.
    lw = words(rng, 3)
    rw = np.stack([with_bits(lw[i], 49 + i, rng) for i in range(3)])
    cases["hamming_edge"] = (kp([[100, 10], [100, 20], [100, 30]]), kp([[90, 10], [90, 20], [90, 30]]), lw, rw,
                             dict(max_hamming=50))
    lk, rk, lw, rw = synth(200, 150, 4)
    cases["max_hamming_ffff"] = (lk, rk, lw, rw, dict(max_hamming=0xFFFF))
    cases["max_hamming_wrap"] = (lk, rk, lw, rw, dict(max_hamming=0x10000 + 30))
    cases["max_hamming_256"] = (lk, rk, lw, rw, dict(max_hamming=256))

    lk, rk, lw, rw = synth(120, 130, 5)
    lk["position"][3] = [np.nan, 40.0]
    lk["position"][7] = [100.0, np.nan]
    lk["position"][11] = [np.inf, 60.0]
    lk["position"][13] = [200.0, np.inf]
    rk["position"][2] = [np.nan, np.nan]
    rk["position"][5] = [-np.inf, lk["position"][20][1]]
    rk["position"][9] = [lk["position"][21][0], np.inf]
    cases["nonfinite"] = (lk, rk, lw, rw, {})
    cases["nonfinite_inf_range"] = (lk, rk, lw, rw, dict(max_epipolar=np.inf, max_disparity=np.inf))

    # Bounds hit exactly: dy == max_epipolar, d == min_disparity, d == max_disparity.
    lw = words(rng, 4)
    rw = np.stack([with_bits(lw[i], 5, rng) for i in range(4)])
    cases["bounds_exact"] = (kp([[50.25, 10.0], [80.0, 20.5], [200.0, 30.0], [300.0, 40.0]]),
                             kp([[40.25, 12.0], [79.0, 20.5], [80.0, 30.0], [179.0, 40.0]]), lw, rw,
                             dict(max_epipolar=2.0, min_disparity=1.0, max_disparity=120.0))
    lk, rk, lw, rw = synth(150, 150, 6)
    cases["negative_epipolar"] = (lk, rk, lw, rw, dict(max_epipolar=-1.0))
    cases["empty_range"] = (lk, rk, lw, rw, dict(min_disparity=50.0, max_disparity=10.0))
    cases["zero_disparity"] = (lk, rk, lw, rw, dict(min_disparity=-5.0, max_disparity=5.0, max_hamming=256,
                                                    cx=0.0))
    # Every keypoint on four rows: many candidates per left keypoint.
    lk, rk, lw, rw = synth(400, 400, 7, height=4)
    cases["four_rows"] = (lk, rk, lw, rw, dict(max_hamming=120))
    cases["random_3000x2800"] = (*synth(3000, 2800, 8, width=1280, height=720),
                                 dict(max_epipolar=1.5, min_disparity=0.5, max_disparity=96.0, max_hamming=64,
                                      fx=700.0, fy=701.0, cx=640.0, cy=360.0, baseline=0.2))

    out = {}
    names = []
    for name, (lk, rk, lw, rw, cfg) in cases.items():
        c = dict(oracle.STEREO_DEFAULTS)
        c.update(cfg)
        m = oracle.ref_stereo_match(lk, rk, lw, rw, c)
        names.append(name)
        out[f"{name}/lk"] = np.asarray(lk).view(np.float32).reshape(-1, 4)
        out[f"{name}/rk"] = np.asarray(rk).view(np.float32).reshape(-1, 4)
        out[f"{name}/ld"] = np.asarray(lw, np.uint32).reshape(-1, 8)
        out[f"{name}/rd"] = np.asarray(rw, np.uint32).reshape(-1, 8)
        out[f"{name}/cfg_f"] = np.array([c[k] for k in CFG_KEYS if k != "max_hamming"], np.float32)
        out[f"{name}/max_hamming"] = np.array([int(c["max_hamming"])], np.uint64)
        out[f"{name}/matches"] = m.view(np.uint32).reshape(-1, 7)
        print(f"{name}: {len(lk)} x {len(rk)} -> {len(m)} matches")
    out["names"] = np.array(names)
    np.savez_compressed(os.path.join(os.path.dirname(os.path.abspath(__file__)), "stereo_match_cases.npz"), **out)


if __name__ == "__main__":
    main()
