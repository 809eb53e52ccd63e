"""Sparse ORB stereo matching (vx-vision StereoMatcher: stereo_hamming + stereo_extract).

CPU: the oracle restatement (oracle/stereo_oracle.cpp) equals the reference
shader's own matches (tests/golden/stereo_match_cases.npz, made by
tests/golden/make_stereo_golden.py from shaders/StereoMatch.metal compiled as
C++), record for record, bit for bit; host-side argument checks.
GPU: the CUDA matcher through the C ABI (host-buffer and device-buffer entry
points) against the same fixtures and against the oracle at sizes up to
16384 x 16384 keypoints: integer fields and floats bit-exact (the kernels use
IEEE round-to-nearest arithmetic in the shader's operation order), except that
NaN equals NaN whatever its bits (0 * inf from an infinite keypoint: x86 gives
0xffc00000, CUDA 0x7fffffff; the reference does not fix a NaN encoding)."""
import os

import numpy as np
import pytest

import oracle
import vx_sgm

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "stereo_match_cases.npz")
CFG_F = ["max_epipolar", "min_disparity", "max_disparity", "ratio_thresh", "fx", "fy", "cx", "cy", "baseline"]


def _cases():
    z = np.load(GOLDEN)
    out = []
    for name in z["names"]:
        name = str(name)
        cfg = {k: float(v) for k, v in zip(CFG_F, z[f"{name}/cfg_f"])}
        cfg["max_hamming"] = int(z[f"{name}/max_hamming"][0])
        out.append((name, z[f"{name}/lk"], z[f"{name}/rk"], z[f"{name}/ld"], z[f"{name}/rd"], cfg,
                    z[f"{name}/matches"]))
    return out


def _words(m):
    return np.ascontiguousarray(m).view(np.uint32).reshape(-1, 7)


def _same_records(got, want):
    """Bit-equal records, a NaN field matching any NaN."""
    a, b = _words(got), _words(want)
    if a.shape != b.shape:
        return False
    fa, fb = a[:, 2:6].view(np.float32), b[:, 2:6].view(np.float32)
    both_nan = np.isnan(fa) & np.isnan(fb)
    return bool(np.array_equal(a[:, [0, 1, 6]], b[:, [0, 1, 6]]) and np.all((a[:, 2:6] == b[:, 2:6]) | both_nan))


def _lib_cfg(cfg):
    return vx_sgm.StereoConfig(**cfg)


def test_oracle_equals_reference_fixtures():
    cases = _cases()
    assert len(cases) >= 20
    for name, lk, rk, ld, rd, cfg, want in cases:
        got = oracle.stereo_match(lk, rk, ld, rd, cfg)
        assert np.array_equal(_words(got), want), name


def test_fixtures_cover_the_edge_cases():
    """The cases the kernel's semantics hinge on are present and non-trivial."""
    by = {c[0]: c for c in _cases()}
    assert len(by["empty_left"][6]) == 0 and len(by["empty_right"][6]) == 0
    ffff = by["max_hamming_ffff"]
    assert len(ffff[6]) == len(ffff[1])  # every left keypoint is matched, candidates or not
    edge = by["hamming_edge"][6]
    assert sorted(edge[:, 0].tolist()) == [0, 1]  # distances 49 and 50 pass, 51 does not
    ties = by["ties"]
    for rec in ties[6]:
        li, ri = int(rec[0]), int(rec[1])
        dist = lambda j: sum(bin(int(a ^ b)).count("1") for a, b in zip(ties[3][li], ties[4][j]))  # noqa: E731
        lx, ly = ties[1][li][:2]
        cands = [j for j in range(len(ties[2]))
                 if abs(np.float32(ly) - ties[2][j][1]) <= 2.0 and 1.0 <= np.float32(lx) - ties[2][j][0] <= 120.0]
        best = min(dist(j) for j in cands)
        assert ri == min(j for j in cands if dist(j) == best)  # first minimum in right index order
    assert len(by["negative_epipolar"][6]) == 0 and len(by["empty_range"][6]) == 0


def test_tier1_equals_oracle_on_fresh_cases():
    if not oracle.ref_stereo_available():
        pytest.skip("the reference shader is not built here (reference sources not mounted)")
    for seed in range(3):
        lk, rk, ld, rd = vx_sgm.synth_orb_stereo(400 + 37 * seed, 350 + 51 * seed, 100 + seed)
        cfg = dict(max_hamming=40 + 20 * seed, max_epipolar=1.0 + seed)
        a = oracle.stereo_match(lk, rk, ld["desc"], rd["desc"], cfg)
        b = oracle.ref_stereo_match(lk, rk, ld["desc"], rd["desc"], cfg)
        assert np.array_equal(_words(a), _words(b))


def test_synthetic_keypoints_are_seeded():
    a = vx_sgm.synth_orb_stereo(300, 280, 5)
    b = vx_sgm.synth_orb_stereo(300, 280, 5)
    for x, y in zip(a, b):
        assert x.tobytes() == y.tobytes()
    lk, rk, ld, rd = a
    assert lk.dtype.itemsize == 16 and ld.dtype.itemsize == 36 and vx_sgm.STEREO_MATCH_RESULT.itemsize == 28


def test_config_defaults_match_reference():
    """StereoConfig::default (stereomatch.rs:54-69)."""
    c = vx_sgm.StereoConfig()
    assert (c.max_epipolar, c.min_disparity, c.max_disparity, c.max_hamming, c.ratio_thresh) == (
        2.0, 1.0, 120.0, 50, pytest.approx(0.8))
    assert (c.fx, c.fy, c.cx, c.cy, c.baseline) == (600.0, 600.0, 320.0, 240.0, pytest.approx(0.12))


# ---------------------------------------------------------------------------- GPU


@pytest.fixture(scope="module")
def matcher(gpu_ctx):
    m = vx_sgm.StereoMatcher(gpu_ctx)
    yield m
    m.close()


@pytest.fixture(params=["brute", "banded"])
def stereo_form(request, monkeypatch):
    """Runs a test through each matching form: every pair tested (brute), or the
    right keypoints bucketed by row and only the epipolar band scanned (banded;
    it applies where 0 <= max_epipolar < 2^20, elsewhere the brute form runs)."""
    monkeypatch.setenv("VX_STEREO_FORM", request.param)
    return request.param


@pytest.mark.gpu
def test_gpu_equals_reference_fixtures(gpu_ctx, matcher, stereo_form):
    for name, lk, rk, ld, rd, cfg, want in _cases():
        got = matcher.run(gpu_ctx, lk, rk, ld, rd, _lib_cfg(cfg)).matches
        assert _same_records(got, want), name


@pytest.mark.gpu
@pytest.mark.parametrize("n_left,n_right,seed", [(1, 700, 1), (257, 255, 2), (2048, 2048, 3), (5000, 300, 4),
                                                 (300, 9000, 5), (16384, 16384, 6)])
def test_gpu_equals_oracle(gpu_ctx, matcher, stereo_form, n_left, n_right, seed):
    """Single-chunk (few right keypoints) and multi-chunk launches (the keys of a
    tile meet by atomicMin), partial tiles, one left keypoint, 16384 x 16384."""
    lk, rk, ld, rd = vx_sgm.synth_orb_stereo(n_left, n_right, seed)
    cfg = dict(max_hamming=60)
    want = oracle.stereo_match(lk, rk, ld["desc"], rd["desc"], cfg)
    got = matcher.run(gpu_ctx, lk, rk, ld, rd, _lib_cfg(cfg)).matches
    assert len(got) == len(want) and len(want) > 0
    assert _same_records(got, want)


@pytest.mark.gpu
def test_gpu_device_entry_point_and_scratch_reuse(gpu_ctx, matcher, stereo_form):
    """The device-buffer entry point on torch memory, on the context's stream,
    several calls in a row with growing and shrinking sizes and both launch
    shapes: the scratch the kernels restore between calls stays valid."""
    import torch
    dev = torch.device("cuda", 0)
    for i, (nl, nr) in enumerate([(3000, 4000), (100, 200), (6000, 6000), (3000, 4000), (10, 10)]):
        lk, rk, ld, rd = vx_sgm.synth_orb_stereo(nl, nr, 40 + i)
        cfg = vx_sgm.StereoConfig(max_hamming=55, max_epipolar=1.5)
        want = oracle.stereo_match(lk, rk, ld["desc"], rd["desc"], dict(max_hamming=55, max_epipolar=1.5))
        t_lk = torch.from_numpy(lk.view(np.float32).reshape(-1, 4).copy()).to(dev)
        t_rk = torch.from_numpy(rk.view(np.float32).reshape(-1, 4).copy()).to(dev)
        t_ld = torch.from_numpy(ld["desc"].view(np.int32).copy()).to(dev)
        t_rd = torch.from_numpy(rd["desc"].view(np.int32).copy()).to(dev)
        t_out = torch.full((nl, 7), -1, dtype=torch.int32, device=dev)
        t_cnt = torch.full((1,), -1, dtype=torch.int32, device=dev)
        torch.cuda.synchronize()  # inputs and output fills (torch's stream) land before the call
        stream = torch.cuda.ExternalStream(gpu_ctx.stream)
        with torch.cuda.stream(stream):
            matcher.run_device(gpu_ctx, t_lk.data_ptr(), nl, t_rk.data_ptr(), nr, t_ld.data_ptr(),
                               t_rd.data_ptr(), cfg, t_out.data_ptr(), t_cnt.data_ptr(), stream=gpu_ctx.stream)
        stream.synchronize()
        n = int(t_cnt.item())
        assert n == len(want)
        got = t_out[:n].cpu().numpy().view(np.uint32)
        assert _same_records(got, want), (nl, nr)


@pytest.mark.gpu
def test_gpu_is_deterministic(gpu_ctx, matcher, stereo_form):
    lk, rk, ld, rd = vx_sgm.synth_orb_stereo(4096, 4096, 77, height=16)  # many candidates and ties
    cfg = vx_sgm.StereoConfig(max_hamming=128)
    a = matcher.run(gpu_ctx, lk, rk, ld, rd, cfg).matches
    for _ in range(3):
        assert a.tobytes() == matcher.run(gpu_ctx, lk, rk, ld, rd, cfg).matches.tobytes()
    want = oracle.stereo_match(lk, rk, ld["desc"], rd["desc"], dict(max_hamming=128))
    assert _same_records(a, want)


@pytest.mark.gpu
def test_gpu_argument_checks(gpu_ctx, matcher):
    lk, rk, ld, rd = vx_sgm.synth_orb_stereo(10, 10, 1)
    with pytest.raises(vx_sgm.VxError, match="left_kpts and left_descs length mismatch"):
        matcher.run(gpu_ctx, lk, rk, ld[:9], rd)
    with pytest.raises(vx_sgm.VxError, match="right_kpts and right_descs length mismatch"):
        matcher.run(gpu_ctx, lk, rk[:9], ld, rd)
    assert len(matcher.run(gpu_ctx, lk[:0], rk, ld[:0], rd).matches) == 0
    import torch
    buf = torch.zeros(1024, dtype=torch.int32, device="cuda:0")
    p = buf.data_ptr()
    with pytest.raises(vx_sgm.VxError, match="16-byte aligned"):
        matcher.run_device(gpu_ctx, p + 4, 4, p + 256, 4, p + 512, p + 768, vx_sgm.StereoConfig(), p + 1024,
                           p + 2000, stream=None)


ROW_BUCKETS = 8192


def _band_covers(ly, ry, e):
    """The banded kernel's choice for left y `ly` and right y `ry` (float32
    arrays), emulated in float32: True where ry lies in the rows the left
    keypoint scans or in the special bucket it always scans."""
    f = np.float32
    special = ~((ry >= f(0)) & (ry < f(ROW_BUCKETS)))
    bucket = np.where(special, 0, np.floor(np.where(special, 0, ry))).astype(np.int64)
    in_range = np.abs(ly) < f(4194304.0)
    with np.errstate(invalid="ignore", over="ignore"):
        fa = np.floor(np.where(in_range, ly - e, 0)).astype(f)
        fb = np.floor(np.where(in_range, ly + e, 0)).astype(f)
        lo = fa.astype(np.int64) - 1
        hi = fb.astype(np.int64) + 1
        below = np.nextafter(fa, f(-np.inf))
        lo += (fa >= f(1)) & ~(np.abs(ly - below) <= e)
        hi -= ~(np.abs(ly - (fb + f(1))) <= e)
    lo = np.maximum(lo, 0)
    hi = np.minimum(hi, ROW_BUCKETS - 1)
    return special | (in_range & (bucket >= lo) & (bucket <= hi))


def test_band_bounds_cover_the_epipolar_test():
    """Every (left, right) pair that passes |yl - yr| <= e in float32 is scanned
    by the banded form, for 0 <= e < 2^20: random and adversarial values
    (bucket borders, one ulp off, large and tiny magnitudes, signed zeros)."""
    rng = np.random.default_rng(11)
    f = np.float32
    n = 2_000_000
    ly = np.concatenate([rng.uniform(-50, 8300, n), rng.uniform(-5e6, 5e6, n // 4),
                         np.round(rng.uniform(0, 8192, n // 4))]).astype(f)
    e = np.concatenate([rng.uniform(0, 8, n), rng.uniform(0, 2 ** 20, n // 4),
                        rng.choice([0.0, -0.0, 0.5, 1.0, 2.0, 2.5], n // 4)]).astype(f)
    m = len(ly)
    # right y at the edge of acceptance: ly +- e nudged by a few ulps either way
    side = rng.choice([-1.0, 1.0], m).astype(f)
    base = (ly + side * e).astype(f)
    steps = rng.integers(-3, 4, m)
    ry = base.copy()
    for k in range(1, 4):
        up = steps >= k
        dn = steps <= -k
        ry[up] = np.nextafter(ry[up], f(np.inf))
        ry[dn] = np.nextafter(ry[dn], f(-np.inf))
    ry[: m // 10] = np.round(ry[: m // 10])  # whole rows (pyramid level 0)
    with np.errstate(invalid="ignore"):
        passes = np.abs(ly - ry) <= e
    assert passes.sum() > m // 4
    covered = _band_covers(ly, ry, e)
    assert np.all(covered[passes]), np.flatnonzero(passes & ~covered)[:5]


@pytest.mark.gpu
@pytest.mark.parametrize("e", [0.0, -0.0, 0.5, 2.0, 7.25, 3000.0, 2.0 ** 20 - 64, 2.0 ** 20])
def test_gpu_banded_edge_geometry(gpu_ctx, matcher, monkeypatch, e):
    """Keypoints on bucket borders, one ulp either side, below row 0, above the
    last bucket, beyond 2^22, subnormal and signed-zero y, with tolerances from
    0 to 2^20 (2^20 runs the brute form): both forms equal the oracle."""
    rng = np.random.default_rng(int(abs(e)) + 3)
    f = np.float32
    n = 3000
    ly = np.concatenate([np.round(rng.uniform(0, 8192, n // 3)), rng.uniform(-40, 8240, n // 3),
                         rng.choice([-0.0, 0.0, 1e-40, -1e-40, 8191.999, 8192.0, 4194304.0, 4194305.0,
                                     -3.0, 5e6, 1e30], n - 2 * (n // 3))]).astype(f)
    ry = np.empty(n, f)
    side = rng.choice([-1.0, 1.0], n).astype(f)
    ry[:] = ly + side * f(min(abs(e), 50.0)) * rng.uniform(0, 1.05, n).astype(f)
    k = rng.integers(-2, 3, n)
    ry[k > 0] = np.nextafter(ry[k > 0], f(np.inf))
    ry[k < 0] = np.nextafter(ry[k < 0], f(-np.inf))
    lx = rng.uniform(100, 700, n).astype(f)
    rx = (lx - rng.uniform(0, 100, n)).astype(f)
    lk = np.zeros((n, 4), f)
    lk[:, 0], lk[:, 1] = lx, ly
    rk = np.zeros((n, 4), f)
    order = rng.permutation(n)
    rk[:, 0], rk[:, 1] = rx[order], ry[order]
    ld = rng.integers(0, 2 ** 32, (n, 8), dtype=np.uint64).astype(np.uint32)
    rd = ld[order].copy()
    rd[:, 0] ^= rng.integers(0, 2 ** 16, n).astype(np.uint32)
    cfg = dict(max_epipolar=e, max_hamming=200)
    want = oracle.stereo_match(lk, rk, ld, rd, cfg)
    assert len(want) > n // 4
    for form in ("brute", "banded"):
        monkeypatch.setenv("VX_STEREO_FORM", form)
        got = matcher.run(gpu_ctx, lk, rk, ld, rd, _lib_cfg(cfg)).matches
        assert _same_records(got, want), form


def _frames(sizes, seed):
    frames = [vx_sgm.synth_orb_stereo(nl, nr, seed + i) for i, (nl, nr) in enumerate(sizes)]
    lo = np.concatenate([[0], np.cumsum([len(f[0]) for f in frames])]).astype(np.uint32)
    ro = np.concatenate([[0], np.cumsum([len(f[1]) for f in frames])]).astype(np.uint32)
    cat = lambda i, dt: np.concatenate([f[i] for f in frames]) if len(frames) else np.zeros(0, dt)  # noqa: E731
    return frames, lo, ro, cat(0, vx_sgm.CORNER_POINT), cat(1, vx_sgm.CORNER_POINT), cat(2, vx_sgm.ORB_OUTPUT), \
        cat(3, vx_sgm.ORB_OUTPUT)


@pytest.mark.gpu
@pytest.mark.parametrize("max_hamming", [60, 0xFFFF])
def test_gpu_frames_equal_per_frame_runs(gpu_ctx, matcher, max_hamming):
    """Many frames in one launch: every frame's matches equal the oracle's for that
    frame alone (frames without left or right keypoints, one keypoint, several
    tiles of left keypoints, several shared-memory stages of right ones)."""
    import torch
    sizes = [(512, 512), (0, 40), (40, 0), (1, 1), (300, 700), (2000, 1100), (700, 2600), (257, 255)] * 3
    frames, lo, ro, lk, rk, ld, rd = _frames(sizes, 300)
    dev = torch.device("cuda", 0)
    t = lambda a, dt: torch.from_numpy(np.ascontiguousarray(a).view(dt).copy()).to(dev)  # noqa: E731
    t_lk, t_rk = t(lk, np.float32), t(rk, np.float32)
    t_ld, t_rd = t(ld["desc"], np.int32), t(rd["desc"], np.int32)
    t_out = torch.full((int(lo[-1]), 7), -1, dtype=torch.int32, device=dev)
    t_cnt = torch.full((len(sizes),), -1, dtype=torch.int32, device=dev)
    torch.cuda.synchronize()
    cfg = dict(max_hamming=max_hamming)
    for _ in range(2):  # twice: nothing carries over between calls
        matcher.run_frames_device(gpu_ctx, lo, ro, t_lk.data_ptr(), t_rk.data_ptr(), t_ld.data_ptr(),
                                  t_rd.data_ptr(), _lib_cfg(dict(oracle.STEREO_DEFAULTS, **cfg)), t_out.data_ptr(),
                                  t_cnt.data_ptr(), stream=None)
        out = t_out.cpu().numpy().view(np.uint32)
        cnt = t_cnt.cpu().numpy()
        for f, (flk, frk, fld, frd) in enumerate(frames):
            want = oracle.stereo_match(flk, frk, fld["desc"], frd["desc"], cfg)
            assert cnt[f] == len(want), f
            assert _same_records(out[lo[f]:lo[f] + cnt[f]], want), f


@pytest.mark.gpu
def test_gpu_frames_argument_checks(gpu_ctx, matcher):
    """Offsets are checked on the host before anything runs."""
    import torch
    cnt = torch.zeros(4, dtype=torch.int32, device="cuda:0")
    cfg = vx_sgm.StereoConfig()
    with pytest.raises(vx_sgm.VxError, match="start at 0"):
        matcher.run_frames_device(gpu_ctx, [1, 2], [0, 2], 0, 0, 0, 0, cfg, 0, cnt.data_ptr())
    with pytest.raises(vx_sgm.VxError, match="decrease"):
        matcher.run_frames_device(gpu_ctx, [0, 5, 3], [0, 1, 2], 0, 0, 0, 0, cfg, 0, cnt.data_ptr())


@pytest.mark.gpu
def test_gpu_matcher_shared_between_host_threads(gpu_ctx, matcher):
    """StereoMatcher is Send + Sync in the reference (stereomatch.rs:338-339): calls
    from several host threads on one matcher (the library serialises them on its
    scratch) each return their own frame's matches."""
    import threading
    frames = [vx_sgm.synth_orb_stereo(600 + 50 * i, 700, 900 + i) for i in range(6)]
    want = [oracle.stereo_match(lk, rk, ld["desc"], rd["desc"]) for lk, rk, ld, rd in frames]
    got = [None] * len(frames)
    errors = []

    def work(i):
        try:
            for _ in range(5):
                lk, rk, ld, rd = frames[i]
                got[i] = matcher.run(gpu_ctx, lk, rk, ld, rd, vx_sgm.StereoConfig()).matches
        except Exception as e:  # noqa: BLE001 (reported below)
            errors.append(e)

    threads = [threading.Thread(target=work, args=(i,)) for i in range(len(frames))]
    for t in threads:
        t.start()
    for t in threads:
        t.join()
    assert not errors, errors
    for g, w in zip(got, want):
        assert _same_records(g, w)
