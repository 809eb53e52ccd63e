"""GPU parity of the two per-path slab formats. Byte slabs hold a vector as bytes
unless it escapes (some value is 255 or more; 0xFF in byte 0 is the escape
marker), in which case the exact u16 vector goes to the shadow slab; wide slabs
hold every vector as u16. The format follows P2 by default; VX_SGM_SLAB_FORMAT
forces one, so each format also runs on the configurations that normally pick
the other: byte slabs with P2 >= 191 escape on most vectors, including vectors
whose largest value is exactly 255 (the marker value)."""
import numpy as np
import pytest

import oracle
import vx_sgm
from gpu_helpers import assert_disparity_equal, cfg_pair, run_pair

pytestmark = pytest.mark.gpu

FORMATS = ("bytes", "wide")

# (w, h, nd, rx, ry, p1, p2, seed): default P2 (rare escapes from wrapped
# values), P2 = 240 (most vectors escape; hundreds of vectors peak at exactly
# 255), P2 = 2000 (values far above a byte).
CASES = [
    (160, 90, 64, 2, 2, 10, 120, 1),
    (200, 100, 64, 2, 2, 10, 240, 3),
    (120, 64, 48, 4, 3, 6, 2000, 5),
    (150, 40, 200, 2, 2, 10, 120, 9),   # Dv = 208 > Dp = 200: the last byte chunk is half used
]


def _escape_stats(Lk):
    """Vectors of one path slab that byte slabs must escape, and those whose
    largest value is exactly the marker value 255."""
    mx = Lk.max(axis=-1)
    return int((mx >= 255).sum()), int((mx == 255).sum())


@pytest.mark.parametrize("fmt", FORMATS)
@pytest.mark.parametrize("case", CASES)
def test_paths_bit_exact_in_both_formats(gpu_ctx, sgm, monkeypatch, fmt, case, agg_form):
    w, h, nd, rx, ry, p1, p2, seed = case
    monkeypatch.setenv("VX_SGM_SLAB_FORMAT", fmt)
    L, R, _ = vx_sgm.synth_pair(0, w, h, 2, max(1, nd - 4), seed)
    cfg, _ = cfg_pair(num_disparities=nd, census_radius_x=rx, census_radius_y=ry, num_paths=8,
                      p1=float(p1), p2=float(p2))
    tl = gpu_ctx.texture_gray8(L, w, h)
    tr = gpu_ctx.texture_gray8(R, w, h)
    _, _, Lg, S = sgm.debug_dump(gpu_ctx, tl, tr, cfg)
    ocl, ocr = oracle.census(L, rx, ry), oracle.census(R, rx, ry)
    esc = coll = 0
    S_want = np.zeros((h, w, nd), np.uint16)
    for k in range(8):
        dx, dy = oracle.path_dir(k)
        want = oracle.path_costs(ocl, ocr, nd, p1, p2, dx, dy)
        e, c = _escape_stats(want)
        esc, coll = esc + e, coll + c
        bad = np.argwhere(Lg[k] != want)
        assert bad.size == 0, f"{fmt}: path {k} ({dx},{dy}) differs at {bad[:5]}"
        S_want = (S_want + want).astype(np.uint16)
    assert np.array_equal(S, S_want)
    assert esc > 0, "the case must exercise the escape"
    if p2 == 240:
        assert coll > 0, "the case must hold vectors that peak at the marker value"


@pytest.mark.parametrize("fmt", FORMATS)
@pytest.mark.parametrize("case", CASES)
def test_disparity_matches_oracle_in_both_formats(gpu_ctx, sgm, monkeypatch, fmt, case, agg_form):
    """WTA reads escaped vectors from the shadow (byte slabs) or every vector (wide)."""
    w, h, nd, rx, ry, p1, p2, seed = case
    monkeypatch.setenv("VX_SGM_SLAB_FORMAT", fmt)
    L, R, _ = vx_sgm.synth_pair(1, w, h, 2, max(1, nd - 4), seed + 100)
    cfg, ocfg = cfg_pair(num_disparities=nd, census_radius_x=rx, census_radius_y=ry, num_paths=8,
                         p1=float(p1), p2=float(p2), lr_check=True)
    got = run_pair(gpu_ctx, sgm, L, R, cfg)
    d, di, _ = oracle.sgm(L, R, ocfg)
    assert_disparity_equal(got, (d, di), what=f"{fmt} {case}")


@pytest.mark.parametrize("fmt", FORMATS)
def test_golden_cases_in_both_formats(gpu_ctx, sgm, golden, monkeypatch, fmt, agg_form):
    """The reference's own outputs (f32 disparity bits, cost volume) in either format."""
    monkeypatch.setenv("VX_SGM_SLAB_FORMAT", fmt)
    for c in golden:
        cfg = vx_sgm.SGMStereoConfig(num_disparities=c["nd"], p1=c["p1"], p2=c["p2"],
                                     census_radius_x=c["rx"], census_radius_y=c["ry"])
        h, w = c["left"].shape
        tl = gpu_ctx.texture_gray8(c["left"], w, h)
        tr = gpu_ctx.texture_gray8(c["right"], w, h)
        _, _, _, S = sgm.debug_dump(gpu_ctx, tl, tr, cfg)
        assert int(S.astype(np.uint64).sum()) == int(c["S_sum"][0]), (fmt, c["name"])
        out = gpu_ctx.texture_output_r32float(w, h)
        sgm.compute_disparity(gpu_ctx, tl, tr, out, cfg)
        d = out.read_r32float()
        assert np.array_equal(d.view(np.uint32), c["disparity"].view(np.uint32)), (fmt, c["name"])

