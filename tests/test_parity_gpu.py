"""GPU parity: the CUDA path through the C ABI against the reference's own outputs
(golden fixtures) and against the oracle. Integers bit-exact; subpixel within 1e-4 px."""
import numpy as np
import pytest

import oracle
import vx_sgm
from gpu_helpers import assert_disparity_equal, cfg_pair, run_batch, run_pair

pytestmark = pytest.mark.gpu


def test_golden_reference_cases(gpu_ctx, sgm, golden, agg_form):
    """Reference configuration (2 paths, subpixel, no LR) reproduces the reference shader's
    census words, cost volume and f32 disparity bit for bit."""
    for c in golden:
        cfg = vx_sgm.SGMStereoConfig(num_disparities=c["nd"], p1=c["p1"], p2=c["p2"],
                                     census_radius_x=c["rx"], census_radius_y=c["ry"])
        h, w = c["left"].shape
        tl = gpu_ctx.texture_gray8(c["left"], w, h)
        tr = gpu_ctx.texture_gray8(c["right"], w, h)
        cl, cr, L, S = sgm.debug_dump(gpu_ctx, tl, tr, cfg)
        assert np.array_equal(cl, c["census_l"]) and np.array_equal(cr, c["census_r"]), c["name"]
        assert int(S.astype(np.uint64).sum()) == int(c["S_sum"][0]), c["name"]
        if c["S"] is not None:
            assert np.array_equal(S, c["S"]), c["name"]
        out = gpu_ctx.texture_output_r32float(w, h)
        sgm.compute_disparity(gpu_ctx, tl, tr, out, cfg)
        d = out.read_r32float()
        assert np.array_equal(d.view(np.uint32), c["disparity"].view(np.uint32)), c["name"]


@pytest.mark.parametrize("nd,rx,ry,w,h", [
    (64, 2, 2, 77, 41), (128, 2, 2, 150, 33), (192, 4, 3, 213, 29), (256, 2, 2, 300, 20),
    (48, 4, 3, 61, 37), (100, 1, 1, 90, 31), (7, 2, 2, 19, 13), (1, 1, 1, 9, 7),
])
def test_each_path_bit_exact(gpu_ctx, sgm, nd, rx, ry, w, h, agg_form):
    """All 8 path directions' L_r, dumped from the path slabs, equal the oracle's."""
    L, R, _ = vx_sgm.synth_pair(0, w, h, 0, max(1, nd - 4), nd * 1000 + w)
    cfg, _ = cfg_pair(num_disparities=nd, census_radius_x=rx, census_radius_y=ry, num_paths=8)
    tl = gpu_ctx.texture_gray8(L, w, h)
    tr = gpu_ctx.texture_gray8(R, w, h)
    cl, cr, Lg, S = sgm.debug_dump(gpu_ctx, tl, tr, cfg)
    ocl, ocr = oracle.census(L, rx, ry), oracle.census(R, rx, ry)
    assert np.array_equal(cl, ocl) and np.array_equal(cr, ocr)
    for k in range(8):
        dx, dy = oracle.path_dir(k)
        want = oracle.path_costs(ocl, ocr, nd, 10, 120, dx, dy)
        bad = np.argwhere(Lg[k] != want)
        assert bad.size == 0, f"path {k} ({dx},{dy}) differs at {bad[:5]}"


@pytest.mark.parametrize("case", [
    dict(scene=0, w=640, h=480, lo=4, hi=60, num_disparities=64, census_radius_x=2,
         census_radius_y=2, num_paths=4, lr_check=True),                       # 640x480 D=64 4 paths LR
    dict(scene=1, w=1242, h=375, lo=0, hi=120, num_disparities=128, census_radius_x=2,
         census_radius_y=2, num_paths=8, lr_check=True),                       # 1242x375 D=128 8 paths LR
    dict(scene=2, w=512, h=384, lo=0, hi=250, num_disparities=256, census_radius_x=2,
         census_radius_y=2, num_paths=8, lr_check=True),                       # D=256, textureless patches
    dict(scene=0, w=320, h=240, lo=4, hi=60, num_disparities=64, census_radius_x=4,
         census_radius_y=3, num_paths=2),                                      # reference defaults
    dict(scene=0, w=333, h=111, lo=2, hi=90, num_disparities=96, census_radius_x=3,
         census_radius_y=2, num_paths=8, p1=15, p2=300, lr_check=True,
         lr_tolerance=0),                                                      # u16-range values
])
def test_full_pipeline_matches_oracle(gpu_ctx, sgm, case, agg_form):
    case = dict(case)
    scene, w, h, lo, hi = (case.pop(k) for k in ("scene", "w", "h", "lo", "hi"))
    L, R, _ = vx_sgm.synth_pair(scene, w, h, lo, hi, 42)
    cfg, ocfg = cfg_pair(**case)
    got = run_pair(gpu_ctx, sgm, L, R, cfg)
    d, di, _ = oracle.sgm(L, R, ocfg)
    assert_disparity_equal(got, (d, di), what=str(case))


def test_edge_shapes(gpu_ctx, sgm, agg_form):
    for (w, h, nd) in [(1, 1, 1), (1, 17, 8), (23, 1, 16), (5, 9, 64), (16384, 2, 8), (2, 300, 256)]:
        L, R, _ = vx_sgm.synth_pair(0, w, h, 0, max(0, min(nd - 1, w - 1)), w * 7 + h)
        cfg, ocfg = cfg_pair(num_disparities=nd, census_radius_x=2, census_radius_y=2,
                             num_paths=8, lr_check=True)
        got = run_pair(gpu_ctx, sgm, L, R, cfg)
        d, di, _ = oracle.sgm(L, R, ocfg)
        assert_disparity_equal(got, (d, di), what=f"{w}x{h} D={nd}")


@pytest.mark.parametrize("rx,ry", [(2, 2), (4, 3), (3, 4), (0, 3), (31, 0), (10, 1), (5, 2), (20, 0), (1, 1)])
def test_census_staging_forms_match_oracle(gpu_ctx, sgm, rx, ry):
    """Interior census tiles of 16-byte aligned views are staged with cp.async, border tiles
    and unaligned views byte by byte with clamped coordinates: both give the oracle's words
    (vx-vision/shaders/SGMStereo.metal:25-66) for an aligned texture and for a wrapped one
    whose base and pitch are odd."""
    import torch
    w, h = 301, 141
    L, R, _ = vx_sgm.synth_pair(1, w, h, 0, 12, rx * 100 + ry)
    cfg = vx_sgm.SGMStereoConfig(num_disparities=16, census_radius_x=rx, census_radius_y=ry, num_paths=2)
    want_l, want_r = oracle.census(L, rx, ry), oracle.census(R, rx, ry)
    tl, tr = gpu_ctx.texture_gray8(L, w, h), gpu_ctx.texture_gray8(R, w, h)
    assert tl.pitch % 16 == 0
    cl, cr, _, _ = sgm.debug_dump(gpu_ctx, tl, tr, cfg)
    assert np.array_equal(cl, want_l) and np.array_equal(cr, want_r)
    pitch = w + 1
    bufs = [torch.zeros(pitch * h + 1, dtype=torch.uint8, device="cuda") for _ in range(2)]
    wl, wr = (vx_sgm.Texture.wrap_device(gpu_ctx, b.data_ptr() + 1, pitch, w, h, vx_sgm.FORMAT_U8) for b in bufs)
    wl.upload(L)
    wr.upload(R)
    cl2, cr2, _, _ = sgm.debug_dump(gpu_ctx, wl, wr, cfg)
    assert np.array_equal(cl2, want_l) and np.array_equal(cr2, want_r)
    torch.cuda.synchronize()
    del wl, wr, bufs


@pytest.mark.parametrize("nd,paths,p2", [
    (128, 8, 120), (129, 2, 120), (144, 8, 300), (160, 4, 120), (192, 8, 300), (193, 4, 120),
    (208, 8, 120), (248, 2, 300), (256, 4, 300), (80, 8, 300), (24, 4, 120),
])
def test_wta_lane_forms_match_oracle(gpu_ctx, sgm, nd, paths, p2):
    """The WTA's row-loop forms (16 disparities a lane; 8 a lane where D = 129..192
    fills its lanes better; padded right-view keys) on each side of the form
    boundaries, every path count, with LR and with escaped byte vectors (P2 = 300
    lifts path costs past a byte)."""
    w, h = 233, 19
    L, R, _ = vx_sgm.synth_pair(nd % 3, w, h, 0, nd - 3, nd * 31 + paths)
    for lr in (True, False):
        cfg, ocfg = cfg_pair(num_disparities=nd, census_radius_x=2, census_radius_y=2, num_paths=paths,
                             p1=15 if p2 == 300 else 10, p2=p2, lr_check=lr, lr_tolerance=1)
        got = run_pair(gpu_ctx, sgm, L, R, cfg)
        d, di, _ = oracle.sgm(L, R, ocfg)
        assert_disparity_equal(got, (d, di), what=f"D={nd} P={paths} p2={p2} lr={lr}")


def test_batch_equals_solo(gpu_ctx, sgm, agg_form):
    rng = np.random.default_rng(1)
    pairs, cfgs = [], []
    for i in range(9):
        w, h = int(rng.integers(20, 200)), int(rng.integers(10, 120))
        nd = int(rng.choice([16, 64, 128, 192, 33]))
        L, R, _ = vx_sgm.synth_pair(i % 3, w, h, 0, max(1, nd - 2), 100 + i)
        pairs.append((L, R))
        cfgs.append(vx_sgm.SGMStereoConfig(num_disparities=nd, census_radius_x=int(rng.integers(0, 4)),
                                           census_radius_y=int(rng.integers(0, 3)),
                                           num_paths=int(rng.choice([2, 4, 8])),
                                           lr_check=bool(i % 2), p1=float(rng.integers(0, 30)),
                                           p2=float(rng.integers(30, 400))))
    batch = run_batch(gpu_ctx, sgm, pairs, cfgs)
    for (L, R), cfg, got in zip(pairs, cfgs, batch):
        solo = run_pair(gpu_ctx, sgm, L, R, cfg)
        assert_disparity_equal(got, solo, tol=0.0, what="batch vs solo")
        _, ocfg = cfg_pair(**{k: getattr(cfg, k) for k in cfg.__dataclass_fields__})
        d, di, _ = oracle.sgm(L, R, ocfg)
        assert_disparity_equal(got, (d, di), what="batch vs oracle")


def test_invalid_arguments(gpu_ctx, sgm):
    L, R, _ = vx_sgm.synth_pair(0, 32, 16, 1, 8, 1)
    tl = gpu_ctx.texture_gray8(L, 32, 16)
    tr_small = gpu_ctx.texture_gray8(R[:, :31], 31, 16)
    out = gpu_ctx.texture_output_r32float(32, 16)
    with pytest.raises(vx_sgm.VxError) as e:
        sgm.compute_disparity(gpu_ctx, tl, tr_small, out, vx_sgm.SGMStereoConfig.new(16))
    assert e.value.status == 5  # VX_ERR_SIZE_MISMATCH
    tr = gpu_ctx.texture_gray8(R, 32, 16)
    for bad in (dict(num_disparities=0), dict(num_disparities=257),
                dict(census_radius_x=5, census_radius_y=3), dict(num_paths=3), dict(p1=-1.0),
                dict(p2=float("nan"))):
        with pytest.raises(vx_sgm.VxError) as e:
            sgm.compute_disparity(gpu_ctx, tl, tr, out, vx_sgm.SGMStereoConfig(**{"num_disparities": 16, **bad}))
        assert e.value.status == 6, bad  # VX_ERR_INVALID_CONFIG


def test_kernels_actually_launch(gpu_ctx, sgm):
    L, R, _ = vx_sgm.synth_pair(0, 64, 32, 1, 20, 3)
    before = vx_sgm.kernel_launch_count()
    run_pair(gpu_ctx, sgm, L, R, vx_sgm.SGMStereoConfig(num_disparities=32, num_paths=8))
    assert vx_sgm.kernel_launch_count() - before >= 3  # census, [cost volume,] aggregation, WTA
