"""Helpers shared by the GPU tests: run one pair or a batch through the C ABI."""
import numpy as np

import oracle
import vx_sgm


def cfg_pair(**kw):
    """(library config, oracle config) with the same fields."""
    c = vx_sgm.SGMStereoConfig(**kw)
    o = oracle.config(**{k: getattr(c, k) for k in (
        "num_disparities", "p1", "p2", "census_radius_x", "census_radius_y", "num_paths",
        "subpixel", "lr_check", "lr_tolerance", "invalid_value")})
    return c, o


def run_pair(ctx, sgm, left, right, cfg):
    h, w = left.shape
    tl = ctx.texture_gray8(left, w, h)
    tr = ctx.texture_gray8(right, w, h)
    out = ctx.texture_output_r32float(w, h)
    oi = ctx.texture_output_i16(w, h)
    sgm.compute_disparity(ctx, tl, tr, out, cfg, output_i16=oi)
    return out.read_r32float(), oi.download()


def run_batch(ctx, sgm, pairs, cfgs):
    tl, tr, of, oi = [], [], [], []
    for (left, right) in pairs:
        h, w = left.shape
        tl.append(ctx.texture_gray8(left, w, h))
        tr.append(ctx.texture_gray8(right, w, h))
        of.append(ctx.texture_output_r32float(w, h))
        oi.append(ctx.texture_output_i16(w, h))
    sgm.compute_batch(ctx, tl, tr, of, cfgs, outputs_i16=oi)
    return [(f.read_r32float(), i.download()) for f, i in zip(of, oi)]


SUBPIXEL_TOL = 1e-4  # px; the kernels use IEEE division, so results are expected bit-equal


def assert_disparity_equal(got, want, tol=SUBPIXEL_TOL, what=""):
    (gf, gi), (wf, wi) = got, want
    assert np.array_equal(gi, wi), f"{what}: integer disparity differs at {np.argwhere(gi != wi)[:5]}"
    diff = np.abs(gf.astype(np.float64) - wf.astype(np.float64))
    assert diff.max() <= tol, f"{what}: subpixel max diff {diff.max()} at {np.unravel_index(diff.argmax(), diff.shape)}"
