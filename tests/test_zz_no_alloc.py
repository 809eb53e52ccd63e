"""The no-allocation entry point (vx_sgm_compute_disparity_noalloc).

It serves callers that cannot allocate device memory during a call (a host that
owns all GPU memory through its own allocator, a real-time loop that must not
take cudaMalloc's implicit synchronisation, a plugin whose host forbids
allocation): its scratch is a static 64 MiB device array. This file is named to
be collected last, so that a stop at its first failure has run every other test.
"""
import ctypes

import numpy as np
import pytest
import torch

import vx_sgm
from gpu_helpers import SUBPIXEL_TOL

pytestmark = pytest.mark.gpu


def _outputs(ctx, w, h):
    return ctx.texture_output_r32float(w, h), ctx.texture_output_i16(w, h)


def test_noalloc_matches_pool_entry_point_on_two_calls():
    ctx = vx_sgm.Context(0)
    sgm = vx_sgm.SGMStereo(ctx)
    torch.cuda.set_device(0)
    w, h = 320, 240
    L, R, _ = vx_sgm.synth_pair(vx_sgm.SCENE_PLANES, w, h, 4, 60, 31)
    cfg = vx_sgm.SGMStereoConfig(num_disparities=64, census_radius_x=2, census_radius_y=2,
                                 num_paths=4, lr_check=True)
    assert vx_sgm.workspace_bytes(w, h, cfg) < vx_sgm.static_scratch_bytes()
    tl, tr = ctx.texture_gray8(L, w, h), ctx.texture_gray8(R, w, h)
    ref_f, ref_i = _outputs(ctx, w, h)
    sgm.compute_disparity(ctx, tl, tr, ref_f, cfg, output_i16=ref_i)
    want_f, want_i = ref_f.read_r32float(), ref_i.download()

    # Two calls in a row (different inputs in between would also share the array).
    for call in range(2):
        out_f, out_i = _outputs(ctx, w, h)
        allocs = vx_sgm.memory_allocation_count()
        vx_sgm.compute_disparity_noalloc(tl, tr, out_f, cfg, output_i16=out_i)
        # the library's own allocation counter: neither call (the first does the
        # device set-up) asks for device or pinned memory
        assert vx_sgm.memory_allocation_count() == allocs, f"call {call} allocated"
        got_f, got_i = out_f.read_r32float(), out_i.download()
        assert np.array_equal(got_i, want_i), f"call {call}: integer disparity differs"
        assert np.abs(got_f - want_f).max() <= SUBPIXEL_TOL, f"call {call}: subpixel differs"


def test_noalloc_rejects_pairs_larger_than_the_scratch():
    ctx = vx_sgm.Context(0)
    w, h = 1242, 375
    cfg = vx_sgm.SGMStereoConfig(num_disparities=128, num_paths=8)
    assert vx_sgm.workspace_bytes(w, h, cfg) > vx_sgm.static_scratch_bytes()
    tl = vx_sgm.Texture.create(ctx, w, h, vx_sgm.FORMAT_U8)
    tr = vx_sgm.Texture.create(ctx, w, h, vx_sgm.FORMAT_U8)
    of = ctx.texture_output_r32float(w, h)
    with pytest.raises(vx_sgm.VxError) as e:
        vx_sgm.compute_disparity_noalloc(tl, tr, of, cfg)
    assert e.value.status == 8  # VX_ERR_BUDGET
    assert "scratch" in e.value.message
