"""CPU tests of the C ABI: the library loads, exports every function that
include/*.h declares, and its host-side logic (config defaults, validation of
arguments, error reporting) behaves like the reference's (no kernel launches)."""
import ctypes
import os
import re

import numpy as np
import pytest

import vx_sgm

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_functions():
    names = []
    for fn in sorted(os.listdir(os.path.join(REPO, "include"))):
        if not fn.endswith(".h"):
            continue
        src = open(os.path.join(REPO, "include", fn)).read()
        src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
        src = re.sub(r"//[^\n]*", "", src)
        for m in re.finditer(r"\b(vx_\w+)\s*\(", src):
            names.append(m.group(1))
    return sorted(set(names))


def test_every_declared_symbol_is_exported():
    lib = ctypes.CDLL(vx_sgm.LIB_PATH)
    names = declared_functions()
    assert len(names) >= 20
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing


def test_config_defaults_match_reference():
    # SGMStereoConfig::default(), vx-vision/src/kernels/sgm.rs:39-49
    c = vx_sgm.SGMStereoConfig.from_c_default()
    assert (c.num_disparities, c.p1, c.p2, c.census_radius_x, c.census_radius_y) == (128, 10.0, 120.0, 4, 3)
    # extensions default to the reference's behaviour: 2 paths, subpixel on, no LR check
    assert (c.num_paths, c.subpixel, c.lr_check) == (2, True, False)
    assert vx_sgm.SGMStereoConfig.new(64).num_disparities == 64


def test_workspace_bytes_formula():
    cfg = vx_sgm.SGMStereoConfig(num_disparities=64, census_radius_x=2, census_radius_y=2, num_paths=4)
    b = vx_sgm.workspace_bytes(640, 480, cfg)
    # guarded row-major census planes + 32-row banded copies (480 = 15 bands)
    # + byte slabs (Dv = 64) + u16 shadow slabs (Dp = 64) + the cost volume (Dv bytes a pixel)
    al = lambda v: (v + 255) // 256 * 256
    assert b == (2 * al(640 * 480 * 4 + 2 * 352 * 4) + 2 * 640 * 480 * 4 + 640 * 480 * 64 * 4
                 + 640 * 480 * 64 * 4 * 2 + 640 * 480 * 64)
    # 9x7 census -> u64 words; D = 60 -> Dp = 64 (u16 shadow), Dv = 64 (bytes)
    cfg64 = vx_sgm.SGMStereoConfig(num_disparities=60, num_paths=8)
    assert vx_sgm.workspace_bytes(100, 10, cfg64) == (2 * al(1000 * 8 + 2 * 352 * 8) + 2 * al(32 * 100 * 8)
                                                      + 1000 * 64 * 8 + 1000 * 64 * 8 * 2 + 1000 * 64)
    # D = 72: Dp = 72 for the shadow, Dv = 80 for the byte vectors
    cfg72 = vx_sgm.SGMStereoConfig(num_disparities=72, census_radius_x=2, census_radius_y=2, num_paths=2)
    assert vx_sgm.workspace_bytes(100, 10, cfg72) == (2 * al(1000 * 4 + 2 * 352 * 4) + 2 * al(32 * 100 * 4)
                                                      + al(1000 * 80 * 2) + al(1000 * 72 * 2 * 2)
                                                      + al(1000 * 80))
    # P2 > 190: most costs exceed a byte, so the vectors go to u16 slabs alone
    cfg_wide = vx_sgm.SGMStereoConfig(num_disparities=72, census_radius_x=2, census_radius_y=2,
                                      num_paths=2, p2=191.0)
    assert vx_sgm.workspace_bytes(100, 10, cfg_wide) == (2 * al(1000 * 4 + 2 * 352 * 4)
                                                         + 2 * al(32 * 100 * 4) + al(1000 * 72 * 2 * 2)
                                                         + al(1000 * 80))


def test_workspace_follows_the_slab_format(monkeypatch):
    cfg = vx_sgm.SGMStereoConfig(num_disparities=64, census_radius_x=2, census_radius_y=2, num_paths=4)
    auto = vx_sgm.workspace_bytes(640, 480, cfg)          # P2 = 120: byte slabs + shadow
    monkeypatch.setenv("VX_SGM_SLAB_FORMAT", "wide")
    assert vx_sgm.workspace_bytes(640, 480, cfg) == auto - 640 * 480 * 64 * 4
    monkeypatch.setenv("VX_SGM_SLAB_FORMAT", "bytes")
    assert vx_sgm.workspace_bytes(640, 480, vx_sgm.SGMStereoConfig(
        num_disparities=64, census_radius_x=2, census_radius_y=2, num_paths=4, p2=1000.0)) == auto


def test_context_without_gpu_reports_device_not_found():
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    with pytest.raises(vx_sgm.VxError) as ei:
        vx_sgm.Context(0)
    assert ei.value.status == 1  # VX_ERR_DEVICE_NOT_FOUND
    assert "device" in vx_sgm.last_error().lower()


def test_null_arguments_are_rejected_without_crashing():
    lib = ctypes.CDLL(vx_sgm.LIB_PATH)
    lib.vx_sgm_compute_disparity.restype = ctypes.c_int
    r = lib.vx_sgm_compute_disparity(None, None, None, None, None, None, None, None)
    assert r == 10  # VX_ERR_INVALID_ARGUMENT
    lib.vx_ctx_create.restype = ctypes.c_int
    assert lib.vx_ctx_create(0, None) == 10


def test_status_names_cover_header():
    src = open(os.path.join(REPO, "include", "vx_sgm.h")).read()
    codes = {int(v): k for k, v in re.findall(r"(VX_(?:OK|ERR_\w+))\s*=\s*(\d+)", src)}
    assert codes == vx_sgm.STATUS_NAMES


def test_noalloc_rejects_misaligned_outputs_before_any_launch():
    """vx_sgm_compute_disparity_noalloc checks the output planes' alignment itself
    (the WTA kernel stores whole floats and int16s): an odd pointer or pitch is
    VX_ERR_INVALID_ARGUMENT, returned before any device work. The pointers here are
    never dereferenced."""
    lib = ctypes.CDLL(vx_sgm.LIB_PATH)
    fn = lib.vx_sgm_compute_disparity_noalloc
    fn.restype = ctypes.c_int
    fn.argtypes = [ctypes.c_void_p, ctypes.c_size_t, ctypes.c_void_p, ctypes.c_size_t, ctypes.c_uint32,
                   ctypes.c_uint32, ctypes.c_void_p, ctypes.c_size_t, ctypes.c_void_p, ctypes.c_size_t,
                   ctypes.c_void_p, ctypes.c_void_p]
    cfg = vx_sgm.SGMStereoConfig(num_disparities=16).to_c()
    w, h = 33, 8
    launches = vx_sgm.kernel_launch_count()
    base = 1 << 20                                    # aligned stand-in addresses
    cases = [
        (base + 2, 4 * w, 0, 0),                      # f32 plane not 4-byte aligned
        (base, 4 * w + 2, 0, 0),                      # f32 pitch not a multiple of 4
        (base, 4 * w, base + 1, 2 * w),               # i16 plane not 2-byte aligned
        (base, 4 * w, base, 2 * w + 1),               # i16 pitch odd
    ]
    for f32, f32_pitch, i16, i16_pitch in cases:
        r = fn(base, w, base, w, w, h, f32, f32_pitch, i16 or None, i16_pitch, ctypes.addressof(cfg), None)
        assert r == 10, (f32, f32_pitch, i16, i16_pitch)        # VX_ERR_INVALID_ARGUMENT
        assert "misaligned" in vx_sgm.last_error()
    assert vx_sgm.kernel_launch_count() == launches


def test_noalloc_wrapper_checks_sizes_and_formats():
    """The Python wrapper passes one width and height for all planes, so it rejects
    textures of other sizes or formats before calling the library."""
    T = vx_sgm.Texture
    left = T(None, None, 40, 20, vx_sgm.FORMAT_U8)
    right = T(None, None, 40, 20, vx_sgm.FORMAT_U8)
    out = T(None, None, 40, 20, vx_sgm.FORMAT_F32)
    cfg = vx_sgm.SGMStereoConfig(num_disparities=16)
    bad = [
        dict(right=T(None, None, 39, 20, vx_sgm.FORMAT_U8)),              # narrower right image
        dict(output=T(None, None, 40, 19, vx_sgm.FORMAT_F32)),            # shorter output
        dict(output_i16=T(None, None, 20, 20, vx_sgm.FORMAT_I16)),        # smaller integer output
        dict(output=T(None, None, 40, 20, vx_sgm.FORMAT_I16)),            # wrong output format
        dict(right=T(None, None, 40, 20, vx_sgm.FORMAT_F32)),             # wrong input format
        dict(output_i16=T(None, None, 40, 20, vx_sgm.FORMAT_F32)),
    ]
    for b in bad:
        args = dict(left=left, right=right, output=out, output_i16=None, **{})
        args.update(b)
        with pytest.raises(vx_sgm.VxError) as e:
            vx_sgm.compute_disparity_noalloc(args["left"], args["right"], args["output"], cfg,
                                             output_i16=args["output_i16"])
        assert e.value.status in (5, 10), b      # VX_ERR_SIZE_MISMATCH / VX_ERR_INVALID_ARGUMENT


def test_allocation_counter_is_exported():
    assert vx_sgm.memory_allocation_count() >= 0
