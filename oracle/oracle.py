"""ctypes front end of the CPU oracle (liboracle.so) and of the literal reference
shader compiled as C++ (_ref/libsgm_ref.so).

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and the
CPU-baseline leg of bench.py, always as the checker or the timed CPU baseline,
never as the thing measured or shipped.
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE_SO = os.path.join(HERE, "liboracle.so")
REF_SO = os.path.join(HERE, "_ref", "libsgm_ref.so")
_P = ctypes.c_void_p


class OracleConfig(ctypes.Structure):
    _fields_ = [("num_disparities", ctypes.c_int32), ("p1", ctypes.c_float),
                ("p2", ctypes.c_float), ("census_radius_x", ctypes.c_int32),
                ("census_radius_y", ctypes.c_int32), ("num_paths", ctypes.c_int32),
                ("subpixel", ctypes.c_int32), ("lr_check", ctypes.c_int32),
                ("lr_tolerance", ctypes.c_int32), ("invalid_value", ctypes.c_float)]


class OracleStats(ctypes.Structure):
    _fields_ = [("pixel_steps", ctypes.c_uint64), ("wrap_steps", ctypes.c_uint64),
                ("wide_values", ctypes.c_uint64)]


_lib = None
_ref = None


def build():
    subprocess.run(["make", "-s", "-C", HERE], check=True)


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(ORACLE_SO):
            build()
        _lib = ctypes.CDLL(ORACLE_SO)
    return _lib


def ref_available() -> bool:
    return os.path.exists(REF_SO)


def ref_lib():
    global _ref
    if _ref is None:
        _ref = ctypes.CDLL(REF_SO)
    return _ref


def config(num_disparities=128, p1=10.0, p2=120.0, census_radius_x=4, census_radius_y=3,
           num_paths=2, subpixel=True, lr_check=False, lr_tolerance=1, invalid_value=-1.0,
           **_ignored) -> OracleConfig:
    return OracleConfig(int(num_disparities), float(p1), float(p2), int(census_radius_x),
                        int(census_radius_y), int(num_paths), int(bool(subpixel)),
                        int(bool(lr_check)), int(lr_tolerance), float(invalid_value))


def path_dir(k: int):
    dx, dy = ctypes.c_int(), ctypes.c_int()
    lib().oracle_path_dir(k, ctypes.byref(dx), ctypes.byref(dy))
    return dx.value, dy.value


def census(img: np.ndarray, rx: int, ry: int, nthreads: int = 0) -> np.ndarray:
    img = np.ascontiguousarray(img, np.uint8)
    h, w = img.shape
    out = np.zeros((h, w), np.uint64)
    r = lib().oracle_census(_P(img.ctypes.data), ctypes.c_size_t(w), w, h, rx, ry,
                            _P(out.ctypes.data), nthreads)
    if r != 0:
        raise ValueError("oracle_census rejected its arguments")
    return out


def path_costs(cl, cr, nd, p1, p2, dx, dy, nthreads=0):
    """L_r of one path direction, (H, W, D) u16."""
    h, w = cl.shape
    L = np.zeros((h, w, nd), np.uint16)
    r = lib().oracle_path(_P(cl.ctypes.data), _P(cr.ctypes.data), w, h, nd, int(p1), int(p2),
                          dx, dy, _P(L.ctypes.data), None, None, nthreads)
    if r != 0:
        raise ValueError("oracle_path rejected its arguments")
    return L


def sgm(left, right, cfg: OracleConfig, want_S=False, nthreads=0, stats=None):
    """Full pipeline. Returns (disparity f32, disparity i16, S or None)."""
    left = np.ascontiguousarray(left, np.uint8)
    right = np.ascontiguousarray(right, np.uint8)
    h, w = left.shape
    disp = np.zeros((h, w), np.float32)
    di = np.zeros((h, w), np.int16)
    S = np.zeros((h, w, cfg.num_disparities), np.uint16) if want_S else None
    r = lib().oracle_sgm(_P(left.ctypes.data), ctypes.c_size_t(w), _P(right.ctypes.data),
                         ctypes.c_size_t(w), w, h, ctypes.byref(cfg), _P(disp.ctypes.data),
                         _P(di.ctypes.data), _P(S.ctypes.data) if want_S else None,
                         ctypes.byref(stats) if stats is not None else None, nthreads)
    if r != 0:
        raise ValueError("oracle_sgm rejected its arguments")
    return disp, di, S


def wta(S, cfg: OracleConfig, nthreads=0):
    S = np.ascontiguousarray(S, np.uint16)
    h, w, _ = S.shape
    disp = np.zeros((h, w), np.float32)
    di = np.zeros((h, w), np.int16)
    r = lib().oracle_wta(_P(S.ctypes.data), w, h, ctypes.byref(cfg), _P(disp.ctypes.data),
                         _P(di.ctypes.data), nthreads)
    if r != 0:
        raise ValueError("oracle_wta rejected its arguments")
    return disp, di


def reference_sgm(left, right, nd, p1=10.0, p2=120.0, rx=4, ry=3, nthreads=0):
    """The reference shader itself (2 paths, subpixel). Returns (census_l, census_r, S, disp)."""
    left = np.ascontiguousarray(left, np.uint8)
    right = np.ascontiguousarray(right, np.uint8)
    h, w = left.shape
    cl = np.zeros((h, w, 2), np.uint32)
    cr = np.zeros((h, w, 2), np.uint32)
    S = np.zeros((h, w, nd), np.uint16)
    disp = np.zeros((h, w), np.float32)
    r = ref_lib().ref_sgm_compute(_P(left.ctypes.data), _P(right.ctypes.data), w, h, nd,
                                  ctypes.c_float(p1), ctypes.c_float(p2), rx, ry,
                                  _P(cl.ctypes.data), _P(cr.ctypes.data), _P(S.ctypes.data),
                                  _P(disp.ctypes.data), nthreads)
    if r != 0:
        raise ValueError("ref_sgm_compute rejected its arguments")
    as64 = lambda c: c[..., 0].astype(np.uint64) | (c[..., 1].astype(np.uint64) << np.uint64(32))
    return as64(cl), as64(cr), S, disp


# ---- depth-map post-filters (vx-vision/shaders/DepthFilter.metal) ----

REF_DEPTH_SO = os.path.join(HERE, "_ref", "libdepth_ref.so")


def ref_depth_available() -> bool:
    return os.path.exists(REF_DEPTH_SO)


def _f32(a):
    return np.ascontiguousarray(a, np.float32)


def depth_median(depth: np.ndarray, radius: int = 1) -> np.ndarray:
    """Restatement of depth_median (DepthFilter.metal:84-120)."""
    d = _f32(depth)
    h, w = d.shape
    out = np.empty_like(d)
    if lib().oracle_depth_median(_P(d.ctypes.data), _P(out.ctypes.data), w, h, int(radius)) != 0:
        raise ValueError("oracle_depth_median rejected its arguments")
    return out


def depth_bilateral(depth: np.ndarray, radius: int = 3, sigma_spatial: float = 5.0,
                    sigma_depth: float = 0.05) -> np.ndarray:
    """Restatement of depth_bilateral (DepthFilter.metal:20-66)."""
    d = _f32(depth)
    h, w = d.shape
    out = np.empty_like(d)
    f = lib().oracle_depth_bilateral
    f.argtypes = [_P, _P, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_float, ctypes.c_float]
    if f(_P(d.ctypes.data), _P(out.ctypes.data), w, h, int(radius), float(sigma_spatial),
         float(sigma_depth)) != 0:
        raise ValueError("oracle_depth_bilateral rejected its arguments")
    return out


def ref_depth_median(depth: np.ndarray, radius: int = 1) -> np.ndarray:
    """The reference shader itself (tier 1, built where the reference is mounted)."""
    d = _f32(depth)
    h, w = d.shape
    out = np.empty_like(d)
    ctypes.CDLL(REF_DEPTH_SO).ref_depth_median(_P(d.ctypes.data), _P(out.ctypes.data), w, h, int(radius))
    return out


def ref_depth_bilateral(depth: np.ndarray, radius: int, sigma_spatial: float,
                        sigma_depth: float) -> np.ndarray:
    d = _f32(depth)
    h, w = d.shape
    out = np.empty_like(d)
    f = ctypes.CDLL(REF_DEPTH_SO).ref_depth_bilateral
    f.argtypes = [_P, _P, ctypes.c_uint, ctypes.c_uint, ctypes.c_int, ctypes.c_float, ctypes.c_float]
    f(_P(d.ctypes.data), _P(out.ctypes.data), w, h, int(radius), float(sigma_spatial), float(sigma_depth))
    return out


# ---- sparse ORB stereo matcher (vx-vision/shaders/StereoMatch.metal) ----

REF_STEREO_SO = os.path.join(HERE, "_ref", "libstereo_ref.so")

# StereoMatchResult as the host reads it (vx-vision/src/types.rs:64-70).
MATCH_DTYPE = np.dtype([("left_idx", "<u4"), ("right_idx", "<u4"), ("disparity", "<f4"),
                        ("point_3d", "<f4", (3,)), ("_pad", "<f4")])

STEREO_DEFAULTS = dict(max_epipolar=2.0, min_disparity=1.0, max_disparity=120.0, max_hamming=50,
                       ratio_thresh=0.8, fx=600.0, fy=600.0, cx=320.0, cy=240.0, baseline=0.12)


class OracleStereoConfig(ctypes.Structure):
    _fields_ = [("max_epipolar", ctypes.c_float), ("min_disparity", ctypes.c_float),
                ("max_disparity", ctypes.c_float), ("max_hamming", ctypes.c_uint32),
                ("ratio_thresh", ctypes.c_float), ("fx", ctypes.c_float), ("fy", ctypes.c_float),
                ("cx", ctypes.c_float), ("cy", ctypes.c_float), ("baseline", ctypes.c_float)]


def ref_stereo_available() -> bool:
    return os.path.exists(REF_STEREO_SO)


def _stereo_inputs(left_kpts, right_kpts, left_desc, right_desc):
    lk = np.ascontiguousarray(np.asarray(left_kpts).view(np.float32).reshape(-1, 4))
    rk = np.ascontiguousarray(np.asarray(right_kpts).view(np.float32).reshape(-1, 4))
    ld = np.ascontiguousarray(left_desc, np.uint32).reshape(-1, 8)
    rd = np.ascontiguousarray(right_desc, np.uint32).reshape(-1, 8)
    if len(lk) != len(ld) or len(rk) != len(rd):
        raise ValueError("keypoint and descriptor counts differ")
    return lk, rk, ld, rd


def _stereo_cfg(cfg):
    c = dict(STEREO_DEFAULTS)
    c.update(cfg or {})
    return c


def stereo_match(left_kpts, right_kpts, left_desc, right_desc, cfg=None, nthreads=0) -> np.ndarray:
    """Restatement of StereoMatcher::run (stereomatch.rs:115-249): the matches in
    ascending left index. kpts: (n, 4) float32 rows (x, y, response, level bits)
    or CornerPoint records; desc: (n, 8) uint32 words."""
    lk, rk, ld, rd = _stereo_inputs(left_kpts, right_kpts, left_desc, right_desc)
    c = _stereo_cfg(cfg)
    oc = OracleStereoConfig(**{k: c[k] for k, _ in OracleStereoConfig._fields_})
    out = np.zeros(max(len(lk), 1), MATCH_DTYPE)
    f = lib().oracle_stereo_match
    f.argtypes = [_P, ctypes.c_uint32, _P, ctypes.c_uint32, _P, _P, _P, _P, ctypes.c_int]
    n = f(_P(lk.ctypes.data), len(lk), _P(rk.ctypes.data), len(rk), _P(ld.ctypes.data), _P(rd.ctypes.data),
          ctypes.byref(oc), _P(out.ctypes.data), int(nthreads))
    if n < 0:
        raise ValueError("oracle_stereo_match rejected its arguments")
    return out[:n].copy()


def ref_stereo_match(left_kpts, right_kpts, left_desc, right_desc, cfg=None) -> np.ndarray:
    """The reference shader itself (tier 1, built where the reference is mounted):
    stereo_hamming over the full distance matrix, then stereo_extract per left."""
    lk, rk, ld, rd = _stereo_inputs(left_kpts, right_kpts, left_desc, right_desc)
    c = _stereo_cfg(cfg)
    out = np.zeros(max(len(lk), 1), MATCH_DTYPE)
    f = ctypes.CDLL(REF_STEREO_SO).ref_stereo_match
    fl = ctypes.c_float
    f.argtypes = [_P, ctypes.c_uint32, _P, ctypes.c_uint32, _P, _P, fl, fl, fl, ctypes.c_uint32, fl, fl, fl,
                  fl, fl, fl, _P]
    n = f(_P(lk.ctypes.data), len(lk), _P(rk.ctypes.data), len(rk), _P(ld.ctypes.data), _P(rd.ctypes.data),
          c["max_epipolar"], c["min_disparity"], c["max_disparity"], int(c["max_hamming"]) & 0xFFFFFFFF,
          c["ratio_thresh"], c["fx"], c["fy"], c["cx"], c["cy"], c["baseline"], _P(out.ctypes.data))
    return out[:n].copy()


# ---------------------------------------------------------------------------
# Colour ingest and depth unprojection (vx-vision ColorConvert::rgba_to_gray,
# DepthToCloud): tier 2 (cloud_oracle.cpp) and tier 1 (the shaders compiled
# as C++, _ref/libcloud_ref.so).
CLOUD_REF_SO = os.path.join(HERE, "_ref", "libcloud_ref.so")
_cloud_ref = None
POINT3D = np.dtype([("position", "<f4", (3,)), ("_pad0", "<f4"), ("color", "u1", (4,)),
                    ("normal", "<f4", (3,)), ("_pad1", "<f4")])
CLOUD_DEFAULTS = dict(min_depth=0.1, max_depth=10.0, depth_scale=1.0, max_points=1_000_000)


def ref_cloud_available() -> bool:
    return os.path.exists(CLOUD_REF_SO)


def _cloud_ref_lib():
    global _cloud_ref
    if _cloud_ref is None:
        _cloud_ref = ctypes.CDLL(CLOUD_REF_SO)
        _cloud_ref.ref_depth_to_cloud.restype = ctypes.c_uint
        _cloud_ref.ref_depth_to_cloud.argtypes = [_P, ctypes.c_uint, ctypes.c_uint, _P, ctypes.c_int] + \
            [ctypes.c_float] * 7 + [ctypes.c_uint, _P]
    return _cloud_ref


def _color_args(color):
    if color is None:
        return None, 0
    color = np.ascontiguousarray(color, np.uint8)
    return color, (2 if color.ndim == 3 else 1)


def rgba_to_gray(rgba: np.ndarray, ref: bool = False) -> np.ndarray:
    """(H, W, 4) u8 -> (H, W) u8."""
    rgba = np.ascontiguousarray(rgba, np.uint8)
    h, w, _ = rgba.shape
    out = np.zeros((h, w), np.uint8)
    fn = _cloud_ref_lib().ref_rgba_to_gray if ref else lib().oracle_rgba_to_gray
    r = fn(_P(rgba.ctypes.data), _P(out.ctypes.data), w, h)
    if r != 0:
        raise ValueError("rgba_to_gray rejected its arguments")
    return out


def depth_to_cloud(depth, color=None, fx=500.0, fy=500.0, cx=0.0, cy=0.0, min_depth=0.1, max_depth=10.0,
                   depth_scale=1.0, max_points=1_000_000, ref: bool = False):
    """Returns (points as POINT3D records, number of pixels that passed); colour: None,
    (H, W) u8 or (H, W, 4) u8. Points in row-major pixel order, min(count, max_points,
    W*H) of them."""
    depth = np.ascontiguousarray(depth, np.float32)
    h, w = depth.shape
    cap = min(int(max_points), w * h)
    pts = np.zeros(max(cap, 1), POINT3D)
    col, fmt = _color_args(color)
    cp = _P(col.ctypes.data) if col is not None else None
    if ref:
        n = _cloud_ref_lib().ref_depth_to_cloud(_P(depth.ctypes.data), w, h, cp, fmt, fx, fy, cx, cy, min_depth,
                                                max_depth, depth_scale, cap, _P(pts.ctypes.data))
    else:
        fn = lib().oracle_depth_to_cloud
        fn.restype = ctypes.c_long
        fn.argtypes = [_P, ctypes.c_int, ctypes.c_int, _P, ctypes.c_int] + [ctypes.c_float] * 7 + \
            [ctypes.c_uint, _P]
        n = fn(_P(depth.ctypes.data), w, h, cp, fmt, fx, fy, cx, cy, min_depth, max_depth, depth_scale, cap,
               _P(pts.ctypes.data))
    return pts[:min(int(n), cap)].copy(), int(n)
