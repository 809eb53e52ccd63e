"""Python binding of the B200 SGM stereo library (ctypes over include/vx_sgm.h).

Mirrors vx-vision's SGM API (MisterEkole/vx-rs):

    ctx = Context()                                  # Context::new()         context.rs:26
    sgm = SGMStereo(ctx)                             # SGMStereo::new(&ctx)   kernels/sgm.rs:73
    left = ctx.texture_gray8(l, w, h)                # Context::texture_gray8 context.rs:39
    out = ctx.texture_output_r32float(w, h)          # context.rs:64
    sgm.compute_disparity(ctx, left, right, out, SGMStereoConfig.new(64))   # sgm.rs:108
    disp = out.read_r32float()                       # Texture::read_r32float texture.rs:404

Errors raise VxError carrying the C status (the reference's Error variants,
vx-vision/src/error.rs:8-23). The CUDA library is required: importing this
module fails loudly if libvx_sgm.so is missing or does not load.
"""
from __future__ import annotations

import ctypes
import os
from dataclasses import dataclass, fields

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libvx_sgm.so")

if not os.path.exists(LIB_PATH):
    raise ImportError(f"{LIB_PATH} is missing: build it with `make -C {_HERE}` "
                      "(or __graft_entry__.build())")
_lib = ctypes.CDLL(LIB_PATH)

_P = ctypes.c_void_p

VX_OK = 0
STATUS_NAMES = {
    0: "VX_OK", 1: "VX_ERR_DEVICE_NOT_FOUND", 2: "VX_ERR_SHADER_MISSING",
    3: "VX_ERR_PIPELINE_COMPILE", 4: "VX_ERR_BUFFER_ALLOC", 5: "VX_ERR_SIZE_MISMATCH",
    6: "VX_ERR_INVALID_CONFIG", 7: "VX_ERR_GPU", 8: "VX_ERR_BUDGET", 9: "VX_ERR_TIMEOUT",
    10: "VX_ERR_INVALID_ARGUMENT", 11: "VX_ERR_NOT_READY", 12: "VX_ERR_CANCELLED",
}
FORMAT_U8, FORMAT_F32, FORMAT_I16, FORMAT_RGBA8 = 0, 1, 2, 3
_FORMAT_DTYPE = {FORMAT_U8: np.uint8, FORMAT_F32: np.float32, FORMAT_I16: np.int16, FORMAT_RGBA8: np.uint8}


def _host_shape(fmt, width, height):
    return (height, width, 4) if fmt == FORMAT_RGBA8 else (height, width)


class VxError(RuntimeError):
    def __init__(self, status: int, message: str):
        super().__init__(f"{STATUS_NAMES.get(status, status)}: {message}")
        self.status = status
        self.message = message


class _CConfig(ctypes.Structure):
    _fields_ = [("num_disparities", ctypes.c_uint32), ("p1", ctypes.c_float),
                ("p2", ctypes.c_float), ("census_radius_x", ctypes.c_uint32),
                ("census_radius_y", ctypes.c_uint32), ("num_paths", ctypes.c_uint32),
                ("subpixel", ctypes.c_uint32), ("lr_check", ctypes.c_uint32),
                ("lr_tolerance", ctypes.c_uint32), ("invalid_value", ctypes.c_float)]


class _CIntrinsics(ctypes.Structure):
    _fields_ = [("fx", ctypes.c_float), ("fy", ctypes.c_float), ("cx", ctypes.c_float),
                ("cy", ctypes.c_float), ("width", ctypes.c_uint32), ("height", ctypes.c_uint32)]


class _CDepthMap(ctypes.Structure):
    _fields_ = [("texture", _P), ("intrinsics", _CIntrinsics), ("min_depth", ctypes.c_float),
                ("max_depth", ctypes.c_float)]


@dataclass
class CameraIntrinsics:
    """vx-vision/src/types_3d.rs:254-267."""
    fx: float
    fy: float
    cx: float
    cy: float
    width: int
    height: int

    def to_c(self) -> _CIntrinsics:
        return _CIntrinsics(self.fx, self.fy, self.cx, self.cy, self.width, self.height)


@dataclass
class DepthMap:
    """vx-vision/src/types_3d.rs:384-410: the disparity texture with intrinsics and range."""
    texture: "Texture"
    intrinsics: CameraIntrinsics
    min_depth: float
    max_depth: float


def _sig(name, restype, *argtypes):
    fn = getattr(_lib, name)
    fn.restype = restype
    fn.argtypes = list(argtypes)
    return fn


_last_error = _sig("vx_last_error", ctypes.c_char_p)
_launch_count = _sig("vx_kernel_launch_count", ctypes.c_uint64)
_alloc_count = _sig("vx_memory_allocation_count", ctypes.c_uint64)
_ctx_create = _sig("vx_ctx_create", ctypes.c_int, ctypes.c_int, ctypes.POINTER(_P))
_ctx_destroy = _sig("vx_ctx_destroy", None, _P)
_ctx_stream = _sig("vx_ctx_stream", _P, _P)
_ctx_sync = _sig("vx_ctx_synchronize", ctypes.c_int, _P)
_ctx_timing = _sig("vx_ctx_enable_stage_timing", ctypes.c_int, _P, ctypes.c_int)
_ctx_times = _sig("vx_ctx_stage_times_detail", ctypes.c_int, _P, ctypes.POINTER(ctypes.c_float),
                  ctypes.POINTER(ctypes.c_float), ctypes.POINTER(ctypes.c_float), ctypes.POINTER(ctypes.c_float))
_img_create = _sig("vx_image_create", ctypes.c_int, _P, ctypes.c_uint32, ctypes.c_uint32,
                   ctypes.c_int, ctypes.POINTER(_P))
_img_wrap = _sig("vx_image_wrap_device", ctypes.c_int, _P, _P, ctypes.c_size_t, ctypes.c_uint32,
                 ctypes.c_uint32, ctypes.c_int, ctypes.POINTER(_P))
_img_destroy = _sig("vx_image_destroy", None, _P)
_img_upload = _sig("vx_image_upload", ctypes.c_int, _P, _P, ctypes.c_size_t, _P)
_img_download = _sig("vx_image_download", ctypes.c_int, _P, _P, ctypes.c_size_t, _P)
_img_ptr = _sig("vx_image_device_ptr", _P, _P)
_img_pitch = _sig("vx_image_pitch", ctypes.c_size_t, _P)
_cfg_default = _sig("vx_sgm_config_default", None, ctypes.POINTER(_CConfig))
_sgm_create = _sig("vx_sgm_create", ctypes.c_int, _P, ctypes.POINTER(_P))
_sgm_destroy = _sig("vx_sgm_destroy", None, _P)
_sgm_compute_depth = _sig("vx_sgm_compute", ctypes.c_int, _P, _P, _P, _P, ctypes.POINTER(_CConfig),
                          ctypes.POINTER(_CIntrinsics), ctypes.c_float, _P,
                          ctypes.POINTER(_CDepthMap))
_ctx_ws_limit = _sig("vx_ctx_set_workspace_limit", ctypes.c_int, _P, ctypes.c_size_t)
_sgm_compute = _sig("vx_sgm_compute_disparity", ctypes.c_int, _P, _P, _P, _P, _P, _P,
                    ctypes.POINTER(_CConfig), _P)
_sgm_batch = _sig("vx_sgm_compute_batch", ctypes.c_int, _P, _P, ctypes.c_uint32,
                  ctypes.POINTER(_P), ctypes.POINTER(_P), ctypes.POINTER(_P), ctypes.POINTER(_P),
                  ctypes.POINTER(_CConfig), _P)
_sgm_autotune = _sig("vx_sgm_autotune_batch", ctypes.c_int, _P, _P, ctypes.c_uint32,
                     ctypes.POINTER(_P), ctypes.POINTER(_P), ctypes.POINTER(_P), ctypes.POINTER(_P),
                     ctypes.POINTER(_CConfig), ctypes.c_uint32, ctypes.POINTER(ctypes.c_uint32),
                     ctypes.POINTER(ctypes.c_float), ctypes.POINTER(ctypes.c_uint32))
_graph_cache = _sig("vx_sgm_set_graph_cache", ctypes.c_int, _P, ctypes.c_uint32)
_tuning_save = _sig("vx_sgm_tuning_save", ctypes.c_int, _P, ctypes.c_char_p)
_tuning_load = _sig("vx_sgm_tuning_load", ctypes.c_int, _P, ctypes.c_char_p)
_sgm_ws = _sig("vx_sgm_workspace_bytes", ctypes.c_size_t, ctypes.c_uint32, ctypes.c_uint32,
               ctypes.POINTER(_CConfig))
_sgm_noalloc = _sig("vx_sgm_compute_disparity_noalloc", ctypes.c_int, _P, ctypes.c_size_t, _P,
                    ctypes.c_size_t, ctypes.c_uint32, ctypes.c_uint32, _P, ctypes.c_size_t, _P,
                    ctypes.c_size_t, ctypes.POINTER(_CConfig), _P)
_static_scratch_bytes = _sig("vx_sgm_static_scratch_bytes", ctypes.c_size_t)
_sgm_dump = _sig("vx_sgm_debug_dump", ctypes.c_int, _P, _P, _P, _P, ctypes.POINTER(_CConfig),
                 _P, _P, _P, _P)


def _check(status: int):
    if status != VX_OK:
        raise VxError(status, _last_error().decode(errors="replace"))


def last_error() -> str:
    return _last_error().decode(errors="replace")


def kernel_launch_count() -> int:
    """Kernel launches this library has issued since it was loaded."""
    return int(_launch_count())


def memory_allocation_count() -> int:
    """Device and pinned-host memory allocations this library has requested since it
    was loaded (pool allocations, cudaMalloc*, cudaMallocHost)."""
    return int(_alloc_count())


@dataclass
class SGMStereoConfig:
    """vx-vision/src/kernels/sgm.rs:23-59 plus the opt-in extensions."""
    num_disparities: int = 128
    p1: float = 10.0
    p2: float = 120.0
    census_radius_x: int = 4
    census_radius_y: int = 3
    num_paths: int = 2
    subpixel: bool = True
    lr_check: bool = False
    lr_tolerance: int = 1
    invalid_value: float = -1.0

    @classmethod
    def new(cls, num_disparities: int) -> "SGMStereoConfig":
        return cls(num_disparities=num_disparities)

    @classmethod
    def from_c_default(cls) -> "SGMStereoConfig":
        c = _CConfig()
        _cfg_default(ctypes.byref(c))
        return cls(**{f.name: getattr(c, f.name) for f in fields(cls)})

    def to_c(self) -> _CConfig:
        return _CConfig(int(self.num_disparities), float(self.p1), float(self.p2),
                        int(self.census_radius_x), int(self.census_radius_y), int(self.num_paths),
                        int(bool(self.subpixel)), int(bool(self.lr_check)),
                        int(self.lr_tolerance), float(self.invalid_value))


class Context:
    """A CUDA device with its stream and stream-ordered memory pool."""

    def __init__(self, device: int = 0):
        h = _P()
        _check(_ctx_create(int(device), ctypes.byref(h)))
        self._h = h
        self.device = device

    @property
    def handle(self):
        return self._h

    @property
    def stream(self) -> int:
        return _ctx_stream(self._h) or 0

    def synchronize(self):
        _check(_ctx_sync(self._h))

    def set_workspace_limit(self, nbytes: int):
        """Batches needing more device workspace run as consecutive sub-batches."""
        _check(_ctx_ws_limit(self._h, int(nbytes)))

    def enable_stage_timing(self, on: bool = True):
        _check(_ctx_timing(self._h, int(bool(on))))

    def stage_times(self):
        """(census_ms, aggregate_ms, wta_ms), the mean per timed batch from CUDA events;
        census_ms includes the cost volume (stage_times_detail has it apart)."""
        a, b, c, d = self.stage_times_detail()
        return a + b, c, d

    def stage_times_detail(self):
        """(census_ms, costs_ms, aggregate_ms, wta_ms), the mean per timed batch."""
        a, b, c, d = ctypes.c_float(), ctypes.c_float(), ctypes.c_float(), ctypes.c_float()
        _check(_ctx_times(self._h, ctypes.byref(a), ctypes.byref(b), ctypes.byref(c), ctypes.byref(d)))
        return a.value, b.value, c.value, d.value

    def close(self):
        if self._h:
            _ctx_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def texture_gray8(self, pixels, width: int, height: int) -> "Texture":
        t = Texture.create(self, width, height, FORMAT_U8)
        t.upload(np.asarray(pixels, dtype=np.uint8).reshape(height, width))
        return t

    def texture_output_r32float(self, width: int, height: int) -> "Texture":
        return Texture.create(self, width, height, FORMAT_F32)

    def texture_rgba8(self, pixels, width: int, height: int) -> "Texture":
        """Context::texture_rgba8 (context.rs:54): an RGBA8 image from (H, W, 4) bytes."""
        t = Texture.create(self, width, height, FORMAT_RGBA8)
        t.upload(np.asarray(pixels, dtype=np.uint8).reshape(height, width, 4))
        return t

    def texture_output_rgba8(self, width: int, height: int) -> "Texture":
        return Texture.create(self, width, height, FORMAT_RGBA8)

    def texture_output_gray8(self, width: int, height: int) -> "Texture":
        return Texture.create(self, width, height, FORMAT_U8)

    def texture_r32float(self, data, width: int, height: int) -> "Texture":
        """Context::texture_r32float (an F32 image from host data)."""
        t = Texture.create(self, width, height, FORMAT_F32)
        t.upload(np.asarray(data, dtype=np.float32).reshape(height, width))
        return t

    def texture_output_i16(self, width: int, height: int) -> "Texture":
        return Texture.create(self, width, height, FORMAT_I16)


class Texture:
    """A pitched device image (U8 in, F32 / I16 out)."""

    def __init__(self, ctx: Context, handle, width: int, height: int, fmt: int):
        self.ctx, self._h, self.width, self.height, self.format = ctx, handle, width, height, fmt

    @classmethod
    def create(cls, ctx: Context, width: int, height: int, fmt: int) -> "Texture":
        h = _P()
        _check(_img_create(ctx.handle, width, height, fmt, ctypes.byref(h)))
        return cls(ctx, h, width, height, fmt)

    @classmethod
    def wrap_device(cls, ctx: Context, ptr: int, pitch: int, width: int, height: int,
                    fmt: int) -> "Texture":
        h = _P()
        _check(_img_wrap(ctx.handle, _P(ptr), pitch, width, height, fmt, ctypes.byref(h)))
        return cls(ctx, h, width, height, fmt)

    @property
    def handle(self):
        return self._h

    @property
    def device_ptr(self) -> int:
        return _img_ptr(self._h) or 0

    @property
    def pitch(self) -> int:
        return int(_img_pitch(self._h))

    def upload(self, host: np.ndarray, stream: int | None = None):
        a = np.ascontiguousarray(host, dtype=_FORMAT_DTYPE[self.format])
        assert a.shape == _host_shape(self.format, self.width, self.height), (a.shape, self.height, self.width)
        _check(_img_upload(self._h, _P(a.ctypes.data), a.strides[0], _P(stream) if stream else None))

    def download(self, host: np.ndarray | None = None, stream: int | None = None) -> np.ndarray:
        if host is None:
            host = np.empty(_host_shape(self.format, self.width, self.height), dtype=_FORMAT_DTYPE[self.format])
        _check(_img_download(self._h, _P(host.ctypes.data), host.strides[0],
                             _P(stream) if stream else None))
        return host

    def read_r32float(self) -> np.ndarray:
        assert self.format == FORMAT_F32
        return self.download()

    def close(self):
        if self._h:
            _img_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class SGMStereo:
    """vx-vision's SGMStereo (kernels/sgm.rs:62) on the B200 kernels."""

    def __init__(self, ctx: Context):
        h = _P()
        _check(_sgm_create(ctx.handle, ctypes.byref(h)))
        self._h = h
        self._ctx = ctx  # the handle must be destroyed before its context

    @classmethod
    def new(cls, ctx: Context) -> "SGMStereo":
        return cls(ctx)

    @property
    def handle(self):
        return self._h

    def compute_disparity(self, ctx: Context, left: Texture, right: Texture, output: Texture,
                          config: SGMStereoConfig, output_i16: Texture | None = None,
                          stream: int | None = None):
        c = config.to_c()
        _check(_sgm_compute(self._h, ctx.handle, left.handle, right.handle, output.handle,
                            output_i16.handle if output_i16 is not None else None,
                            ctypes.byref(c), _P(stream) if stream else None))

    def compute(self, ctx: Context, left: Texture, right: Texture, config: SGMStereoConfig,
                intrinsics: CameraIntrinsics, baseline: float,
                depth_out: Texture | None = None) -> DepthMap:
        """SGMStereo::compute (kernels/sgm.rs:268-288): a DepthMap over a new F32 disparity
        texture (no conversion, like the reference); depth_out optionally receives
        fx * baseline / disparity."""
        c = config.to_c()
        ci = intrinsics.to_c()
        dm = _CDepthMap()
        _check(_sgm_compute_depth(self._h, ctx.handle, left.handle, right.handle, ctypes.byref(c),
                                  ctypes.byref(ci), float(baseline),
                                  depth_out.handle if depth_out is not None else None,
                                  ctypes.byref(dm)))
        tex = Texture(ctx, _P(dm.texture), left.width, left.height, FORMAT_F32)
        return DepthMap(tex, intrinsics, float(dm.min_depth), float(dm.max_depth))

    def compute_batch(self, ctx: Context, lefts, rights, outputs, configs, outputs_i16=None,
                      stream: int | None = None):
        n = len(lefts)
        arr = lambda ts: (_P * n)(*[t.handle if t is not None else None for t in ts])
        cfgs = (_CConfig * n)(*[c.to_c() for c in configs])
        oi = arr(outputs_i16) if outputs_i16 is not None else None
        _check(_sgm_batch(self._h, ctx.handle, n, arr(lefts), arr(rights), arr(outputs), oi, cfgs,
                          _P(stream) if stream else None))

    def autotune_batch(self, ctx: Context, lefts, rights, outputs, configs, outputs_i16=None,
                       iterations: int = 2):
        """Times every aggregation form and launch shape on this batch and keeps the
        fastest for batches like it. Returns (warpgroups, aggregate_ms,
        unit_scanlines) of the winner (unit_scanlines 32: single-scanline kernel,
        64: scanline-pair kernel, 1: across-lanes scan kernel)."""
        n = len(lefts)
        arr = lambda ts: (_P * n)(*[t.handle if t is not None else None for t in ts])
        cfgs = (_CConfig * n)(*[c.to_c() for c in configs])
        oi = arr(outputs_i16) if outputs_i16 is not None else None
        w, ms, us = ctypes.c_uint32(), ctypes.c_float(), ctypes.c_uint32()
        _check(_sgm_autotune(self._h, ctx.handle, n, arr(lefts), arr(rights), arr(outputs), oi,
                             cfgs, iterations, ctypes.byref(w), ctypes.byref(ms), ctypes.byref(us)))
        return int(w.value), float(ms.value), int(us.value)

    def set_graph_cache(self, max_buckets: int):
        """CUDA graphs per shape bucket for compute_batch / compute_disparity."""
        _check(_graph_cache(self._h, int(max_buckets)))

    def tuning_save(self, path: str):
        _check(_tuning_save(self._h, path.encode()))

    def tuning_load(self, path: str):
        _check(_tuning_load(self._h, path.encode()))

    def debug_dump(self, ctx: Context, left: Texture, right: Texture, config: SGMStereoConfig):
        """Census words, per-path costs L_r and summed cost volume S of one pair."""
        h, w, d, p = left.height, left.width, config.num_disparities, config.num_paths
        cl = np.zeros((h, w), np.uint64)
        cr = np.zeros((h, w), np.uint64)
        L = np.zeros((p, h, w, d), np.uint16)
        S = np.zeros((h, w, d), np.uint16)
        c = config.to_c()
        _check(_sgm_dump(self._h, ctx.handle, left.handle, right.handle, ctypes.byref(c),
                         _P(cl.ctypes.data), _P(cr.ctypes.data), _P(L.ctypes.data),
                         _P(S.ctypes.data)))
        return cl, cr, L, S

    def close(self):
        if self._h:
            _sgm_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class _CDepthFilterConfig(ctypes.Structure):
    _fields_ = [("radius", ctypes.c_int32), ("sigma_spatial", ctypes.c_float),
                ("sigma_depth", ctypes.c_float)]


class _CDepthMedianConfig(ctypes.Structure):
    _fields_ = [("radius", ctypes.c_int32)]


_df_create = _sig("vx_depth_filter_create", ctypes.c_int, _P, ctypes.POINTER(_P))
_df_destroy = _sig("vx_depth_filter_destroy", None, _P)
_df_median = _sig("vx_depth_filter_apply_median", ctypes.c_int, _P, _P, _P, _P,
                  ctypes.POINTER(_CDepthMedianConfig), _P)
_df_bilateral = _sig("vx_depth_filter_apply_bilateral", ctypes.c_int, _P, _P, _P, _P,
                     ctypes.POINTER(_CDepthFilterConfig), _P)


class DepthFilterConfig:
    """DepthFilterConfig (depth_filter.rs:19-49): bilateral window and sigmas."""

    def __init__(self, radius: int = 3, sigma_spatial: float = 5.0, sigma_depth: float = 0.05):
        self.radius, self.sigma_spatial, self.sigma_depth = radius, sigma_spatial, sigma_depth

    @classmethod
    def new(cls, radius: int, sigma_spatial: float, sigma_depth: float) -> "DepthFilterConfig":
        return cls(radius, sigma_spatial, sigma_depth)


class DepthMedianConfig:
    """DepthMedianConfig (depth_filter.rs:51-63): radius 1 = 3x3, 2 = 5x5."""

    def __init__(self, radius: int = 1):
        self.radius = radius


class DepthFilter:
    """DepthFilter (depth_filter.rs): median and bilateral depth-map filters."""

    def __init__(self, ctx: Context):
        h = _P()
        _check(_df_create(ctx.handle, ctypes.byref(h)))
        self._h, self._ctx = h, ctx

    @classmethod
    def new(cls, ctx: Context) -> "DepthFilter":
        return cls(ctx)

    def apply_median(self, ctx: Context, input: Texture, output: Texture,
                     config: DepthMedianConfig = None, stream=None):
        c = _CDepthMedianConfig((config or DepthMedianConfig()).radius)
        _check(_df_median(self._h, ctx.handle, input.handle, output.handle, ctypes.byref(c),
                         _P(stream) if stream else None))

    def apply_bilateral(self, ctx: Context, input: Texture, output: Texture,
                        config: DepthFilterConfig = None, stream=None):
        cfg = config or DepthFilterConfig()
        c = _CDepthFilterConfig(cfg.radius, cfg.sigma_spatial, cfg.sigma_depth)
        _check(_df_bilateral(self._h, ctx.handle, input.handle, output.handle, ctypes.byref(c),
                         _P(stream) if stream else None))

    def close(self):
        if self._h:
            _df_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


# ---------------------------------------------------------------------------
# The depth chain's ends: colour ingest (vx-vision/src/kernels/color.rs) and
# point clouds (vx-vision/src/kernels/depth_to_cloud.rs)

# GpuPoint3D (vx-vision/src/types.rs:440-448), 36 bytes.
POINT3D = np.dtype([("position", "<f4", (3,)), ("_pad0", "<f4"), ("color", "u1", (4,)),
                    ("normal", "<f4", (3,)), ("_pad1", "<f4")])
assert POINT3D.itemsize == 36


class _CDepthToCloudConfig(ctypes.Structure):
    _fields_ = [("min_depth", ctypes.c_float), ("max_depth", ctypes.c_float), ("depth_scale", ctypes.c_float),
                ("max_points", ctypes.c_uint32)]


_color_gray = _sig("vx_color_rgba_to_gray", ctypes.c_int, _P, _P, _P, _P)
_d2c_create = _sig("vx_depth_to_cloud_create", ctypes.c_int, _P, ctypes.POINTER(_P))
_d2c_destroy = _sig("vx_depth_to_cloud_destroy", None, _P)
_d2c_raw = _sig("vx_depth_to_cloud_compute_raw", ctypes.c_int, _P, _P, _P, _P, ctypes.c_float, ctypes.c_float,
                ctypes.c_float, ctypes.c_float, ctypes.POINTER(_CDepthToCloudConfig), _P, ctypes.c_size_t,
                ctypes.POINTER(ctypes.c_size_t))
_d2c_device = _sig("vx_depth_to_cloud_compute_device", ctypes.c_int, _P, _P, _P, _P, ctypes.c_float, ctypes.c_float,
                   ctypes.c_float, ctypes.c_float, ctypes.POINTER(_CDepthToCloudConfig), _P, ctypes.c_uint32, _P, _P)


class ColorConvert:
    """ColorConvert (color.rs:20-80): here its rgba_to_gray, the ingest of colour pairs."""

    def __init__(self, ctx: Context):
        self._ctx = ctx

    @classmethod
    def new(cls, ctx: Context) -> "ColorConvert":
        return cls(ctx)

    def rgba_to_gray(self, ctx: Context, input: Texture, output: Texture, stream=None):
        _check(_color_gray(ctx.handle, input.handle, output.handle, _P(stream) if stream else None))


@dataclass
class DepthToCloudConfig:
    """DepthToCloudConfig (depth_to_cloud.rs:23-59)."""
    min_depth: float = 0.1
    max_depth: float = 10.0
    depth_scale: float = 1.0
    max_points: int = 1_000_000

    @classmethod
    def new(cls, min_depth: float, max_depth: float) -> "DepthToCloudConfig":
        return cls(min_depth=min_depth, max_depth=max_depth)

    def to_c(self) -> _CDepthToCloudConfig:
        return _CDepthToCloudConfig(self.min_depth, self.max_depth, self.depth_scale, self.max_points)


@dataclass
class PointCloud:
    """PointCloud (types_3d.rs:50-90): the points as POINT3D records."""
    points: np.ndarray

    def __len__(self):
        return len(self.points)


class DepthToCloud:
    """DepthToCloud (depth_to_cloud.rs:62-188): depth map -> point cloud."""

    def __init__(self, ctx: Context):
        h = _P()
        _check(_d2c_create(ctx.handle, ctypes.byref(h)))
        self._h, self._ctx = h, ctx

    @classmethod
    def new(cls, ctx: Context) -> "DepthToCloud":
        return cls(ctx)

    def compute_raw(self, ctx: Context, depth: Texture, color: Texture | None, fx: float, fy: float, cx: float,
                    cy: float, config: DepthToCloudConfig | None = None) -> PointCloud:
        cfg = config or DepthToCloudConfig()
        cap = min(int(cfg.max_points), depth.width * depth.height)
        out = np.zeros(cap, POINT3D)
        n = ctypes.c_size_t()
        c = cfg.to_c()
        _check(_d2c_raw(self._h, ctx.handle, depth.handle, color.handle if color is not None else None, fx, fy, cx,
                        cy, ctypes.byref(c), _P(out.ctypes.data) if cap else None, cap, ctypes.byref(n)))
        return PointCloud(out[:n.value].copy())

    def compute(self, ctx: Context, depth: "DepthMap", color: Texture | None = None,
                config: DepthToCloudConfig | None = None) -> PointCloud:
        k = depth.intrinsics
        return self.compute_raw(ctx, depth.texture, color, k.fx, k.fy, k.cx, k.cy, config)

    def compute_device(self, ctx: Context, depth: Texture, color: Texture | None, fx: float, fy: float, cx: float,
                       cy: float, config: DepthToCloudConfig, points_ptr: int, capacity: int, count_ptr: int,
                       stream=None):
        c = config.to_c()
        _check(_d2c_device(self._h, ctx.handle, depth.handle, color.handle if color is not None else None, fx, fy,
                           cx, cy, ctypes.byref(c), _P(points_ptr), capacity, _P(count_ptr),
                           _P(stream) if stream else None))

    def close(self):
        if self._h:
            _d2c_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


# ---------------------------------------------------------------------------
# Sparse ORB stereo matching (vx-vision/src/kernels/stereomatch.rs)

# CornerPoint (types.rs:8-12), ORBOutput (types.rs:36-39), StereoMatchResult (types.rs:64-70).
CORNER_POINT = np.dtype([("position", "<f4", (2,)), ("response", "<f4"), ("pyramid_level", "<u4")])
ORB_OUTPUT = np.dtype([("desc", "<u4", (8,)), ("angle", "<f4")])
STEREO_MATCH_RESULT = np.dtype([("left_idx", "<u4"), ("right_idx", "<u4"), ("disparity", "<f4"),
                                ("point_3d", "<f4", (3,)), ("_pad", "<f4")])


class _CStereoConfig(ctypes.Structure):
    _fields_ = [("max_epipolar", ctypes.c_float), ("min_disparity", ctypes.c_float),
                ("max_disparity", ctypes.c_float), ("max_hamming", ctypes.c_uint32),
                ("ratio_thresh", ctypes.c_float), ("fx", ctypes.c_float), ("fy", ctypes.c_float),
                ("cx", ctypes.c_float), ("cy", ctypes.c_float), ("baseline", ctypes.c_float)]


_sm_create = _sig("vx_stereo_matcher_create", ctypes.c_int, _P, ctypes.POINTER(_P))
_sm_destroy = _sig("vx_stereo_matcher_destroy", None, _P)
_sm_run = _sig("vx_stereo_matcher_run", ctypes.c_int, _P, _P, _P, ctypes.c_size_t, _P, ctypes.c_size_t,
               _P, ctypes.c_size_t, _P, ctypes.c_size_t, ctypes.POINTER(_CStereoConfig), _P,
               ctypes.c_size_t, ctypes.POINTER(ctypes.c_size_t))
_sm_run_device = _sig("vx_stereo_matcher_run_device", ctypes.c_int, _P, _P, _P, ctypes.c_uint32, _P,
                      ctypes.c_uint32, _P, _P, ctypes.POINTER(_CStereoConfig), _P, _P, _P)
_sm_run_frames = _sig("vx_stereo_matcher_run_frames_device", ctypes.c_int, _P, _P, ctypes.c_uint32, _P, _P,
                      _P, _P, _P, _P, ctypes.POINTER(_CStereoConfig), _P, _P, _P)


@dataclass
class StereoConfig:
    """StereoConfig (stereomatch.rs:19-69), with the reference's defaults."""
    max_epipolar: float = 2.0
    min_disparity: float = 1.0
    max_disparity: float = 120.0
    max_hamming: int = 50
    ratio_thresh: float = 0.8
    fx: float = 600.0
    fy: float = 600.0
    cx: float = 320.0
    cy: float = 240.0
    baseline: float = 0.12

    def to_c(self) -> _CStereoConfig:
        return _CStereoConfig(self.max_epipolar, self.min_disparity, self.max_disparity,
                              int(self.max_hamming) & 0xFFFFFFFF, self.ratio_thresh, self.fx, self.fy,
                              self.cx, self.cy, self.baseline)


@dataclass
class StereoResult:
    """StereoResult (stereomatch.rs:77-82): STEREO_MATCH_RESULT records."""
    matches: np.ndarray


def as_corner_points(kpts) -> np.ndarray:
    """CornerPoint records from CORNER_POINT arrays or (n, 4) float32 rows
    (x, y, response, level bits)."""
    a = np.asarray(kpts)
    if a.dtype == CORNER_POINT:
        return np.ascontiguousarray(a)
    return np.ascontiguousarray(a, np.float32).reshape(-1, 4).view(CORNER_POINT).reshape(-1)


def as_orb_outputs(descs) -> np.ndarray:
    """ORBOutput records from ORB_OUTPUT arrays or (n, 8) uint32 descriptor words."""
    a = np.asarray(descs)
    if a.dtype == ORB_OUTPUT:
        return np.ascontiguousarray(a)
    w = np.ascontiguousarray(a, np.uint32).reshape(-1, 8)
    out = np.zeros(len(w), ORB_OUTPUT)
    out["desc"] = w
    return out


class StereoMatcher:
    """StereoMatcher (stereomatch.rs:71-249): sparse ORB matching on rectified pairs."""

    def __init__(self, ctx: Context):
        h = _P()
        _check(_sm_create(ctx.handle, ctypes.byref(h)))
        self._h, self._ctx = h, ctx

    @classmethod
    def new(cls, ctx: Context) -> "StereoMatcher":
        return cls(ctx)

    def run(self, ctx: Context, left_kpts, right_kpts, left_descs, right_descs,
            config: StereoConfig = None) -> StereoResult:
        """StereoMatcher::run (stereomatch.rs:115-249): host arrays in and out, synchronous."""
        lk, rk = as_corner_points(left_kpts), as_corner_points(right_kpts)
        ld, rd = as_orb_outputs(left_descs), as_orb_outputs(right_descs)
        c = (config or StereoConfig()).to_c()
        out = np.zeros(max(len(lk), 1), STEREO_MATCH_RESULT)
        n = ctypes.c_size_t(0)
        _check(_sm_run(self._h, ctx.handle, _P(lk.ctypes.data), len(lk), _P(rk.ctypes.data), len(rk),
                       _P(ld.ctypes.data), len(ld), _P(rd.ctypes.data), len(rd), ctypes.byref(c),
                       _P(out.ctypes.data), len(out), ctypes.byref(n)))
        return StereoResult(out[:n.value].copy())

    def run_device(self, ctx: Context, left_kpts: int, n_left: int, right_kpts: int, n_right: int,
                   left_desc_words: int, right_desc_words: int, config: StereoConfig,
                   matches: int, match_count: int, stream: int | None = None):
        """Device pointers in and out (vx_stereo_matcher_run_device); asynchronous on `stream`."""
        c = config.to_c()
        _check(_sm_run_device(self._h, ctx.handle, _P(left_kpts), n_left, _P(right_kpts), n_right,
                              _P(left_desc_words), _P(right_desc_words), ctypes.byref(c), _P(matches),
                              _P(match_count), _P(stream) if stream else None))

    def run_frames_device(self, ctx: Context, left_offsets, right_offsets, left_kpts: int, right_kpts: int,
                          left_desc_words: int, right_desc_words: int, config: StereoConfig, matches: int,
                          match_counts: int, stream: int | None = None):
        """Many frames in one launch (vx_stereo_matcher_run_frames_device): offsets
        are host arrays of n_frames + 1 (numpy or lists), the rest device pointers."""
        lo = np.ascontiguousarray(left_offsets, np.uint32)
        ro = np.ascontiguousarray(right_offsets, np.uint32)
        if lo.shape != ro.shape or lo.size < 1:
            raise ValueError("left and right offsets need n_frames + 1 entries each")
        c = config.to_c()
        _check(_sm_run_frames(self._h, ctx.handle, lo.size - 1, _P(lo.ctypes.data), _P(ro.ctypes.data),
                              _P(left_kpts), _P(right_kpts), _P(left_desc_words), _P(right_desc_words),
                              ctypes.byref(c), _P(matches), _P(match_counts), _P(stream) if stream else None))

    def close(self):
        if self._h:
            _sm_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class _CServerConfig(ctypes.Structure):
    _fields_ = [("memory_budget_bytes", ctypes.c_size_t), ("max_batch", ctypes.c_uint32),
                ("max_inflight_batches", ctypes.c_uint32), ("host_staging_bytes", ctypes.c_size_t)]


class ServerStats(ctypes.Structure):
    _fields_ = [("submitted", ctypes.c_uint64), ("completed", ctypes.c_uint64),
                ("rejected", ctypes.c_uint64), ("cancelled", ctypes.c_uint64),
                ("failed", ctypes.c_uint64), ("batches", ctypes.c_uint64),
                ("queued", ctypes.c_uint64), ("inflight_bytes", ctypes.c_uint64),
                ("completed_pixel_disparities", ctypes.c_uint64),
                ("pool_reserved_bytes", ctypes.c_uint64), ("pinned_bytes", ctypes.c_uint64),
                ("max_launch_us", ctypes.c_uint64), ("max_pinned_alloc_us", ctypes.c_uint64),
                ("staging_overflows", ctypes.c_uint64), ("shadow_reruns", ctypes.c_uint64),
                ("max_batches_in_flight", ctypes.c_uint64)]

    def as_dict(self):
        return {f: int(getattr(self, f)) for f, _ in self._fields_}


_srv_create = _sig("vx_sgm_server_create", ctypes.c_int, _P, _P, ctypes.POINTER(_CServerConfig),
                   ctypes.POINTER(_P))
_srv_destroy = _sig("vx_sgm_server_destroy", None, _P)
_srv_submit = _sig("vx_sgm_server_submit", ctypes.c_int, _P, _P, _P, ctypes.c_uint32,
                   ctypes.c_uint32, ctypes.c_size_t, ctypes.POINTER(_CConfig), ctypes.c_int,
                   ctypes.POINTER(ctypes.c_uint64))
_srv_wait = _sig("vx_sgm_server_wait", ctypes.c_int, _P, ctypes.c_uint64, _P, _P,
                 ctypes.POINTER(ctypes.c_double), ctypes.c_uint32)
_srv_cancel = _sig("vx_sgm_server_cancel", ctypes.c_int, _P, ctypes.c_uint64)
_srv_stats = _sig("vx_sgm_server_get_stats", ctypes.c_int, _P, ctypes.POINTER(ServerStats))


class Server:
    """Continuous-batching SGM server under a device-memory budget (see vx_sgm.h)."""

    def __init__(self, sgm: "SGMStereo", ctx: Context, memory_budget_bytes: int,
                 max_batch: int = 32, max_inflight_batches: int = 2, host_staging_bytes: int = 0):
        c = _CServerConfig(int(memory_budget_bytes), int(max_batch), int(max_inflight_batches),
                           int(host_staging_bytes))
        h = _P()
        _check(_srv_create(sgm.handle, ctx.handle, ctypes.byref(c), ctypes.byref(h)))
        self._h = h
        self._keep = (sgm, ctx)
        self._shapes = {}

    def submit(self, left: np.ndarray, right: np.ndarray, config: SGMStereoConfig,
               want_i16: bool = True) -> int:
        left = np.ascontiguousarray(left, np.uint8)
        right = np.ascontiguousarray(right, np.uint8)
        h, w = left.shape
        c = config.to_c()
        rid = ctypes.c_uint64()
        _check(_srv_submit(self._h, left.ctypes.data, right.ctypes.data, w, h, w, ctypes.byref(c),
                           int(want_i16), ctypes.byref(rid)))
        self._shapes[rid.value] = (h, w, want_i16)
        return rid.value

    def wait(self, rid: int, timeout_ms: int = 60000):
        """(disparity f32, disparity i16 or None, latency_ms); raises VxError."""
        h, w, want_i16 = self._shapes[rid]
        d = np.empty((h, w), np.float32)
        di = np.empty((h, w), np.int16) if want_i16 else None
        lat = ctypes.c_double()
        st = _srv_wait(self._h, rid, d.ctypes.data, di.ctypes.data if di is not None else None,
                       ctypes.byref(lat), int(timeout_ms))
        if st == 11:  # VX_ERR_NOT_READY (poll)
            return None
        del self._shapes[rid]
        _check(st)
        return d, di, lat.value

    def cancel(self, rid: int):
        _check(_srv_cancel(self._h, rid))

    def stats(self) -> dict:
        st = ServerStats()
        _check(_srv_stats(self._h, ctypes.byref(st)))
        return st.as_dict()

    def close(self):
        if self._h:
            _srv_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def compute_disparity_noalloc(left: Texture, right: Texture, output: Texture,
                              config: SGMStereoConfig, output_i16: Texture | None = None,
                              stream: int | None = None):
    """vx_sgm_compute_disparity_noalloc on the planes of existing textures: for callers that
    cannot allocate device memory during the call (scratch is a static 64 MiB device array).

    The C entry point takes one width and height for all four planes, so the
    textures' sizes and formats are checked here: U8 left and right, F32 output,
    I16 integer output, all of the left image's size (VX_ERR_SIZE_MISMATCH /
    VX_ERR_INVALID_ARGUMENT otherwise, raised before anything runs)."""
    planes = [("left", left, FORMAT_U8), ("right", right, FORMAT_U8), ("output", output, FORMAT_F32)]
    if output_i16 is not None:
        planes.append(("output_i16", output_i16, FORMAT_I16))
    for name, tex, fmt in planes:
        if tex.format != fmt:
            raise VxError(10, f"compute_disparity_noalloc: {name} has format {tex.format}, expected {fmt}")
        if (tex.width, tex.height) != (left.width, left.height):
            raise VxError(5, f"compute_disparity_noalloc: {name} is {tex.width}x{tex.height}, "
                             f"left is {left.width}x{left.height}")
    c = config.to_c()
    _check(_sgm_noalloc(_P(left.device_ptr), left.pitch, _P(right.device_ptr), right.pitch,
                        left.width, left.height, _P(output.device_ptr), output.pitch,
                        _P(output_i16.device_ptr) if output_i16 is not None else None,
                        output_i16.pitch if output_i16 is not None else 0, ctypes.byref(c),
                        _P(stream) if stream else None))


def static_scratch_bytes() -> int:
    return int(_static_scratch_bytes())


def workspace_bytes(width: int, height: int, config: SGMStereoConfig) -> int:
    c = config.to_c()
    return int(_sgm_ws(width, height, ctypes.byref(c)))


# ---------------------------------------------------------------------------
# Synthetic pairs (libvx_synth.so): R(x - d, y) = L(x, y), the shader's convention.
from vx_synth import SCENE_PLANES, SCENE_SLANTED, SCENE_SURFACE, synth_pair  # noqa: E402,F401


def synth_orb_stereo(n_left: int, n_right: int, seed: int, width: int = 752, height: int = 480,
                     overlap: float = 0.8, d_lo: float = 0.5, d_hi: float = 130.0):
    """Seeded synthetic ORB keypoints of a rectified pair (EuRoC-sized frames by
    default): returns (left CORNER_POINT, right CORNER_POINT, left ORB_OUTPUT,
    right ORB_OUTPUT). A share `overlap` of the left keypoints reappears on the
    right at x - d (d uniform in [d_lo, d_hi), partly outside the usual search
    range), y + N(0, 0.8) px, with 0-60 descriptor bits flipped; the remaining
    right keypoints are distractors, some on the same rows as a left keypoint
    with a descriptor 40-90 bits away. Positions are whole pixels at pyramid
    level 0 and multiples of 1.2^level above, as FAST on a pyramid gives."""
    rng = np.random.default_rng(seed)

    def positions(n):
        level = np.where(rng.random(n) < 0.6, 0, rng.integers(1, 4, n)).astype(np.uint32)
        scale = (1.2 ** level).astype(np.float32)
        x = (rng.integers(0, width, n) / scale).astype(np.int64) * scale
        y = (rng.integers(0, height, n) / scale).astype(np.int64) * scale
        return x.astype(np.float32), y.astype(np.float32), level

    def flip(desc, nbits):
        out = desc.copy()
        for i, k in enumerate(nbits):
            bits = rng.choice(256, int(k), replace=False)
            for b in bits:
                out[i, b >> 5] ^= np.uint32(1) << np.uint32(b & 31)
        return out

    lx, ly, llev = positions(n_left)
    ldesc = rng.integers(0, 2 ** 32, (n_left, 8), dtype=np.uint64).astype(np.uint32)
    n_pair = min(int(round(overlap * n_left)), n_right)
    src = rng.permutation(n_left)[:n_pair]
    rx = np.empty(n_right, np.float32)
    ry = np.empty(n_right, np.float32)
    rlev = np.zeros(n_right, np.uint32)
    rdesc = rng.integers(0, 2 ** 32, (n_right, 8), dtype=np.uint64).astype(np.uint32)
    rx[:n_pair] = lx[src] - rng.uniform(d_lo, d_hi, n_pair).astype(np.float32)
    ry[:n_pair] = ly[src] + rng.normal(0.0, 0.8, n_pair).astype(np.float32)
    rlev[:n_pair] = llev[src]
    rdesc[:n_pair] = flip(ldesc[src], rng.integers(0, 61, n_pair))
    n_rest = n_right - n_pair
    if n_rest > 0:
        dx, dy, dlev = positions(n_rest)
        near = rng.random(n_rest) < 0.5
        if n_left > 0 and near.any():
            k = int(near.sum())
            anchor = rng.integers(0, n_left, k)
            dy[near] = ly[anchor] + rng.uniform(-2.5, 2.5, k).astype(np.float32)
            dx[near] = lx[anchor] - rng.uniform(0.0, 125.0, k).astype(np.float32)
            rdesc[n_pair:][near] = flip(ldesc[anchor], rng.integers(40, 91, k))
        rx[n_pair:], ry[n_pair:], rlev[n_pair:] = dx, dy, dlev
    order = rng.permutation(n_right)
    rx, ry, rlev, rdesc = rx[order], ry[order], rlev[order], rdesc[order]

    lk = np.zeros(n_left, CORNER_POINT)
    lk["position"] = np.stack([lx, ly], 1) if n_left else np.zeros((0, 2), np.float32)
    lk["response"] = rng.random(n_left).astype(np.float32)
    lk["pyramid_level"] = llev
    rk = np.zeros(n_right, CORNER_POINT)
    rk["position"] = np.stack([rx, ry], 1) if n_right else np.zeros((0, 2), np.float32)
    rk["response"] = rng.random(n_right).astype(np.float32)
    rk["pyramid_level"] = rlev
    ld = np.zeros(n_left, ORB_OUTPUT)
    ld["desc"] = ldesc
    ld["angle"] = rng.uniform(-np.pi, np.pi, n_left).astype(np.float32)
    rd = np.zeros(n_right, ORB_OUTPUT)
    rd["desc"] = rdesc
    rd["angle"] = rng.uniform(-np.pi, np.pi, n_right).astype(np.float32)
    return lk, rk, ld, rd
