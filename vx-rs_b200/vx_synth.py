"""Seeded synthetic rectified stereo pairs (ctypes over libvx_synth.so).

Standalone: it loads only the generator library, not the SGM library, so the
CPU-side benchmark arm can build its inputs without mapping any CUDA code.
Convention: R(x - d, y) = L(x, y), what the SGM shader matches
(vx-vision/shaders/SGMStereo.metal:133-141).
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
SYNTH_PATH = os.path.join(_HERE, "libvx_synth.so")
SCENE_PLANES, SCENE_SLANTED, SCENE_SURFACE = 0, 1, 2
_synth = None


def _lib():
    global _synth
    if _synth is None:
        if not os.path.exists(SYNTH_PATH):
            raise ImportError(f"{SYNTH_PATH} is missing: build it with `make -C {_HERE}`")
        lib = ctypes.CDLL(SYNTH_PATH)
        lib.vx_synth_pair.restype = ctypes.c_int
        lib.vx_synth_pair.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_float,
                                      ctypes.c_float, ctypes.c_uint64, ctypes.c_void_p, ctypes.c_void_p,
                                      ctypes.c_void_p]
        _synth = lib
    return _synth


def synth_pair(scene: int, width: int, height: int, d_lo: float, d_hi: float, seed: int):
    """Returns (left u8, right u8, ground-truth disparity f32), each (H, W)."""
    L = np.empty((height, width), np.uint8)
    R = np.empty((height, width), np.uint8)
    G = np.empty((height, width), np.float32)
    r = _lib().vx_synth_pair(scene, width, height, d_lo, d_hi, seed, L.ctypes.data, R.ctypes.data,
                             G.ctypes.data)
    if r != 0:
        raise ValueError("vx_synth_pair rejected its arguments")
    return L, R, G
