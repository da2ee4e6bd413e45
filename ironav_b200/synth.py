"""Seeded synthetic luma sequences (binding of csrc/synth.cpp).

The benchmark configurations of the stage are reproduced with these settings:

- ``cif``:   352x288, background value noise panned by up to 8 px (quarter-sample steps), sigma 2;
- ``1080p``: 1920x1080, pan up to 6 px, 8 moving rectangles at up to 12 px/frame, sigma 3;
- ``4k``:    3840x2160, pan up to 6 px, 32 rectangles at up to 24 px/frame, sigma 3;
- ``stream``: a batched-form stream (any resolution), the 1080p generator's settings.
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

from . import build as _build

CONFIGS = {
    # name: (width, height, seed, pan_q, nobj, vmax, sigma)
    "cif": (352, 288, 0x1A2B0000, 32, 0, 0.0, 2.0),
    "1080p": (1920, 1080, 0x1A2B0001, 24, 8, 12.0, 3.0),
    "4k": (3840, 2160, 0x1A2B0002, 24, 32, 24.0, 3.0),
}

_LIB = None


def _lib() -> ctypes.CDLL:
    global _LIB
    if _LIB is None:
        path = _build.SYNTH_LIB
        if not os.path.exists(path):
            _build.build_synth()
        lib = ctypes.CDLL(path)
        lib.ironav_synth_create.restype = ctypes.c_void_p
        lib.ironav_synth_create.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_uint64,
                                            ctypes.c_int, ctypes.c_int, ctypes.c_double, ctypes.c_double]
        lib.ironav_synth_destroy.argtypes = [ctypes.c_void_p]
        lib.ironav_synth_frame.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p, ctypes.c_int]
        lib.ironav_synth_draws.argtypes = [ctypes.c_uint64, ctypes.c_int, ctypes.c_int, ctypes.c_void_p]
        lib.ironav_synth_pan.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.POINTER(ctypes.c_int),
                                         ctypes.POINTER(ctypes.c_int)]
        _LIB = lib
    return _LIB


# The batched configuration: 64 streams, resolutions drawn from these by std::mt19937_64(0x1A2B03FF),
# stream s seeded 0x1A2B0300 + s, each with the encoder's slice count on a >= 8-core host.
BATCH_SIZES = [(640, 360, 2), (854, 480, 3), (1280, 720, 5), (1920, 1080, 8)]
BATCH_SEED = 0x1A2B03FF


def batch_streams(n: int = 64) -> list[tuple[int, int, int, int]]:
    """(width, height, slice bands, seed) of the batched configuration's streams."""
    idx = np.zeros(n, dtype=np.int32)
    _lib().ironav_synth_draws(BATCH_SEED, n, len(BATCH_SIZES), idx.ctypes.data)
    return [BATCH_SIZES[int(k)] + (0x1A2B0300 + s,) for s, k in enumerate(idx)]


class Sequence:
    """Frames 0..frames-1 of one seeded sequence; each frame can be generated on its own."""

    def __init__(self, width: int, height: int, frames: int, seed: int, pan_q: int, nobj: int, vmax: float,
                 sigma: float):
        self.width, self.height, self.frames, self.seed = width, height, frames, seed
        self._h = _lib().ironav_synth_create(width, height, frames, seed, pan_q, nobj, vmax, sigma)
        if not self._h:
            raise ValueError("bad synthetic sequence parameters")

    @classmethod
    def config(cls, name: str, frames: int, seed: int | None = None, size: tuple[int, int] | None = None):
        w, h, s, pan_q, nobj, vmax, sigma = CONFIGS[name]
        if size is not None:
            w, h = size
        return cls(w, h, frames, s if seed is None else seed, pan_q, nobj, vmax, sigma)

    def frame(self, t: int) -> np.ndarray:
        out = np.empty((self.height, self.width), dtype=np.uint8)
        st = _lib().ironav_synth_frame(self._h, t, out.ctypes.data, self.width)
        if st != 0:
            raise IndexError(t)
        return out

    def frame10(self, t: int) -> np.ndarray:
        """Frame t as 10-bit luma (the encoder's Yuv420p10 input): the 8-bit frame times 4 plus two seeded
        low bits per sample, so the low bits carry detail the 8-bit frame does not have."""
        rng = np.random.default_rng([self.seed, t, 10])
        low = rng.integers(0, 4, size=(self.height, self.width), dtype=np.uint16)
        return (self.frame(t).astype(np.uint16) << 2) | low

    def pan(self, t: int) -> tuple[int, int]:
        qx, qy = ctypes.c_int(), ctypes.c_int()
        _lib().ironav_synth_pan(self._h, t, ctypes.byref(qx), ctypes.byref(qy))
        return qx.value, qy.value

    def __del__(self):
        h = getattr(self, "_h", None)
        if h:
            _lib().ironav_synth_destroy(h)
            self._h = None
