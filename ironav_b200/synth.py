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
from .inter import DBK_MB_DTYPE, DBK_SLICE_DTYPE

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

    def chroma(self, t: int, bd: int = 8) -> tuple[np.ndarray, np.ndarray]:
        """4:2:0 chroma for frame t (the sequences are generated as luma; chroma is derived from it so that it
        moves with the picture): Cb from the 2x2 luma means compressed around 128, Cr inverted; 10-bit
        from the 10-bit frame."""
        y = (self.frame10(t) if bd > 8 else self.frame(t)).astype(np.int32)
        h2, w2 = self.height // 2, self.width // 2
        m = (y[0:2 * h2:2, 0:2 * w2:2] + y[1:2 * h2:2, 0:2 * w2:2] + y[0:2 * h2:2, 1:2 * w2:2] + y[1:2 * h2:2, 1:2 * w2:2] + 2) >> 2
        half = 1 << (bd - 1)
        cb = half + ((m - half) * 3 >> 2)
        cr = half - ((m - half) >> 1)
        dt = np.uint8 if bd == 8 else np.uint16
        return cb.astype(dt), cr.astype(dt)

    def pan(self, t: int) -> tuple[int, int]:
        qx, qy = ctypes.c_int(), ctypes.c_int()
        _lib().ironav_synth_pan(self._h, t, ctypes.byref(qx), ctypes.byref(qy))
        return qx.value, qy.value

    def __del__(self):
        h = getattr(self, "_h", None)
        if h:
            _lib().ironav_synth_destroy(h)
            self._h = None


# ---- deblocking inputs ---------------------------------------------------------------------------------
# Seeded stand-ins for a reconstructed 4:2:0 picture and its macroblock records (h264/deblock.rs reads
# them): the 4x4 blocks carry small steps so that the filter's thresholds pass on many edges, and the
# records exercise every branch of the filter: intra and inter neighbours, coded blocks, one and two
# reference lists, vectors around the whole-sample limit, uniform inter macroblocks, the 8x8 transform,
# I_PCM / lossless (keep) macroblocks, uncoded macroblocks, and slices that are filtered, left alone, or
# filtered only inside their edges, with filter and chroma QP offsets.

def dbk_planes(rng, mb_w: int, mb_h: int, bd: int = 8):
    """(y, cb, cr): a smooth ramp plus per-4x4-block offsets plus sample noise, clipped to bd bits."""
    maxv = (1 << bd) - 1
    s = 1 << (bd - 8)

    def one(h, w, blk):
        yy, xx = np.mgrid[0:h, 0:w]
        base = 96 * s + (xx * 3 + yy * 2) * s // 4
        steps = rng.integers(-12 * s, 13 * s, size=(h // blk + 1, w // blk + 1))
        v = base + steps[yy // blk, xx // blk] + rng.integers(-2 * s, 3 * s, size=(h, w))
        # a few sharp features the filter must leave alone
        v[rng.random((h, w)) < 0.01] = maxv
        return np.clip(v, 0, maxv).astype(np.uint8 if bd == 8 else np.uint16)

    return one(mb_h * 16, mb_w * 16, 4), one(mb_h * 8, mb_w * 8, 2), one(mb_h * 8, mb_w * 8, 2)


def dbk_records(rng, mb_w: int, mb_h: int, nslices: int, bd: int = 8, slice_rows: bool = False):
    """Macroblock records and a slice table. slice_rows: slices are bands of macroblock rows (as the
    encoder cuts them); otherwise slice ids are drawn per macroblock."""
    n = mb_w * mb_h
    m = np.zeros(n, dtype=DBK_MB_DTYPE)
    if slice_rows:
        rows = np.arange(n) // mb_w
        m["slice"] = 1 + rows * nslices // mb_h
    else:
        m["slice"] = rng.integers(1, nslices + 1, n)
        m["slice"][rng.random(n) < 0.03] = 0  # not coded
    m["inter"] = rng.random(n) < 0.8
    lo = -6 * (bd - 8)
    m["qp"] = rng.integers(max(lo, 10), 52, n)
    low = rng.random(n) < 0.1  # low QPs too (alpha 0: edges left alone), negative ones at 10 bits
    m["qp"][low] = rng.integers(lo, 20, int(low.sum()))
    m["t8x8"] = rng.random(n) < 0.25
    m["keep"] = rng.random(n) < 0.05
    nnz = rng.integers(0, 3, size=(n, 16)) * (rng.random((n, 16)) < 0.3)
    m["nnz"] = nnz
    # references: list 0 in most inter macroblocks, list 1 in some (bi-predicted or list 1 only)
    use0 = rng.random((n, 4)) < 0.85
    use1 = rng.random((n, 4)) < 0.3
    use0 |= ~use1
    rid0 = rng.integers(0, 3, size=(n, 4))
    rid1 = rng.integers(0, 3, size=(n, 4))
    m["ref_id"][:, 0] = np.where(use0, rid0, -1)
    m["ref_id"][:, 1] = np.where(use1, rid1, -1)
    m["ref_idx"][:, 0] = np.where(use0, rid0, -1)
    m["ref_idx"][:, 1] = np.where(use1, rid1, -1)
    base = rng.integers(-20, 21, size=(n, 2, 1, 2))
    jitter = rng.integers(-5, 6, size=(n, 2, 16, 2)) * (rng.random((n, 2, 16, 1)) < 0.4)
    m["mv"] = base + jitter
    # uniform inter macroblocks with no coefficients: their inner edges are not filtered
    uni = rng.random(n) < 0.2
    m["mv"][uni] = m["mv"][uni][:, :, :1, :]
    m["ref_id"][uni] = m["ref_id"][uni][:, :, :1]
    m["ref_idx"][uni] = m["ref_idx"][uni][:, :, :1]
    m["nnz"][uni] = 0
    # intra macroblocks keep no motion
    intra = m["inter"] == 0
    m["ref_id"][intra] = -1
    m["ref_idx"][intra] = -1
    m["mv"][intra] = 0
    s = np.zeros(nslices, dtype=DBK_SLICE_DTYPE)
    s["disable_deblocking"] = rng.choice([0, 0, 0, 1, 2], nslices)
    s["alpha_offset"] = rng.integers(-6, 7, nslices) * 2
    s["beta_offset"] = rng.integers(-6, 7, nslices) * 2
    s["chroma_qp_offset"] = rng.integers(-12, 13, size=(nslices, 2))
    return m, s


def dbk_encoder_slices(nslices: int):
    """The encoder's slice table: every slice filtered with no offsets (enc/mod.rs:653)."""
    return np.zeros(nslices, dtype=DBK_SLICE_DTYPE)
