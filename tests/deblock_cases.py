"""Seeded deblocking inputs for the tests: 4:2:0 reconstructions whose 4x4 blocks carry small steps (so
that the filter's thresholds pass on many edges), and macroblock records / slice tables that exercise
every branch of the reference's filter (h264/deblock.rs): intra and inter neighbours, coded blocks, one
and two reference lists, vectors around the whole-sample limit, uniform inter macroblocks, the 8x8
transform, I_PCM / lossless (keep) macroblocks, uncoded macroblocks, and slices that are filtered, left
alone, or filtered only inside their edges, with filter and chroma QP offsets."""
from __future__ import annotations

import numpy as np

from ironav_b200.inter import DBK_MB_DTYPE, DBK_SLICE_DTYPE


def planes(rng, mb_w: int, mb_h: int, bd: int = 8):
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


def records(rng, mb_w: int, mb_h: int, nslices: int, bd: int = 8, slice_rows: bool = False):
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


def encoder_slices(nslices: int):
    """The encoder's slice table: every slice filtered with no offsets (enc/mod.rs:653)."""
    return np.zeros(nslices, dtype=DBK_SLICE_DTYPE)
