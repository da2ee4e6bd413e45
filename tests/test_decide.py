"""Decide mode: the whole P macroblock decision of the CAVLC encoder (code_mb, enc/frame.rs:715-790) with
intra prediction (best_i16, code_i4, code_i16, code_intra_chroma; h264/intra.rs) and the coding of the
chosen macroblock, in each slice band's raster order.

CPU: the oracle's reconstruction of every intra macroblock is what a decoder makes of its code — checked
by an independent statement of ITU-T H.264 8.3 (intra prediction) and 8.5 (scaling and the inverse
transforms) — its P_Skip macroblocks reconstruct to their prediction, states follow codes, and the
reconstruction follows the source. GPU: the sm_100a library against the oracle, every code field, state
and reconstructed sample.
"""
from __future__ import annotations

import os

import numpy as np
import pytest

from ironav_b200.inter import KIND_I4X4, KIND_I16X16, KIND_INTER, MBCODE_DTYPE, InterStage
from ironav_b200.synth import Sequence

ZZ4 = np.array([0, 1, 4, 8, 5, 2, 3, 6, 9, 12, 13, 10, 7, 11, 14, 15])
V = np.array([[10, 16, 13], [11, 18, 14], [13, 20, 16], [14, 23, 18], [16, 25, 20], [18, 29, 23]])
CHROMA_QP = [29, 30, 31, 32, 32, 33, 34, 34, 35, 35, 36, 36, 37, 37, 37, 38, 38, 38, 39, 39, 39, 39]


def psnr(a, b, maxv=255):
    mse = float(np.mean((a.astype(np.float64) - b.astype(np.float64)) ** 2))
    return 99.0 if mse == 0 else 10 * np.log10(maxv * maxv / mse)


# ---- a decoder's view (ITU-T H.264 8.3, 8.5), written from the standard --------------------------------

def vclass(i):
    r, c = divmod(i, 4)
    return 0 if (r % 2 == 0 and c % 2 == 0) else (1 if (r % 2 == 1 and c % 2 == 1) else 2)


def dequant4(levels_scan, qp, skip_dc=False):
    """Scan-order levels of a 4x4 block to raster coefficients (flat scaling lists: LevelScale4x4 =
    16 * normAdjust4x4, d = (c * LevelScale) << (qP/6) >> 4)."""
    d = np.zeros(16, np.int64)
    for k in range(16):
        if skip_dc and k == 0:
            continue
        p = ZZ4[k]
        d[p] = (int(levels_scan[k]) * 16 * V[qp % 6][vclass(p)] << (qp // 6)) >> 4
    return d


def idct4(d):
    """8.5.12.2: the 4x4 inverse transform, (x + 32) >> 6 residual."""
    d = d.reshape(4, 4).astype(np.int64)
    f = np.zeros((4, 4), np.int64)
    for i in range(4):
        e0, e1 = d[i, 0] + d[i, 2], d[i, 0] - d[i, 2]
        e2, e3 = (d[i, 1] >> 1) - d[i, 3], d[i, 1] + (d[i, 3] >> 1)
        f[i] = [e0 + e3, e1 + e2, e1 - e2, e0 - e3]
    r = np.zeros((4, 4), np.int64)
    for j in range(4):
        g0, g1 = f[0, j] + f[2, j], f[0, j] - f[2, j]
        g2, g3 = (f[1, j] >> 1) - f[3, j], f[1, j] + (f[3, j] >> 1)
        r[:, j] = [g0 + g3, g1 + g2, g1 - g2, g0 - g3]
    return (r + 32) >> 6


def hadamard4(c):
    h = np.array([[1, 1, 1, 1], [1, 1, -1, -1], [1, -1, -1, 1], [1, -1, 1, -1]], np.int64)
    return h @ c.reshape(4, 4).astype(np.int64) @ h.T


def pred4(mode, top, left, tl, have_top, have_left, bd):
    """8.3.1.2: top holds p[x, -1] for x = 0..7, left p[-1, y], tl p[-1, -1]."""
    P = np.zeros((4, 4), np.int64)

    def t(x):
        return tl if x < 0 else top[x]

    def l(y):
        return tl if y < 0 else left[y]

    for y in range(4):
        for x in range(4):
            if mode == 0:
                v = t(x)
            elif mode == 1:
                v = l(y)
            elif mode == 2:
                if have_top and have_left:
                    v = (sum(top[:4]) + sum(left[:4]) + 4) >> 3
                elif have_left:
                    v = (sum(left[:4]) + 2) >> 2
                elif have_top:
                    v = (sum(top[:4]) + 2) >> 2
                else:
                    v = 1 << (bd - 1)
            elif mode == 3:  # diagonal down left
                v = (t(6) + 3 * t(7) + 2) >> 2 if x == 3 and y == 3 else (t(x + y) + 2 * t(x + y + 1) + t(x + y + 2) + 2) >> 2
            elif mode == 4:  # diagonal down right
                if x > y:
                    v = (t(x - y - 2) + 2 * t(x - y - 1) + t(x - y) + 2) >> 2
                elif x < y:
                    v = (l(y - x - 2) + 2 * l(y - x - 1) + l(y - x) + 2) >> 2
                else:
                    v = (t(0) + 2 * tl + l(0) + 2) >> 2
            elif mode == 5:  # vertical right
                z = 2 * x - y
                if z >= 0 and z % 2 == 0:
                    v = (t(x - (y >> 1) - 1) + t(x - (y >> 1)) + 1) >> 1
                elif z >= 0:
                    v = (t(x - (y >> 1) - 2) + 2 * t(x - (y >> 1) - 1) + t(x - (y >> 1)) + 2) >> 2
                elif z == -1:
                    v = (l(0) + 2 * tl + t(0) + 2) >> 2
                else:
                    v = (l(y - 1) + 2 * l(y - 2) + l(y - 3) + 2) >> 2
            elif mode == 6:  # horizontal down
                z = 2 * y - x
                if z >= 0 and z % 2 == 0:
                    v = (l(y - (x >> 1) - 1) + l(y - (x >> 1)) + 1) >> 1
                elif z >= 0:
                    v = (l(y - (x >> 1) - 2) + 2 * l(y - (x >> 1) - 1) + l(y - (x >> 1)) + 2) >> 2
                elif z == -1:
                    v = (l(0) + 2 * tl + t(0) + 2) >> 2
                else:
                    v = (t(x - 1) + 2 * t(x - 2) + t(x - 3) + 2) >> 2
            elif mode == 7:  # vertical left
                i = x + (y >> 1)
                v = (t(i) + t(i + 1) + 1) >> 1 if y % 2 == 0 else (t(i) + 2 * t(i + 1) + t(i + 2) + 2) >> 2
            else:  # horizontal up
                z = x + 2 * y
                if z > 5:
                    v = l(3)
                elif z == 5:
                    v = (l(2) + 3 * l(3) + 2) >> 2
                elif z % 2 == 0:
                    v = (l(y + (x >> 1)) + l(y + (x >> 1) + 1) + 1) >> 1
                else:
                    v = (l(y + (x >> 1)) + 2 * l(y + (x >> 1) + 1) + l(y + (x >> 1) + 2) + 2) >> 2
            P[y, x] = v
    return P


def pred_plane(top, left, tl, n_x, n_y, bd):
    """8.3.3.4 / 8.3.4.4 plane prediction over an n_x x n_y block (16x16 luma or 8x8 chroma)."""
    xc, yc = n_x // 2, n_y // 2

    def t(i):
        return tl if i < 0 else top[i]

    def l(i):
        return tl if i < 0 else left[i]

    H = sum((k + 1) * (t(xc + k) - t(xc - 2 - k)) for k in range(xc))
    Vv = sum((k + 1) * (l(yc + k) - l(yc - 2 - k)) for k in range(yc))
    a = 16 * (left[n_y - 1] + top[n_x - 1])
    b = (5 * H + 32) >> 6 if n_x == 16 else (34 * H + 32) >> 6
    c = (5 * Vv + 32) >> 6 if n_y == 16 else (34 * Vv + 32) >> 6
    y, x = np.mgrid[0:n_y, 0:n_x]
    return np.clip((a + b * (x - (xc - 1)) + c * (y - (yc - 1)) + 16) >> 5, 0, (1 << bd) - 1)


def pred16(mode, top, left, tl, ht, hl, bd):
    if mode == 0:
        return np.tile(np.array(top[:16], np.int64), (16, 1))
    if mode == 1:
        return np.tile(np.array(left[:16], np.int64)[:, None], (1, 16))
    if mode == 2:
        st, sl = sum(top[:16]), sum(left[:16])
        v = (st + sl + 16) >> 5 if ht and hl else ((sl + 8) >> 4 if hl else ((st + 8) >> 4 if ht else 1 << (bd - 1)))
        return np.full((16, 16), v, np.int64)
    return pred_plane(top, left, tl, 16, 16, bd)


def pred_chroma(mode, top, left, tl, ht, hl, bd):
    """8.3.4 with intra_chroma_pred_mode 0 DC, 1 horizontal, 2 vertical, 3 plane (8x8)."""
    if mode == 1:
        return np.tile(np.array(left[:8], np.int64)[:, None], (1, 8))
    if mode == 2:
        return np.tile(np.array(top[:8], np.int64), (8, 1))
    if mode == 3:
        return pred_plane(top, left, tl, 8, 8, bd)
    out = np.zeros((8, 8), np.int64)
    mid = 1 << (bd - 1)
    for by in range(2):
        for bx in range(2):
            st, sl = sum(top[bx * 4:bx * 4 + 4]), sum(left[by * 4:by * 4 + 4])
            if bx == by:  # (0,0) and (1,1): both edges when both exist
                v = (st + sl + 4) >> 3 if ht and hl else ((sl + 2) >> 2 if hl else ((st + 2) >> 2 if ht else mid))
            elif bx == 1:  # (1,0): the row above first
                v = (st + 2) >> 2 if ht else ((sl + 2) >> 2 if hl else mid)
            else:  # (0,1): the column to the left first
                v = (sl + 2) >> 2 if hl else ((st + 2) >> 2 if ht else mid)
            out[by * 4:by * 4 + 4, bx * 4:bx * 4 + 4] = v
    return out


def zorder(bx, by):
    """The decoding order of the 4x4 block at raster position (bx, by) (6.4.3)."""
    return ((by >> 1) << 3) | ((bx >> 1) << 2) | ((by & 1) << 1) | (bx & 1)


def chroma_qp(qp_y, bd):
    q = max(-6 * (bd - 8), min(51, qp_y))
    return q if q < 30 else CHROMA_QP[q - 30]


def check_intra_decodes(st: InterStage, codes, rec, qp_y: int, band_start):
    """Every intra macroblock's reconstruction equals its prediction from the (decoded) samples around it
    plus its dequantised, inverse-transformed residual. Returns the numbers of I4x4 and I16x16 checked."""
    y_rec, cb_rec, cr_rec = (a.astype(np.int64) for a in rec)
    bd = st.bd
    maxv = (1 << bd) - 1
    qp = qp_y + 6 * (bd - 8)
    qpc = chroma_qp(qp_y, bd) + 6 * (bd - 8)
    n4 = n16 = 0
    for mb in np.nonzero(codes["kind"] != KIND_INTER)[0]:
        c = codes[mb]
        mbx, mby = int(mb) % st.mb_w, int(mb) // st.mb_w
        ta, la = mby > band_start[mby], mbx > 0
        tra = ta and mbx + 1 < st.mb_w
        x0, y0 = mbx * 16, mby * 16
        if c["kind"] == KIND_I4X4:
            n4 += 1
            for n in range(16):
                bx, by = ((n >> 2) & 1) * 2 + (n & 1), ((n >> 3) & 1) * 2 + ((n >> 1) & 1)
                x, y = x0 + bx * 4, y0 + by * 4
                ht, hl = by > 0 or ta, bx > 0 or la
                htl = (by > 0 or ta) and (bx > 0 or la)
                if by == 0:
                    htr = ta if bx < 3 else tra
                else:  # inside the macroblock: available when decoded before this block (6.4.11.4)
                    htr = bx < 3 and zorder(bx + 1, by - 1) < zorder(bx, by)
                top = [0] * 8
                if ht:
                    top[:4] = list(y_rec[y - 1, x:x + 4])
                    top[4:] = list(y_rec[y - 1, x + 4:x + 8]) if htr else [top[3]] * 4
                left = list(y_rec[y:y + 4, x - 1]) if hl else [0] * 4
                tl = int(y_rec[y - 1, x - 1]) if htl else 0
                p = pred4(int(c["modes"][by * 4 + bx]), [int(v) for v in top], [int(v) for v in left], tl, ht, hl, bd)
                r = idct4(dequant4(c["res"]["luma"][by * 4 + bx], qp))
                want = np.clip(p + r, 0, maxv)
                got = y_rec[y:y + 4, x:x + 4]
                assert np.array_equal(got, want), f"I4x4 mb {mb} block ({bx},{by}) mode {c['modes'][by * 4 + bx]}"
        else:
            n16 += 1
            top = [int(v) for v in y_rec[y0 - 1, x0:x0 + 16]] if ta else [0] * 16
            left = [int(v) for v in y_rec[y0:y0 + 16, x0 - 1]] if la else [0] * 16
            tl = int(y_rec[y0 - 1, x0 - 1]) if ta and la else 0
            p = pred16(int(c["i16_mode"]), top, left, tl, ta, la, bd)
            dcl = np.zeros(16, np.int64)
            dcl[ZZ4] = c["dc"]
            f = hadamard4(dcl).reshape(16)
            ls = 16 * V[qp % 6][0]
            dcs = (f * ls) << (qp // 6 - 6) if qp >= 36 else (f * ls + (1 << (5 - qp // 6))) >> (6 - qp // 6)
            for b in range(16):
                bx, by = b % 4, b // 4
                d = dequant4(c["res"]["luma"][b], qp, skip_dc=True)
                d[0] = dcs[b]
                want = np.clip(p[by * 4:by * 4 + 4, bx * 4:bx * 4 + 4] + idct4(d), 0, maxv)
                got = y_rec[y0 + by * 4:y0 + by * 4 + 4, x0 + bx * 4:x0 + bx * 4 + 4]
                assert np.array_equal(got, want), f"I16x16 mb {mb} block {b} mode {c['i16_mode']}"
        # intra chroma
        cbpc = int(c["res"]["cbp"]) >> 4
        for comp, plane in enumerate((cb_rec, cr_rec)):
            cx0, cy0 = mbx * 8, mby * 8
            top = [int(v) for v in plane[cy0 - 1, cx0:cx0 + 8]] if ta else [0] * 8
            left = [int(v) for v in plane[cy0:cy0 + 8, cx0 - 1]] if la else [0] * 8
            tl = int(plane[cy0 - 1, cx0 - 1]) if ta and la else 0
            p = pred_chroma(int(c["chroma_mode"]), top, left, tl, ta, la, bd)
            want = np.clip(p + chroma_residual(c["res"], comp, qpc), 0, maxv)
            got = plane[cy0:cy0 + 8, cx0:cx0 + 8]
            assert np.array_equal(got, want), f"intra chroma mb {mb} comp {comp} mode {c['chroma_mode']} cbp {cbpc}"
    return n4, n16


def chroma_residual(res, comp, qpc):
    """The 8x8 residual of one chroma component (8.5.11: the 2x2 DC transform and scaling, then the 4x4
    blocks' AC levels), as coded_block_pattern's chroma part says: 0 none, 1 DC only, 2 DC and AC."""
    cbpc = int(res["cbp"]) >> 4
    out = np.zeros((8, 8), np.int64)
    if cbpc == 0:
        return out
    l4 = res["cdc"][comp].astype(np.int64)
    f = np.array([l4[0] + l4[1] + l4[2] + l4[3], l4[0] - l4[1] + l4[2] - l4[3], l4[0] + l4[1] - l4[2] - l4[3],
                  l4[0] - l4[1] - l4[2] + l4[3]])
    dcc = ((f * 16 * V[qpc % 6][0]) << (qpc // 6)) >> 5
    for blk in range(4):
        d = dequant4(res["cac"][comp][blk], qpc, skip_dc=True) if cbpc == 2 else np.zeros(16, np.int64)
        d[0] = dcc[blk]
        bx, by = blk & 1, blk >> 1
        out[by * 4:by * 4 + 4, bx * 4:bx * 4 + 4] = idct4(d)
    return out


# ---- cases -----------------------------------------------------------------------------------------

def decide_case(lib, cfg="cif", size=None, qp=22, bd=8, nslices=2, refs=1, fast=False, sub8=False, new_content=False,
                threads=True):
    """A P picture (frame 1) from frame 0 (and frame 2 when refs == 2); new_content: the references come
    from an unrelated sequence, so that intra competes everywhere."""
    seq = Sequence.config(cfg, 4, size=size)
    other = Sequence(seq.width, seq.height, 4, seq.seed + 77, 3, 4, 6, 3.0) if new_content else seq
    fr = [seq.frame10(t) if bd == 10 else seq.frame(t) for t in range(4)]
    ch = [seq.chroma(t, bd) for t in range(4)]
    rf = [other.frame10(t) if bd == 10 else other.frame(t) for t in range(4)] if new_content else fr
    rc = [other.chroma(t, bd) for t in range(4)] if new_content else ch
    st = InterStage(seq.width, seq.height, max_refs=3, nslices=nslices, lib=lib, bd=bd)
    if threads and hasattr(lib, "oracle_set_threads"):
        lib.oracle_set_threads(st.ctx, os.cpu_count() or 1)
    for t in {1: [0], 2: [2, 0], 3: [3, 2, 0]}[refs]:
        st.push_reference(rf[t])
        st.push_reference_chroma(*rc[t])
    st.set_source(fr[1])
    st.set_source_chroma(*ch[1])
    st.begin_p_picture(qp + 6 * (bd - 8), nrefs_active=refs, fast=fast, sub8=sub8)
    return st, fr, ch


def band_starts(st: InterStage, nslices: int):
    rows = st.mb_h
    starts = [(rows * k) // nslices for k in range(nslices)]
    out = np.zeros(rows, int)
    for r in range(rows):
        out[r] = max(s for s in starts if s <= r)
    return out


@pytest.mark.parametrize("kw", [dict(), dict(new_content=True), dict(new_content=True, qp=34, nslices=3),
                                dict(new_content=True, bd=10, qp=16), dict(fast=True, qp=28), dict(refs=2, sub8=True, qp=26)])
def test_oracle_intra_macroblocks_decode(oracle_lib, kw):
    st, fr, ch = decide_case(oracle_lib, **kw)
    states, codes, rec = st.decide_p_picture()
    qp = kw.get("qp", 22)
    n4, n16 = check_intra_decodes(st, codes, rec, qp, band_starts(st, kw.get("nslices", 2)))
    if kw.get("new_content"):
        assert n4 > 20 and n16 > 5, (n4, n16)
    # states follow the codes
    inter = codes["kind"] == KIND_INTER
    assert np.array_equal(states["inter"] == 1, inter)
    assert (states["refs"][~inter] == -1).all() and (states["mvs"][~inter] == 0).all()
    assert (states["refs"][inter] >= 0).all()
    # P_Skip: 16x16 from reference 0, no levels
    skip = codes["skip"] == 1
    assert (codes["res"]["cbp"][skip] == 0).all() and (codes["part"][skip] == 0).all() and (codes["refs"][skip] == 0).all()
    assert (codes["mvs"][skip] == codes["mvs"][skip][:, :1]).all()
    assert (codes["kind"][skip] == KIND_INTER).all()
    # the reconstruction follows the source
    h, w = fr[1].shape
    maxv = (1 << st.bd) - 1
    assert psnr(rec[0][:h, :w], fr[1], maxv) > (30 if qp > 30 else 36)


def test_oracle_skip_reconstructs_the_prediction(oracle_lib):
    """A P_Skip macroblock's samples are those code_inter gives its skip vector with no residual: the
    residual stage coding it as P_Skip reproduces them."""
    from ironav_b200.inter import INTERDEC_DTYPE

    st, fr, ch = decide_case(oracle_lib, qp=30)
    states, codes, rec = st.decide_p_picture()
    skip = codes["skip"] == 1
    assert skip.sum() > 50
    decs = np.zeros(st.nmb, dtype=INTERDEC_DTYPE)
    decs["mode"] = np.where(skip, 1, 0)
    decs["mvs"] = codes["mvs"]
    blank = tuple(np.zeros_like(a) for a in rec)
    _, (y2, cb2, cr2) = st.code_inter(30, decs, blank)
    for mb in np.nonzero(skip)[0][:200]:
        mbx, mby = int(mb) % st.mb_w, int(mb) // st.mb_w
        assert np.array_equal(y2[mby * 16:mby * 16 + 16, mbx * 16:mbx * 16 + 16], rec[0][mby * 16:mby * 16 + 16, mbx * 16:mbx * 16 + 16])
        assert np.array_equal(cb2[mby * 8:mby * 8 + 8, mbx * 8:mbx * 8 + 8], rec[1][mby * 8:mby * 8 + 8, mbx * 8:mbx * 8 + 8])


def test_mbcode_layout_matches_the_header():
    assert MBCODE_DTYPE.itemsize == 1516
    assert MBCODE_DTYPE.fields["dc"][1] == 1324 and MBCODE_DTYPE.fields["kind"][1] == 1500


# ---- GPU: the sm_100a library against the oracle ------------------------------------------------------------

def _same_decisions(got, want, what):
    (s_g, c_g, r_g), (s_w, c_w, r_w) = got, want
    if not np.array_equal(c_g, c_w):
        bad = np.nonzero(c_g != c_w)[0]
        i = int(bad[0])
        fields = [f for f in MBCODE_DTYPE.names if not np.array_equal(c_g[i][f], c_w[i][f])]
        if "res" in fields:
            fields += [f"res.{f}" for f in c_g.dtype["res"].names if not np.array_equal(c_g[i]["res"][f], c_w[i]["res"][f])]
        raise AssertionError(f"{what}: {len(bad)} macroblocks' codes differ; first {i} (kind {c_g[i]['kind']} vs "
                             f"{c_w[i]['kind']}), fields {fields}")
    assert np.array_equal(s_g, s_w), f"{what}: states differ at {np.nonzero(s_g != s_w)[0][:5].tolist()}"
    for name, a, b in zip("Y Cb Cr".split(), r_g, r_w):
        assert np.array_equal(a, b), f"{what}: {name} differs at {np.argwhere(a != b)[:4].tolist()}"


@pytest.mark.gpu
@pytest.mark.parametrize("kw", [dict(), dict(qp=30), dict(new_content=True), dict(new_content=True, qp=40, nslices=3),
                                dict(fast=True, qp=28), dict(refs=2, sub8=True, qp=26), dict(new_content=True, bd=10, qp=16),
                                dict(bd=10, qp=24, fast=True), dict(cfg="1080p", nslices=8, qp=27),
                                dict(cfg="1080p", size=(1280, 720), new_content=True, nslices=4, qp=32)])
def test_gpu_decide_matches_oracle(oracle_lib, cuda_lib, kw):
    o, _, _ = decide_case(oracle_lib, **kw)
    c, _, _ = decide_case(cuda_lib, threads=False, **kw)
    _same_decisions(c.decide_p_picture(), o.decide_p_picture(), str(kw))


@pytest.mark.gpu
@pytest.mark.parametrize("kw", [dict(refs=3, sub8=True, qp=18), dict(refs=3, qp=30, nslices=3, new_content=True),
                                dict(refs=2, bd=10, fast=True, qp=22), dict(refs=3, bd=10, sub8=True, qp=20, new_content=True)])
def test_gpu_decide_three_references(oracle_lib, cuda_lib, kw):
    """Up to three active references (the reference-index bits take their ue(v) length), with sub-8x8
    partitions, fast mode and 10-bit pictures."""
    o, _, _ = decide_case(oracle_lib, **kw)
    c, _, _ = decide_case(cuda_lib, threads=False, **kw)
    _same_decisions(c.decide_p_picture(), o.decide_p_picture(), str(kw))


@pytest.mark.gpu
@pytest.mark.parametrize("qp", [0, 10, 51])
def test_gpu_decide_extreme_qp(oracle_lib, cuda_lib, qp):
    o, _, _ = decide_case(oracle_lib, size=(176, 144), qp=qp, new_content=qp == 0)
    c, _, _ = decide_case(cuda_lib, size=(176, 144), qp=qp, new_content=qp == 0, threads=False)
    _same_decisions(c.decide_p_picture(), o.decide_p_picture(), f"qp {qp}")


@pytest.mark.gpu
def test_gpu_decide_device_form_and_refusals(oracle_lib, cuda_lib):
    import torch

    from ironav_b200.inter import MBSTATE_DTYPE

    o, _, _ = decide_case(oracle_lib, new_content=True)
    c, _, _ = decide_case(cuda_lib, new_content=True, threads=False)
    want = o.decide_p_picture()
    c.set_stream(torch.cuda.current_stream().cuda_stream)
    y = torch.zeros((c.mb_h * 16, c.mb_w * 16), dtype=torch.uint8, device="cuda")
    cc = torch.zeros((2, c.mb_h * 8, c.mb_w * 8), dtype=torch.uint8, device="cuda")
    ts = torch.full((c.nmb * 72,), 0x5A, dtype=torch.uint8, device="cuda")
    tc = torch.full((c.nmb * 1516,), 0x5A, dtype=torch.uint8, device="cuda")
    assert c.lib.ironav_decide_p_picture_device(c.ctx, ts.data_ptr(), tc.data_ptr(), y.data_ptr(), y.shape[1], cc[0].data_ptr(),
                                                cc[1].data_ptr(), cc.shape[2]) == 0
    c.sync()
    got = (ts.cpu().numpy().view(MBSTATE_DTYPE), tc.cpu().numpy().view(MBCODE_DTYPE), (y.cpu().numpy(), cc[0].cpu().numpy(), cc[1].cpu().numpy()))
    _same_decisions(got, want, "device form")
    # records the kernel writes word-wise, and a reference without chroma, are refused before any launch
    assert c.lib.ironav_decide_p_picture_device(c.ctx, ts.data_ptr() + 2, tc.data_ptr(), y.data_ptr(), y.shape[1], cc[0].data_ptr(),
                                                cc[1].data_ptr(), cc.shape[2]) == 3
    c.set_stream(None)
    c.push_reference(np.zeros((c.height, c.width), np.uint8))  # no chroma attached
    c.begin_p_picture(22)
    with pytest.raises(Exception):
        c.decide_p_picture()


@pytest.mark.gpu
@pytest.mark.parametrize("size,nslices", [((16, 16), 1), ((32, 16), 1), ((48, 48), 3), ((176, 144), 9), ((200, 120), 2)])
def test_gpu_decide_small_and_ragged_pictures(oracle_lib, cuda_lib, size, nslices):
    """One macroblock, one row, a slice per macroblock row, and sizes that are not whole macroblocks
    (the source and references padded by repeating their edges)."""
    for new_content in (False, True):
        o, _, _ = decide_case(oracle_lib, size=size, nslices=nslices, new_content=new_content, qp=24)
        c, _, _ = decide_case(cuda_lib, size=size, nslices=nslices, new_content=new_content, qp=24, threads=False)
        _same_decisions(c.decide_p_picture(), o.decide_p_picture(), f"{size} {nslices} {new_content}")


@pytest.mark.gpu
@pytest.mark.parametrize("bd", [8, 10])
def test_gpu_batched_decide_matches_single_streams(oracle_lib, cuda_lib, bd):
    """Four streams of different sizes, slice layouts and content decided in one launch: each stream's
    codes, states and reconstruction are those of its own decide call (and so the oracle's); a batch of
    8-bit streams and one of 10-bit streams."""
    import torch

    from ironav_b200.inter import MBSTATE_DTYPE, InterBatch

    cases = [dict(), dict(new_content=True, qp=30), dict(size=(320, 176), nslices=3, fast=True), dict(cfg="1080p", nslices=8, qp=27)]
    cases = [dict(kw, bd=bd) for kw in cases]
    stages = [decide_case(cuda_lib, threads=False, **kw)[0] for kw in cases]
    want = [st.decide_p_picture() for st in stages]
    o = decide_case(oracle_lib, **cases[1])[0]
    _same_decisions(want[1], o.decide_p_picture(), "single stream, intra-heavy")
    stream = torch.cuda.Stream()
    for st in stages:
        st.set_stream(stream.cuda_stream)
    bufs = []
    dt = torch.uint8 if bd == 8 else torch.int16
    for st in stages:
        bufs.append((torch.zeros(st.nmb * 72, dtype=torch.uint8, device="cuda"), torch.full((st.nmb * 1516,), 0x5A, dtype=torch.uint8, device="cuda"),
                     torch.zeros((st.mb_h * 16, st.mb_w * 16), dtype=dt, device="cuda"),
                     torch.zeros((2, st.mb_h * 8, st.mb_w * 8), dtype=dt, device="cuda")))
    batch = InterBatch(stages)
    for _ in range(2):  # twice: the flags are cleared every launch
        batch.decide([b[0].data_ptr() for b in bufs], [b[1].data_ptr() for b in bufs], [b[2].data_ptr() for b in bufs],
                     [b[2].shape[1] for b in bufs], [b[3][0].data_ptr() for b in bufs], [b[3][1].data_ptr() for b in bufs],
                     [b[3].shape[2] for b in bufs])
        batch.sync()
    view = (lambda t: t.cpu().numpy().view(np.uint16)) if bd == 10 else (lambda t: t.cpu().numpy())
    for k, (st, b) in enumerate(zip(stages, bufs)):
        got = (b[0].cpu().numpy().view(MBSTATE_DTYPE), b[1].cpu().numpy().view(MBCODE_DTYPE), (view(b[2]), view(b[3][0]), view(b[3][1])))
        _same_decisions(got, want[k], f"stream {k} {cases[k]}")
    batch.close()


@pytest.mark.gpu
def test_gpu_decide_wait_times_out_and_recovers(oracle_lib, cuda_lib):
    """A macroblock whose flag is never published (the test withholds it, on the host) makes the waits
    behind it give up after a bounded number of polls: the call reports a timeout, the context stays
    usable, and the next picture is the oracle's. The same in a batch, where one stream's wait ends the launch."""
    import torch

    from ironav_b200.inter import InterBatch, IronavError

    o, _, _ = decide_case(oracle_lib, new_content=True)
    c, _, _ = decide_case(cuda_lib, new_content=True, threads=False)
    assert cuda_lib.ironav_debug_wait_limit(c.ctx, 20000) == 0
    assert cuda_lib.ironav_debug_withhold(c.ctx, 5) == 0
    with pytest.raises(IronavError) as e:
        c.decide_p_picture()
    assert e.value.status == 100
    assert cuda_lib.ironav_debug_withhold(c.ctx, -1) == 0
    assert cuda_lib.ironav_debug_wait_limit(c.ctx, 1 << 22) == 0  # the default: a whole picture's waits fit in it
    _same_decisions(c.decide_p_picture(), o.decide_p_picture(), "after a timeout")

    c2, _, _ = decide_case(cuda_lib, threads=False)
    stream = torch.cuda.Stream()
    for st in (c, c2):
        st.set_stream(stream.cuda_stream)
    bufs = [(torch.zeros(st.nmb * 72, dtype=torch.uint8, device="cuda"), torch.zeros(st.nmb * 1516, dtype=torch.uint8, device="cuda"),
             torch.zeros((st.mb_h * 16, st.mb_w * 16), dtype=torch.uint8, device="cuda"),
             torch.zeros((2, st.mb_h * 8, st.mb_w * 8), dtype=torch.uint8, device="cuda")) for st in (c, c2)]
    args = ([b[0].data_ptr() for b in bufs], [b[1].data_ptr() for b in bufs], [b[2].data_ptr() for b in bufs], [b[2].shape[1] for b in bufs],
            [b[3][0].data_ptr() for b in bufs], [b[3][1].data_ptr() for b in bufs], [b[3].shape[2] for b in bufs])
    batch = InterBatch([c, c2])
    assert cuda_lib.ironav_debug_withhold(c2.ctx, 40) == 0
    for st in (c, c2):
        assert cuda_lib.ironav_debug_wait_limit(st.ctx, 20000) == 0
    batch.decide(*args)
    with pytest.raises(IronavError) as e:
        batch.sync()
    assert e.value.status == 100
    assert cuda_lib.ironav_debug_withhold(c2.ctx, -1) == 0
    for st in (c, c2):
        assert cuda_lib.ironav_debug_wait_limit(st.ctx, 1 << 22) == 0
    batch.decide(*args)
    batch.sync()
    batch.close()


# ---- the whole P picture: decide, the filter's records, deblocking ------------------------------------

def _py_records(st, codes, states, qp_y, nslices):
    """finish_mb's MbInfo fields the filter reads (enc/frame.rs:2323-2339), restated from the codes."""
    from ironav_b200.inter import DBK_MB_DTYPE

    m = np.zeros(st.nmb, dtype=DBK_MB_DTYPE)
    rows = np.arange(st.nmb) // st.mb_w
    starts = [(st.mb_h * k) // nslices for k in range(nslices)]
    m["slice"] = 1 + np.array([sum(1 for s in starts[1:] if s <= r) for r in rows])
    inter = codes["kind"] == KIND_INTER
    m["inter"] = inter
    m["qp"] = qp_y
    m["t8x8"] = codes["res"]["t8x8"]
    m["nnz"] = codes["res"]["nnz"]
    m["ref_idx"] = -1
    m["ref_id"] = -1
    m["ref_idx"][inter, 0] = states["refs"][inter]
    m["ref_id"][inter, 0] = 1 + states["refs"][inter].astype(np.int32)
    m["mv"][inter, 0] = states["mvs"][inter]
    return m


@pytest.mark.parametrize("kw", [dict(qp=34, nslices=3), dict(new_content=True, qp=30), dict(refs=2, qp=28, nslices=2)])
def test_oracle_picture_pipeline(oracle_lib, kw):
    from ironav_b200.synth import dbk_encoder_slices

    st, fr, ch = decide_case(oracle_lib, **kw)
    states, codes, rec = st.decide_p_picture()
    mbs = st.decide_dbk_records(codes, states)
    want = _py_records(st, codes, states, kw["qp"], kw.get("nslices", 2))
    for f in mbs.dtype.names:
        assert np.array_equal(mbs[f], want[f]), f
    y, cb, cr = st.deblock(*rec, mbs, dbk_encoder_slices(kw.get("nslices", 2)))
    assert not np.array_equal(y, rec[0])  # the filter acted on block edges
    h, w = fr[1].shape
    assert psnr(y[:h, :w], fr[1]) > psnr(rec[0][:h, :w], fr[1]) - 0.5


@pytest.mark.gpu
@pytest.mark.parametrize("kw", [dict(qp=34, nslices=3), dict(new_content=True, qp=30), dict(cfg="1080p", nslices=8, qp=27),
                                dict(bd=10, qp=30, new_content=True)])
def test_gpu_picture_pipeline_on_the_device(oracle_lib, cuda_lib, kw):
    """decide → the filter's records → deblocking, all on device pointers, equals the oracle's picture."""
    import torch

    from ironav_b200.inter import DBK_MB_DTYPE
    from ironav_b200.synth import dbk_encoder_slices

    ns = kw.get("nslices", 2)
    o, _, _ = decide_case(oracle_lib, **kw)
    s_o, c_o, r_o = o.decide_p_picture()
    m_o = o.decide_dbk_records(c_o, s_o)
    want = o.deblock(*r_o, m_o, dbk_encoder_slices(ns))
    c, _, _ = decide_case(cuda_lib, threads=False, **kw)
    assert np.array_equal(c.decide_dbk_records(c_o, s_o), m_o)
    c.set_stream(torch.cuda.current_stream().cuda_stream)
    dt = torch.uint8 if c.bd == 8 else torch.int16
    y = torch.zeros((c.mb_h * 16, c.mb_w * 16), dtype=dt, device="cuda")
    cc = torch.zeros((2, c.mb_h * 8, c.mb_w * 8), dtype=dt, device="cuda")
    ts = torch.zeros(c.nmb * 72, dtype=torch.uint8, device="cuda")
    tc = torch.zeros(c.nmb * 1516, dtype=torch.uint8, device="cuda")
    tm = torch.zeros(c.nmb * DBK_MB_DTYPE.itemsize, dtype=torch.uint8, device="cuda")
    assert c.lib.ironav_decide_p_picture_device(c.ctx, ts.data_ptr(), tc.data_ptr(), y.data_ptr(), y.shape[1], cc[0].data_ptr(),
                                                cc[1].data_ptr(), cc.shape[2]) == 0
    assert c.lib.ironav_decide_dbk_records_device(c.ctx, tc.data_ptr(), ts.data_ptr(), tm.data_ptr()) == 0
    c.deblock_device(y.data_ptr(), y.shape[1], cc[0].data_ptr(), cc[1].data_ptr(), cc.shape[2], tm.data_ptr(), dbk_encoder_slices(ns))
    c.sync()
    view = (lambda t: t.cpu().numpy().view(np.uint16)) if c.bd == 10 else (lambda t: t.cpu().numpy())
    for name, a, b in zip("Y Cb Cr".split(), (view(y), view(cc[0]), view(cc[1])), want):
        assert np.array_equal(a, b), f"{kw}: {name} differs at {np.argwhere(a != b)[:4].tolist()}"
    assert np.array_equal(tm.cpu().numpy().view(DBK_MB_DTYPE), m_o)


@pytest.mark.gpu
def test_gpu_decide_4k(oracle_lib, cuda_lib):
    """3840x2160 (32,400 macroblocks, 16 slice bands as the encoder cuts 4K on a 16-core host), two
    references with sub-8x8 partitions: the largest picture the benchmarks use."""
    kw = dict(cfg="4k", nslices=16, qp=27, refs=2, sub8=True)
    o, _, _ = decide_case(oracle_lib, **kw)
    c, _, _ = decide_case(cuda_lib, threads=False, **kw)
    _same_decisions(c.decide_p_picture(), o.decide_p_picture(), "4K")
