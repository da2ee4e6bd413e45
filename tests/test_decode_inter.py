"""A decoder rebuilds decide mode's reconstruction from its codes, inter macroblocks included — the
property the reference's own encoder tests hold it to (crates/ironav-codec/src/h264/enc/mod.rs:860-967:
`decoder_rebuilds_the_encoders_reference`, `sub8x8_partitions_decode_to_the_encoders_reference`,
`several_references_decode_to_the_encoders_reference`, `ten_bit_pictures_decode_to_the_encoders_reference`),
on those tests' own content (`scene`, mod.rs:745-772), sizes, slice counts, QPs, reference counts and
sample depths, coded as the reference's CAVLC P pictures (its mode 0).

The decoder here is written from ITU-T H.264, independently of the oracle and the kernels:
- motion vectors from the coded syntax: mb_type (partition), sub_mb_type, ref_idx and mvd, with the
  standard's prediction (8.4.1.3: neighbours A, B, C/D by 6.4.11.7, the directional 16x8/8x16 rules,
  the median) and the P_Skip vector (8.4.1.1);
- fractional sample interpolation (8.4.2.2.1 luma six-tap and quarter-sample averages, 8.4.2.2.2 chroma
  eighth-sample bilinear), clamping reference coordinates to the picture;
- the residual (8.5: flat scaling, the 4x4 inverse transform, the chroma DC transform), present where
  coded_block_pattern says;
- intra macroblocks by the 8.3 statement of `tests/test_decide.py`.

Each chain codes pictures 1.. as P pictures, every picture predicting from the reconstructions before it
(no deblocking: a decoder told disable_deblocking_filter_idc = 1 rebuilds exactly these). The first
reference stands in for the reference encoder's IDR picture: the source of picture 0 itself, its edges
repeated to whole macroblocks (this repository codes no intra pictures).
"""
from __future__ import annotations

import numpy as np
import pytest

from ironav_b200.inter import KIND_INTER, InterStage
from tests.test_decide import band_starts, check_intra_decodes, chroma_qp, chroma_residual, dequant4, idct4, psnr

# ---- the reference tests' content ---------------------------------------------------------------------


def scene(w: int, h: int, t: int):
    """Moving content (enc/mod.rs:745-772): a gradient, two squares sliding at different speeds and a
    little noise from a 32-bit LCG; chroma ramps. Returns (y, u, v) as uint8."""
    seed = (7 + t * 1000) & 0xFFFFFFFF
    y = np.zeros((h, w), np.uint8)
    for r in range(h):
        for c in range(w):
            seed = (seed * 1103515245 + 12345) & 0xFFFFFFFF
            noise = ((seed >> 16) % 9) - 4
            v = c * 160 // w + r * 60 // h + 20
            if (c + 3 * t) % w < w // 4 and h // 5 < r < h // 2:
                v = 220 - ((c + r) % 7) * 10
            q = (c + w - (2 * t) % w) % w
            if w // 2 < q < w // 2 + w // 6 and r > h // 2 + 4:
                v = 30 + (r * 5) % 40
            y[r, c] = min(max(v + noise, 0), 255)
    cw, ch = w // 2, h // 2
    i = np.arange(cw * ch)
    u = ((100 + (i % cw) * 50 // cw + t) & 0xFF).astype(np.uint8).reshape(ch, cw)
    v = ((150 - (i // cw) * 40 // ch) & 0xFF).astype(np.uint8).reshape(ch, cw)
    return y, u, v


def scene10(w: int, h: int, t: int):
    """`scene` at 10 bits (enc/mod.rs:906-911): samples scaled up, the low two bits changing per picture."""
    return tuple(((p.astype(np.uint16) << 2) | (t & 3)).astype(np.uint16) for p in scene(w, h, t))


def pad_to(a: np.ndarray, h: int, w: int) -> np.ndarray:
    return np.pad(a, ((0, h - a.shape[0]), (0, w - a.shape[1])), mode="edge")


# ---- motion vectors from the syntax (8.4.1) -------------------------------------------------------------

# sub-macroblock partitions (x, y, w, h in 4x4 blocks inside the 8x8 block) and SubMbPartWidth, per
# sub_mb_type: P_L0_8x8, P_L0_8x4, P_L0_4x8, P_L0_4x4 (Table 7-17)
SUB_RECTS = {0: [(0, 0, 2, 2)], 1: [(0, 0, 2, 1), (0, 1, 2, 1)], 2: [(0, 0, 1, 2), (1, 0, 1, 2)],
             3: [(0, 0, 1, 1), (1, 0, 1, 1), (0, 1, 1, 1), (1, 1, 1, 1)]}
SUB_WIDTH = {0: 8, 1: 8, 2: 4, 3: 4}


def partitions(part: int, sub):
    """The (sub-)partitions of a P macroblock in decoding order: (rect in 4x4 blocks, mbPartIdx,
    predPartWidth in samples) (Table 7-13; predPartWidth as 8.4.1.3 defines it)."""
    if part == 0:
        return [((0, 0, 4, 4), 0, 16)]
    if part == 1:
        return [((0, 0, 4, 2), 0, 16), ((0, 2, 4, 2), 1, 16)]
    if part == 2:
        return [((0, 0, 2, 4), 0, 8), ((2, 0, 2, 4), 1, 8)]
    out = []
    for k in range(4):
        s = int(sub[k])
        for x, y, w, h in SUB_RECTS[s]:
            out.append((((k & 1) * 2 + x, (k >> 1) * 2 + y, w, h), k, SUB_WIDTH[s]))
    return out


class MotionField:
    """list 0's reference index and vector of every decoded 4x4 luma block (intra: -1 and zero)."""

    def __init__(self, mb_w: int, mb_h: int, band_start):
        self.mb_w, self.band_start = mb_w, band_start
        self.ref = np.full((mb_h * 4, mb_w * 4), -1, np.int64)
        self.mv = np.zeros((mb_h * 4, mb_w * 4, 2), np.int64)
        self.done = np.zeros((mb_h * 4, mb_w * 4), bool)

    def neighbour(self, mbx: int, mby: int, xn: int, yn: int):
        """The block covering luma location (xn, yn) relative to macroblock (mbx, mby) (6.4.12), or None
        when not available: outside the picture or the slice, or not decoded yet (6.4.11.7)."""
        if yn > 15 or (xn > 15 and yn >= 0):
            return None
        dx = -1 if xn < 0 else (0 if xn <= 15 else 1)
        dy = -1 if yn < 0 else 0
        nx, ny = mbx + dx, mby + dy
        if nx < 0 or nx >= self.mb_w or ny < self.band_start[mby]:
            return None
        bx, by = nx * 4 + ((xn % 16) >> 2), ny * 4 + ((yn % 16) >> 2)
        if not self.done[by, bx]:
            return None
        return int(self.ref[by, bx]), (int(self.mv[by, bx, 0]), int(self.mv[by, bx, 1]))

    def paint(self, mbx, mby, rect, ref, mv):
        x, y, w, h = rect
        sl = (slice(mby * 4 + y, mby * 4 + y + h), slice(mbx * 4 + x, mbx * 4 + x + w))
        self.ref[sl] = ref
        self.mv[sl] = mv
        self.done[sl] = True

    def abc(self, mbx, mby, x, y, pw):
        a = self.neighbour(mbx, mby, x - 1, y)
        b = self.neighbour(mbx, mby, x, y - 1)
        c = self.neighbour(mbx, mby, x + pw, y - 1)
        if c is None:  # C not available: D in its place (8.4.1.3.2)
            c = self.neighbour(mbx, mby, x - 1, y - 1)
        return a, b, c

    def mvp(self, mbx, mby, x, y, pw, ref, part=0, idx=0):
        """mvpLX of a (sub-)partition at luma (x, y) of width pw with reference index ref (8.4.1.3)."""
        a, b, c = self.abc(mbx, mby, x, y, pw)
        rv = lambda n: (-1, (0, 0)) if n is None else n  # noqa: E731
        (ra, ma), (rb, mb_), (rc, mc) = rv(a), rv(b), rv(c)
        if part == 1 and idx == 0 and rb == ref:
            return mb_
        if part == 1 and idx == 1 and ra == ref:
            return ma
        if part == 2 and idx == 0 and ra == ref:
            return ma
        if part == 2 and idx == 1 and rc == ref:
            return mc
        # 8.4.1.3.1: B and C both unavailable, A available: A's data for all three
        if b is None and c is None and a is not None:
            (rb, mb_), (rc, mc) = (ra, ma), (ra, ma)
        same = [n for n, r in (("a", ra), ("b", rb), ("c", rc)) if r == ref]
        if len(same) == 1:
            return {"a": ma, "b": mb_, "c": mc}[same[0]]
        return (sorted((ma[0], mb_[0], mc[0]))[1], sorted((ma[1], mb_[1], mc[1]))[1])

    def skip_mv(self, mbx, mby):
        """The P_Skip vector (8.4.1.1)."""
        a = self.neighbour(mbx, mby, -1, 0)
        b = self.neighbour(mbx, mby, 0, -1)
        if a is None or b is None or a == (0, (0, 0)) or b == (0, (0, 0)):
            return (0, 0)
        return self.mvp(mbx, mby, 0, 0, 16, 0)


# ---- fractional sample interpolation (8.4.2.2) --------------------------------------------------------

TAPS = (1, -5, 20, 20, -5, 1)


def luma_pred(refp: np.ndarray, x0: int, y0: int, w: int, h: int, mv, maxv: int) -> np.ndarray:
    """An h x w luma prediction at (x0, y0) displaced by quarter-sample vector mv (8.4.2.2.1)."""
    H, W = refp.shape
    xi, yi, fx, fy = x0 + (mv[0] >> 2), y0 + (mv[1] >> 2), mv[0] & 3, mv[1] & 3
    rows = np.clip(np.arange(yi - 2, yi + h + 4), 0, H - 1)
    cols = np.clip(np.arange(xi - 2, xi + w + 4), 0, W - 1)
    g = refp[np.ix_(rows, cols)].astype(np.int64)  # g[r + 2, c + 2]: the integer sample at (xi + c, yi + r)
    b1 = sum(t * g[:, k:k + w + 1] for k, t in enumerate(TAPS))  # b1[r + 2, c]: between (c, r) and (c + 1, r)
    h1 = sum(t * g[k:k + h + 1, :] for k, t in enumerate(TAPS))  # h1[r, c + 2]: between (c, r) and (c, r + 1)
    j1 = sum(t * b1[k:k + h + 1, :] for k, t in enumerate(TAPS))  # j1[r, c]: the centre of the four
    clip = lambda v: np.clip(v, 0, maxv)  # noqa: E731
    G = g[2:h + 3, 2:w + 3]
    b = clip((b1[2:h + 3, :] + 16) >> 5)
    hh = clip((h1[:, 2:w + 3] + 16) >> 5)
    j = clip((j1 + 512) >> 10)
    G0, Hr, M = G[:h, :w], G[:h, 1:], G[1:, :w]
    b0, s = b[:h, :w], b[1:, :w]
    h0, m = hh[:h, :w], hh[:h, 1:]
    j0 = j[:h, :w]
    avg = lambda p, q: (p + q + 1) >> 1  # noqa: E731
    table = {(0, 0): G0, (0, 1): avg(G0, h0), (0, 2): h0, (0, 3): avg(M, h0),
             (1, 0): avg(G0, b0), (1, 1): avg(b0, h0), (1, 2): avg(h0, j0), (1, 3): avg(h0, s),
             (2, 0): b0, (2, 1): avg(b0, j0), (2, 2): j0, (2, 3): avg(j0, s),
             (3, 0): avg(Hr, b0), (3, 1): avg(b0, m), (3, 2): avg(j0, m), (3, 3): avg(m, s)}
    return table[(fx, fy)]


def chroma_pred(refc: np.ndarray, x0: int, y0: int, w: int, h: int, mv) -> np.ndarray:
    """An h x w 4:2:0 chroma prediction at chroma (x0, y0) for luma vector mv (8.4.1.4: the same vector,
    eighth-sample units; 8.4.2.2.2)."""
    H, W = refc.shape
    xi, yi, fx, fy = x0 + (mv[0] >> 3), y0 + (mv[1] >> 3), mv[0] & 7, mv[1] & 7
    p = refc[np.ix_(np.clip(np.arange(yi, yi + h + 1), 0, H - 1), np.clip(np.arange(xi, xi + w + 1), 0, W - 1))].astype(np.int64)
    return ((8 - fx) * (8 - fy) * p[:h, :w] + fx * (8 - fy) * p[:h, 1:] + (8 - fx) * fy * p[1:, :w] + fx * fy * p[1:, 1:] + 32) >> 6


# ---- one picture --------------------------------------------------------------------------------------

def check_picture_decodes(st: InterStage, codes, rec, refs, qp_y: int, nslices: int, nact: int):
    """Decodes every macroblock of one coded P picture and compares it with the reconstruction. refs:
    the reference pictures (y, cb, cr) the decoder holds, index 0 the newest. Returns counts of what was
    checked: P_Skip, inter by partitioning, sub-partitioned 8x8 blocks, reference indices above 0."""
    bd = st.bd
    maxv = (1 << bd) - 1
    qp = qp_y + 6 * (bd - 8)
    qpc = chroma_qp(qp_y, bd) + 6 * (bd - 8)
    bs = band_starts(st, nslices)
    check_intra_decodes(st, codes, rec, qp_y, bs)
    F = MotionField(st.mb_w, st.mb_h, bs)
    y_rec, cb_rec, cr_rec = (a.astype(np.int64) for a in rec)
    seen = {"skip": 0, "parts": [0, 0, 0, 0], "sub": 0, "ref_above_0": 0}
    for mb in range(st.nmb):
        c = codes[mb]
        mbx, mby = mb % st.mb_w, mb // st.mb_w
        if c["kind"] != KIND_INTER:
            F.paint(mbx, mby, (0, 0, 4, 4), -1, (0, 0))
            continue
        x0, y0 = mbx * 16, mby * 16
        # the vectors, from the syntax
        if c["skip"]:
            seen["skip"] += 1
            mv = F.skip_mv(mbx, mby)
            assert tuple(c["mvs"][0]) == mv, f"mb {mb}: P_Skip vector {tuple(c['mvs'][0])}, the standard's {mv}"
            blocks = [((0, 0, 4, 4), 0, mv)]
            F.paint(mbx, mby, (0, 0, 4, 4), 0, mv)
        else:
            part = int(c["part"])
            seen["parts"][part] += 1
            if part == 3:
                seen["sub"] += int(sum(int(s) != 0 for s in c["sub"]))
            blocks = []
            for k, (rect, idx, pw) in enumerate(partitions(part, c["sub"])):
                ref = int(c["refs"][idx])
                assert 0 <= ref < nact, f"mb {mb}: ref_idx {ref} of {nact}"
                seen["ref_above_0"] += ref > 0
                p = F.mvp(mbx, mby, rect[0] * 4, rect[1] * 4, pw, ref, part if part in (1, 2) else 0, idx)
                mv = (p[0] + int(c["mvds"][k][0]), p[1] + int(c["mvds"][k][1]))
                assert tuple(int(v) for v in c["mvs"][k]) == mv, f"mb {mb} part {part} #{k}: mv {tuple(c['mvs'][k])}, mvp {p} + mvd {tuple(c['mvds'][k])}"
                F.paint(mbx, mby, rect, ref, mv)
                blocks.append((rect, ref, mv))
        # the prediction, then the residual
        pred = np.zeros((16, 16), np.int64)
        cpred = np.zeros((2, 8, 8), np.int64)
        for (x, y, w, h), ref, mv in blocks:
            ry, rcb, rcr = refs[ref]
            pred[y * 4:y * 4 + h * 4, x * 4:x * 4 + w * 4] = luma_pred(ry, x0 + x * 4, y0 + y * 4, w * 4, h * 4, mv, maxv)
            for comp, rc in enumerate((rcb, rcr)):
                cpred[comp, y * 2:y * 2 + h * 2, x * 2:x * 2 + w * 2] = chroma_pred(rc, mbx * 8 + x * 2, mby * 8 + y * 2, w * 2, h * 2, mv)
        cbp = int(c["res"]["cbp"])
        if c["skip"]:
            assert cbp == 0
        res = np.zeros((16, 16), np.int64)
        for blk in range(16):
            bx, by = blk % 4, blk // 4
            if cbp >> ((by >> 1) * 2 + (bx >> 1)) & 1:
                res[by * 4:by * 4 + 4, bx * 4:bx * 4 + 4] = idct4(dequant4(c["res"]["luma"][blk], qp))
            else:  # the stream carries no levels for an 8x8 block outside the pattern
                assert not c["res"]["luma"][blk].any(), f"mb {mb}: levels in luma block {blk} outside cbp {cbp:#x}"
        if cbp >> 4 == 0:
            assert not c["res"]["cdc"].any() and not c["res"]["cac"].any(), f"mb {mb}: chroma levels outside cbp {cbp:#x}"
        elif cbp >> 4 == 1:
            assert not c["res"]["cac"].any(), f"mb {mb}: chroma AC levels outside cbp {cbp:#x}"
        want = np.clip(pred + res, 0, maxv)
        got = y_rec[y0:y0 + 16, x0:x0 + 16]
        assert np.array_equal(got, want), f"mb {mb} (skip {c['skip']}, part {c['part']}, cbp {cbp:#x}): luma differs at {np.argwhere(got != want)[:4].tolist()}"
        for comp, plane in enumerate((cb_rec, cr_rec)):
            want = np.clip(cpred[comp] + chroma_residual(c["res"], comp, qpc), 0, maxv)
            got = plane[mby * 8:mby * 8 + 8, mbx * 8:mbx * 8 + 8]
            assert np.array_equal(got, want), f"mb {mb} chroma {comp} (cbp {cbp:#x}) differs"
    return seen


# ---- chains of pictures --------------------------------------------------------------------------------

def code_chain(lib, w, h, frames, qp, nslices, refs=1, sub8=False, fast=False, bd=8, content=None, check=True):
    """Codes pictures 1..frames-1 of `scene` as P pictures, each from the reconstructions before it (up to
    `refs` of them), checking every picture with the decoder. Returns per picture (states, codes, rec)
    and the totals of what the checks saw."""
    content = content or (scene10 if bd == 10 else scene)
    st = InterStage(w, h, max_refs=refs, nslices=nslices, lib=lib, bd=bd)
    H, W = st.mb_h * 16, st.mb_w * 16
    y0, u0, v0 = content(w, h, 0)
    first = (pad_to(y0, H, W), pad_to(u0, H // 2, W // 2), pad_to(v0, H // 2, W // 2))
    held = [first]  # the decoder's reference list, newest first
    st.push_reference(first[0])
    st.push_reference_chroma(first[1], first[2])
    out = []
    totals = {"skip": 0, "parts": [0, 0, 0, 0], "sub": 0, "ref_above_0": 0}
    maxv = (1 << bd) - 1
    for t in range(1, frames):
        ys, us, vs = content(w, h, t)
        st.set_source(ys)
        st.set_source_chroma(us, vs)
        nact = min(len(held), refs)
        st.begin_p_picture(qp + 6 * (bd - 8), nrefs_active=nact, fast=fast, sub8=sub8)
        states, codes, rec = st.decide_p_picture()
        if check:
            seen = check_picture_decodes(st, codes, rec, held, qp, nslices, nact)
            totals["skip"] += seen["skip"]
            totals["sub"] += seen["sub"]
            totals["ref_above_0"] += seen["ref_above_0"]
            totals["parts"] = [a + b for a, b in zip(totals["parts"], seen["parts"])]
            # the reference tests' quality floors: 36 dB at QP 20 (8 bits); 48/36/28 dB by QP (10 bits)
            floor = {True: 48.0 if qp <= 10 else (36.0 if qp <= 28 else 28.0), False: 36.0 if qp == 20 else None}[bd == 10]
            if floor is not None:
                assert psnr(rec[0][:h, :w], ys, maxv) > floor, f"{w}x{h} qp {qp} picture {t}: PSNR {psnr(rec[0][:h, :w], ys, maxv):.1f}"
        out.append((states, codes, rec))
        st.push_reference(rec[0], states)
        st.push_reference_chroma(rec[1], rec[2])
        held = [rec] + held[:refs - 1]
    return out, totals


def same_chain(got, want, what):
    for t, ((sa, ca, ra), (sb, cb, rb)) in enumerate(zip(got, want)):
        assert ca.tobytes() == cb.tobytes(), f"{what} picture {t + 1}: codes differ at {np.nonzero(ca != cb)[0][:8].tolist()}"
        assert sa.tobytes() == sb.tobytes(), f"{what} picture {t + 1}: states differ"
        for k in range(3):
            assert np.array_equal(ra[k], rb[k]), f"{what} picture {t + 1}: reconstruction plane {k} differs"


# sizes and slice counts of decoder_rebuilds_the_encoders_reference (mod.rs:861)
SIZES = [(64, 48, 1), (200, 120, 3), (16, 16, 1), (34, 18, 2), (96, 80, 5)]


@pytest.mark.parametrize("bd", [8, 10])
def test_luma_interpolation_equals_the_decoders(oracle_lib, bd):
    """luma_pred above equals the oracle's statement of the reference decoder's luma_mc_ref
    (h264/inter.rs:466-546, itself pinned against the encoder's planes by the reference's known-answer
    test): all 16 phases, every partition size, inside the picture, across its edges and far outside.
    The encoder's refinement rarely lands on the diagonal quarter positions, so the chains alone would
    not cover them."""
    pw, ph = 48, 32
    maxv = (1 << bd) - 1
    luma = np.random.default_rng(11 + bd).integers(0, maxv + 1, size=(ph, pw)).astype(np.uint16)
    out = np.zeros(256, np.uint16)
    bad = []
    vecs = [(mx, my) for mx in range(-9, 10) for my in range(-9, 10)] + [(-803, 7), (611, -402), (5, 259), (-2, -331)]
    for x, y, w, h in [(0, 0, 16, 16), (16, 16, 16, 16), (32, 0, 16, 8), (0, 16, 8, 16), (40, 24, 8, 8), (44, 28, 4, 4), (4, 8, 8, 4), (20, 12, 4, 8)]:
        for mx, my in vecs:
            oracle_lib.oracle_luma_mc_ref(luma.ctypes.data, pw, pw, ph, x, y, mx, my, w, h, out.ctypes.data, maxv)
            if not np.array_equal(luma_pred(luma, x, y, w, h, (mx, my), maxv), out[:w * h].reshape(h, w)):
                bad.append((x, y, w, h, mx, my))
    assert not bad, f"{len(bad)} mismatches, first {bad[:5]}"


@pytest.mark.parametrize("qp", [0, 4, 20, 30, 45, 51])
def test_oracle_chain_decodes(oracle_lib, qp):
    """decoder_rebuilds_the_encoders_reference (mod.rs:860-875) on the oracle: six pictures of each size."""
    for w, h, ns in SIZES:
        _, seen = code_chain(oracle_lib, w, h, 6, qp, ns)
        assert sum(seen["parts"]) + seen["skip"] > 0


def test_oracle_sub8x8_and_references_decode(oracle_lib):
    """sub8x8_partitions_decode_to_the_encoders_reference and several_references_decode_to_the_encoders_
    reference (mod.rs:876-912) on the oracle: with three references and sub-8x8 partitions on, the
    pictures decode, sub-partitions are coded at QP 4 and 20, and references other than the newest are
    used."""
    for w, h, ns in [(64, 48, 1), (200, 120, 3)]:
        for qp in (4, 20):
            _, seen = code_chain(oracle_lib, w, h, 8, qp, ns, refs=3, sub8=True)
            assert seen["sub"] > 0, f"{w}x{h} qp {qp}: no sub-partitions were coded"
        used = False
        for qp in (4, 26, 40):
            _, seen = code_chain(oracle_lib, w, h, 8, qp, ns, refs=3)
            used = used or seen["ref_above_0"] > 0
        assert used, f"{w}x{h}: 3 references are never used"


@pytest.mark.parametrize("qp", [4, 20, 36])
def test_oracle_ten_bit_chain_decodes(oracle_lib, qp):
    """ten_bit_pictures_decode_to_the_encoders_reference (mod.rs:914-967), CAVLC, on the oracle."""
    for w, h, ns in [(64, 48, 1), (200, 120, 3)]:
        code_chain(oracle_lib, w, h, 6, qp, ns, bd=10)


def test_oracle_still_picture_skips_and_a_change_is_coded(oracle_lib):
    """realtime_skips_a_still_picture_and_codes_a_change (mod.rs:1280-1300): realtime coding (fast mode,
    one reference, slices of two macroblock rows) of a still 176x144 picture at QP 26 skips every
    macroblock; a bright 16x16 block at the top left is coded, and little else."""
    w, h = 176, 144
    still = scene(w, h, 0)

    def content(w_, h_, t):
        if t < 5:
            return still
        y = still[0].copy()
        y[:16, :16] = 250
        return y, still[1], still[2]

    out, _ = code_chain(oracle_lib, w, h, 6, 26, 4, fast=True, content=content)
    for t in range(4):
        assert out[t][1]["skip"].all(), f"picture {t + 1}: a still picture is all P_Skip"
    codes = out[4][1]
    coded = np.nonzero(codes["skip"] == 0)[0]
    assert 0 in coded and len(coded) <= 4, coded.tolist()
    assert abs(int(out[4][2][0][:16, :16].astype(np.int64).mean()) - 250) <= 2


# ---- the sm_100a library: the same chains, bit-exact with the oracle and decoding ---------------------

@pytest.mark.gpu
@pytest.mark.parametrize("qp", [0, 4, 20, 30, 45, 51])
def test_gpu_chain_decodes_and_matches_oracle(oracle_lib, cuda_lib, qp):
    for w, h, ns in SIZES:
        got, _ = code_chain(cuda_lib, w, h, 6, qp, ns)
        want, _ = code_chain(oracle_lib, w, h, 6, qp, ns, check=False)
        same_chain(got, want, f"{w}x{h} qp {qp}")


@pytest.mark.gpu
@pytest.mark.parametrize("kw", [dict(refs=3, sub8=True, qp=4), dict(refs=3, sub8=True, qp=20), dict(refs=3, qp=26),
                                dict(bd=10, qp=4), dict(bd=10, qp=36), dict(refs=2, bd=10, sub8=True, qp=20)])
def test_gpu_reference_settings_chain(oracle_lib, cuda_lib, kw):
    """The sub-8x8, several-reference and 10-bit chains on the library: each picture decodes, and the
    codes, states and reconstructions equal the oracle's."""
    kw = dict(kw)
    qp = kw.pop("qp")
    for w, h, ns in [(64, 48, 1), (200, 120, 3)]:
        got, _ = code_chain(cuda_lib, w, h, 8, qp, ns, **kw)
        want, _ = code_chain(oracle_lib, w, h, 8, qp, ns, check=False, **kw)
        same_chain(got, want, f"{w}x{h} {kw} qp {qp}")
