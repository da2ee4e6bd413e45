"""Inter residual coding and reconstruction (code_inter, code_inter_residual, code_luma8, code_chroma,
crates/ironav-codec/src/h264/enc/frame.rs:1202-1305, 1856-1915; the transforms and quantisers 46-141,
1025-1046; decimate_score 2369-2440; chroma_mc h264/inter.rs:549-568; idct4_add / idct8_add
h264/idct.rs:8-76).

CPU: the oracle's reconstruction follows the source (PSNR) at low QP, P_Skip macroblocks reconstruct to
their prediction, the coded block pattern agrees with the levels, and the inverse transforms invert the
forward ones within the quantiser's step. GPU: the sm_100a library against the oracle, every level, count
and reconstructed sample."""
from __future__ import annotations

import os

import numpy as np
import pytest

from ironav_b200.inter import INTERDEC_DTYPE, InterStage, IronavError, inter_decisions
from ironav_b200.synth import Sequence


def psnr(a, b, maxv=255):
    mse = float(np.mean((a.astype(np.float64) - b.astype(np.float64)) ** 2))
    return 99.0 if mse == 0 else 10 * np.log10(maxv * maxv / mse)


def p_case(lib, cfg="cif", size=None, qp=22, bd=8, nslices=2, refs=1, threads=True):
    """A P picture (frame 1) from frame 0 (and frame 2 as a second reference when refs == 2): references
    pushed with their chroma (the original frames stand in for reconstructions), decisions by the stage's
    auto mode; returns the stage, the decisions' analysis results and the frames."""
    seq = Sequence.config(cfg, 3, size=size)
    fr = [seq.frame10(t) if bd == 10 else seq.frame(t) for t in range(3)]
    ch = [seq.chroma(t, bd) for t in range(3)]
    st = InterStage(seq.width, seq.height, max_refs=2, nslices=nslices, lib=lib, bd=bd)
    if threads and hasattr(lib, "oracle_set_threads"):
        lib.oracle_set_threads(st.ctx, os.cpu_count() or 1)
    pushed = [2, 0] if refs == 2 else [0]
    for t in pushed:
        st.push_reference(fr[t])
        st.push_reference_chroma(*ch[t])
    st.set_source(fr[1])
    st.set_source_chroma(*ch[1])
    st.begin_p_picture(qp + 6 * (bd - 8), nrefs_active=refs)
    states, res = st.analyse_auto()
    return st, res, fr, ch, seq


def blank_rec(st, bd=8):
    dt = np.uint8 if bd == 8 else np.uint16
    return (np.zeros((st.mb_h * 16, st.mb_w * 16), dt), np.zeros((st.mb_h * 8, st.mb_w * 8), dt),
            np.zeros((st.mb_h * 8, st.mb_w * 8), dt))


@pytest.mark.parametrize("t8", [False, True])
def test_oracle_reconstruction_follows_the_source(oracle_lib, t8):
    st, res, fr, ch, seq = p_case(oracle_lib, qp=22)
    decs = inter_decisions(res, t8=t8)
    decs["mode"] = np.where(decs["mode"] > 0, 2, 0)  # every macroblock coded with its residual (no P_Skip)
    codes, (y, cb, cr) = st.code_inter(22, decs, blank_rec(st))
    h, w = fr[1].shape
    assert psnr(y[:h, :w], fr[1]) > 38
    assert psnr(cb[: h // 2, : w // 2], ch[1][0]) > 38 and psnr(cr[: h // 2, : w // 2], ch[1][1]) > 38
    inter = decs["mode"] == 2
    # the coded block pattern follows the levels
    cbpl = codes["cbp"] & 15
    if t8:
        has = (codes["luma8"] != 0).any(axis=2)
        assert np.array_equal(cbpl[inter], (has[inter] * (1 << np.arange(4))).sum(axis=1))
        assert np.array_equal(codes["t8x8"][inter], (cbpl[inter] != 0).astype(np.uint8))
    else:
        has = (codes["luma"] != 0).any(axis=2).reshape(-1, 2, 2, 2, 2).any(axis=(2, 4)).reshape(-1, 4)
        assert np.array_equal(cbpl[inter], (has[inter] * (1 << np.arange(4))).sum(axis=1))
        assert np.array_equal(codes["nnz"], (codes["luma"] != 0).sum(axis=2))
    assert (codes[decs["mode"] != 2]["cbp"] == 0).all()
    assert (cbpl[inter] != 0).any()


def test_oracle_skip_reconstructs_the_prediction(oracle_lib):
    """P_Skip macroblocks get their prediction; coding them as 16x16 inter at a QP too coarse for any level
    (the residual all quantised away) gives the same samples."""
    st, res, fr, ch, seq = p_case(oracle_lib, qp=22)
    decs = inter_decisions(res)
    decs["mode"] = 1
    decs["part"] = 0
    decs["refs"] = 0
    _, skip = st.code_inter(22, decs, blank_rec(st))
    decs["mode"] = 2
    decs["mvs"][:, 1:] = 0
    c51, coarse = st.code_inter(51, decs, blank_rec(st))
    flat = (c51["cbp"] == 0)
    assert flat.mean() > 0.5
    mb = np.arange(st.nmb)
    for k in mb[flat][:50]:
        x, y = (k % st.mb_w) * 16, (k // st.mb_w) * 16
        assert np.array_equal(skip[0][y:y + 16, x:x + 16], coarse[0][y:y + 16, x:x + 16])


def test_oracle_rejects_bad_decisions(oracle_lib):
    st, res, fr, ch, seq = p_case(oracle_lib)
    decs = inter_decisions(res)
    bad = decs.copy()
    bad["refs"][3] = 1  # one reference held
    with pytest.raises(IronavError):
        st.code_inter(22, bad, blank_rec(st))
    with pytest.raises(IronavError):
        st.code_inter(52, decs, blank_rec(st))


# ---- GPU: the sm_100a library against the oracle ------------------------------------------------------------

def _check_same(got, want, what):
    codes_g, rec_g = got
    codes_w, rec_w = want
    for name, a, b in zip("Y Cb Cr".split(), rec_g, rec_w):
        assert np.array_equal(a, b), f"{what}: {name} differs at {np.argwhere(a != b)[:4].tolist()}"
    if not np.array_equal(codes_g, codes_w):
        bad = np.nonzero(codes_g != codes_w)[0]
        i = int(bad[0])
        fields = [f for f in codes_g.dtype.names if not np.array_equal(codes_g[i][f], codes_w[i][f])]
        raise AssertionError(f"{what}: {len(bad)} macroblocks' codes differ; first {i}, fields {fields}")


def _random_decisions(rng, nmb, nrefs):
    d = np.zeros(nmb, dtype=INTERDEC_DTYPE)
    d["mode"] = rng.choice([0, 1, 2, 2, 2], nmb)
    d["part"] = rng.integers(0, 4, nmb)
    d["sub"] = rng.integers(0, 4, size=(nmb, 4))
    d["refs"] = rng.integers(0, nrefs, size=(nmb, 4))
    d["t8"] = rng.integers(0, 2, nmb)
    mv = np.stack([rng.integers(-200, 200, size=(nmb, 16)), rng.integers(-100, 100, size=(nmb, 16))], axis=-1)
    d["mvs"] = np.where(rng.random((nmb, 1, 1)) < 0.3, mv * 8, mv)  # some far outside the picture
    return d


# ---- the reference's unit tests of the building blocks (enc/frame.rs:2442-2492), on the oracle's --------

MF0, V0 = (13107, 5243, 8066), (10, 16, 13)  # quantisation multipliers and scales at QP % 6 == 0


def _class(p):
    r, c = divmod(p, 4)
    return 0 if r % 2 == 0 and c % 2 == 0 else (1 if r % 2 == 1 and c % 2 == 1 else 2)


def test_forward_and_inverse_transforms_round_trip_at_low_qp(oracle_lib):
    """forward_and_inverse_transforms_round_trip_at_low_qp (enc/frame.rs:2442-2465): fdct4, quant at
    QP 0 with the intra rounding (f = 2^14, 15 bits), scaling and idct4_add give back the residual
    within 1."""
    src = np.array([((i * 37) % 23) * 9 for i in range(16)], np.int32)
    d = (src - 100).astype(np.int32)
    c = np.zeros(16, np.int32)
    oracle_lib.oracle_fdct4(d.ctypes.data, c.ctypes.data)
    co = np.array([oracle_lib.oracle_quant(int(c[p]), MF0[_class(p)], 1 << 14, 15) * V0[_class(p)] for p in range(16)], np.int32)
    out = np.full(16, 100, np.uint16)
    oracle_lib.oracle_idct4_add(co.ctypes.data, out.ctypes.data, 4, 255)
    assert np.abs(out.astype(np.int64) - src).max() <= 1, (out, src)


def test_the_8x8_transform_round_trips_at_low_qp(oracle_lib):
    """the_8x8_transform_round_trips_at_low_qp (enc/frame.rs:2467-2479): quant8 (intra) and idct8_add
    within 1 + QP/3 at QP 0, 1, 5 and 6."""
    src = np.array([((i * 37) % 23) * 9 + (i // 8) * 5 for i in range(64)], np.int32)
    pred = np.full(64, 100, np.int32)
    for qp in (0, 1, 5, 6):
        lv, co = np.zeros(64, np.int32), np.zeros(64, np.int32)
        oracle_lib.oracle_quant8(src.ctypes.data, pred.ctypes.data, qp, 1, lv.ctypes.data, co.ctypes.data)
        out = np.full(64, 100, np.uint16)
        oracle_lib.oracle_idct8_add(co.ctypes.data, out.ctypes.data, 8, 255)
        assert np.abs(out.astype(np.int64) - src).max() <= 1 + qp // 3, (qp, out, src)


def test_decimation_scores_lone_ones_low_and_big_levels_high(oracle_lib):
    """decimation_scores_lone_ones_low_and_big_levels_high (enc/frame.rs:2481-2492)."""
    lv = np.zeros(16, np.int32)

    def score():
        return oracle_lib.oracle_decimate(lv.ctypes.data, 16)

    assert score() == 0
    lv[15] = 1
    assert score() == 0, "a lone level after a long run of zeros"
    lv[15] = 0
    lv[0] = 1
    assert score() == 3
    lv[3] = -2
    assert score() == 9


@pytest.mark.gpu
@pytest.mark.parametrize("kw", [dict(), dict(qp=30), dict(cfg="1080p", nslices=8, qp=27), dict(bd=10, qp=24), dict(refs=2, qp=20)])
@pytest.mark.parametrize("t8", [False, True])
def test_gpu_code_inter_matches_oracle(oracle_lib, cuda_lib, kw, t8):
    o, res, fr, ch, seq = p_case(oracle_lib, **kw)
    c, res_c, _, _, _ = p_case(cuda_lib, threads=False, **kw)
    assert np.array_equal(res["mvs"], res_c["mvs"])
    bd, qp = kw.get("bd", 8), kw.get("qp", 22)
    decs = inter_decisions(res, t8=t8)
    _check_same(c.code_inter(qp, decs, blank_rec(c, bd)), o.code_inter(qp, decs, blank_rec(o, bd)), f"{kw} t8={t8}")


@pytest.mark.gpu
@pytest.mark.parametrize("qp,bd", [(0, 8), (12, 8), (35, 8), (51, 8), (-12, 10), (40, 10)])
def test_gpu_code_inter_random_decisions(oracle_lib, cuda_lib, qp, bd):
    """Every partitioning and sub-partitioning, both references, P_Skip and intra macroblocks, vectors far
    outside the picture, both transforms, across the QP range (the 8x8 dequantisation's two branches)."""
    o, res, fr, ch, seq = p_case(oracle_lib, refs=2, bd=bd)
    c, _, _, _, _ = p_case(cuda_lib, refs=2, bd=bd, threads=False)
    rng = np.random.default_rng(qp + 100)
    decs = _random_decisions(rng, o.nmb, 2)
    rec = blank_rec(o, bd)
    rec = tuple(np.full_like(a, (1 << bd) // 3) for a in rec)  # non-inter macroblocks keep these samples
    _check_same(c.code_inter(qp, decs, rec), o.code_inter(qp, decs, rec), f"random decisions qp {qp}")


@pytest.mark.gpu
def test_gpu_code_inter_rejects_bad_decisions_and_device_form(oracle_lib, cuda_lib):
    import torch

    from ironav_b200.inter import INTERCODE_DTYPE

    o, res, fr, ch, seq = p_case(oracle_lib)
    c, _, _, _, _ = p_case(cuda_lib, threads=False)
    decs = inter_decisions(res, t8=True)
    bad = decs.copy()
    bad["mode"][0] = 2
    bad["refs"][0] = 5
    with pytest.raises(IronavError) as e:
        c.code_inter(22, bad, blank_rec(c))
    assert e.value.status == 2
    decs["mode"][::7] = 0  # left alone: their codes come back zero whatever the buffer held
    want = o.code_inter(22, decs, blank_rec(o))
    c.set_stream(torch.cuda.current_stream().cuda_stream)
    y = torch.zeros((c.mb_h * 16, c.mb_w * 16), dtype=torch.uint8, device="cuda")
    cc = torch.zeros((2, c.mb_h * 8, c.mb_w * 8), dtype=torch.uint8, device="cuda")
    td = torch.from_numpy(decs.view(np.uint8)).cuda()
    tc = torch.full((c.nmb * 1324,), 0x5A, dtype=torch.uint8, device="cuda")
    assert c.lib.ironav_code_inter_picture_device(c.ctx, 22, td.data_ptr(), tc.data_ptr(), y.data_ptr(), y.shape[1], cc[0].data_ptr(),
                                                  cc[1].data_ptr(), cc.shape[2]) == 0
    c.sync()
    got = (tc.cpu().numpy().view(INTERCODE_DTYPE), (y.cpu().numpy(), cc[0].cpu().numpy(), cc[1].cpu().numpy()))
    # records the kernel cannot address word-wise are refused before any launch
    for dd, cd in ((td.data_ptr() + 1, tc.data_ptr()), (td.data_ptr(), tc.data_ptr() + 2)):
        assert c.lib.ironav_code_inter_picture_device(c.ctx, 22, dd, cd, y.data_ptr(), y.shape[1], cc[0].data_ptr(),
                                                      cc[1].data_ptr(), cc.shape[2]) == 3
    _check_same(got, want, "device form")
