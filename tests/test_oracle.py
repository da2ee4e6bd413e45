"""CPU tests of the oracle (the C restatement in oracle/) against the reference's own known answers.

- predictions_equal_the_decoders_interpolation (crates/ironav-codec/src/h264/enc/subpel.rs:160-194):
  HalfPel::predict equals the decoder's per-sample interpolation over the same grid of positions and
  vectors, 8- and 10-bit, including vectors far outside the picture;
- exp_golomb_codes_read_back (enc/bitw.rs:110-135): the code lengths of its values;
- lambda (enc/frame.rs:164-166) and the P_Skip threshold (enc/frame.rs:730) at the stage's QPs;
- the committed golden fixtures (tests/golden/make_golden.py) of the oracle's stage outputs.
"""
import ctypes
import json
import os

import numpy as np
import pytest

from ironav_b200.inter import MBRESULT_DTYPE, MBSTATE_DTYPE, InterStage
from ironav_b200.synth import Sequence

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def _lcg_luma(pw, ph, bd):
    # the reference test's picture: seed = seed * 1103515245 + 12345 (wrapping u32), (seed >> 16) % 2^bd
    seed = 99
    out = np.empty(pw * ph, dtype=np.uint16)
    for i in range(pw * ph):
        seed = (seed * 1103515245 + 12345) & 0xFFFFFFFF
        out[i] = (seed >> 16) % (1 << bd)
    return out


@pytest.mark.parametrize("bd", [8, 10])
def test_predict_equals_decoder_interpolation(oracle_lib, bd):
    lib = oracle_lib
    pw, ph = 48, 32
    luma = _lcg_luma(pw, ph, bd)
    maxv = (1 << bd) - 1
    hp = lib.oracle_halfpel_new(luma.ctypes.data, pw, ph, bd)
    try:
        a = np.zeros(256, dtype=np.uint16)
        b = np.zeros(256, dtype=np.uint16)
        bad = []
        for (x, y) in [(0, 0), (16, 16), (32, 16)]:
            for my in range(-100, 100):
                for mx in [-97, -40, -3, -2, -1, 0, 1, 2, 3, 5, 6, 7, 30, 97]:
                    lib.oracle_halfpel_predict(hp, x, y, mx, my, 16, 16, a.ctypes.data)
                    lib.oracle_luma_mc_ref(luma.ctypes.data, pw, pw, ph, x, y, mx, my, 16, 16, b.ctypes.data, maxv)
                    if not np.array_equal(a, b):
                        bad.append((x, y, mx, my))
        # vectors far outside the picture, as temporal direct prediction can give
        for (x, y) in [(0, 0), (40, 24), (32, 16)]:
            for my in [-2049, -1203, -300, -1, 2, 299, 1205, 2047]:
                for mx in [-8191, -2001, -401, 3, 398, 1999, 8190]:
                    lib.oracle_halfpel_predict(hp, x, y, mx, my, 8, 8, a.ctypes.data)
                    lib.oracle_luma_mc_ref(luma.ctypes.data, pw, pw, ph, x, y, mx, my, 8, 8, b.ctypes.data, maxv)
                    if not np.array_equal(a[:64], b[:64]):
                        bad.append(("8x8", x, y, mx, my))
        assert not bad, f"{len(bad)} mismatches, first {bad[:5]}"
    finally:
        lib.oracle_halfpel_free(hp)


def test_planes_border_rules(oracle_lib):
    """Rows of h and j outside [2, sh-3) and columns of b outside [2, sw-3) stay 0 (enc/subpel.rs:78,95)."""
    lib = oracle_lib
    pw, ph = 32, 16
    luma = (np.arange(pw * ph, dtype=np.uint16) * 7919 % 251 + 3).astype(np.uint16)
    hp = lib.oracle_halfpel_new(luma.ctypes.data, pw, ph, 8)
    sw, sh = pw + 96, ph + 96
    planes = np.zeros((4, sh, sw), dtype=np.uint16)
    for k in range(4):
        lib.oracle_halfpel_plane(hp, k, planes[k].ctypes.data)
    lib.oracle_halfpel_free(hp)
    g, b, h, j = planes
    assert (b[:, :2] == 0).all() and (b[:, sw - 3:] == 0).all()
    assert (h[:2] == 0).all() and (h[sh - 3:] == 0).all()
    assert (j[:2] == 0).all() and (j[sh - 3:] == 0).all() and (j[:, :2] == 0).all()
    # G repeats the picture's edges into the border
    assert (g[0, :48] == luma[0]).all() and (g[sh - 1, sw - 1] == luma[-1])
    assert np.array_equal(g[48:48 + ph, 48:48 + pw], luma.reshape(ph, pw))


def test_exp_golomb_lengths(oracle_lib):
    with open(os.path.join(GOLDEN, "exp_golomb.json")) as f:
        g = json.load(f)
    for v, n in zip(g["ue_values"], g["ue_bits"]):
        assert oracle_lib.ironav_ue_bits(v) == n, v
    for v, n in zip(g["se_values"], g["se_bits"]):
        assert oracle_lib.ironav_se_bits(v) == n, v
    # the reference test's total: every code plus a 5-bit field
    assert sum(g["ue_bits"]) + sum(g["se_bits"]) + 5 == g["total_bits"]


def test_lambda_and_skip_threshold(oracle_lib):
    # lambda = max(1, round(2^((qp-12)/6))): QP22 -> 3, QP26 -> 5, QP27 -> 6, QP32 -> 10
    assert [oracle_lib.ironav_lambda(q) for q in (0, 12, 22, 26, 27, 32, 51)] == [1, 1, 3, 5, 6, 10, 91]
    for qp in range(0, 52):
        thr = 256.0 * 0.625 * 2.0 ** (qp / 6.0)
        t = oracle_lib.ironav_skip_threshold(qp)
        # sad < t  <=>  sad < thr, for every integer sad
        assert t - 1 < thr <= t


def test_satd4_known_values(oracle_lib):
    ones = np.ones(16, dtype=np.int32)
    assert oracle_lib.oracle_satd4(ones.ctypes.data) == 8
    impulse = np.zeros(16, dtype=np.int32)
    impulse[5] = 10
    assert oracle_lib.oracle_satd4(impulse.ctypes.data) == 80  # 16 coefficients of magnitude 10, halved


def _cif_case(lib, qp=26, frames=(0, 1)):
    seq = Sequence.config("cif", 4)
    st = InterStage(352, 288, max_refs=1, nslices=2, lib=lib)
    st.push_reference(seq.frame(frames[0]))
    st.set_source(seq.frame(frames[1]))
    st.begin_p_picture(qp)
    return st


def test_oracle_recovers_the_pan(oracle_lib):
    """The global pan of the synthetic sequence is what most 16x16 vectors find."""
    seq = Sequence.config("cif", 4)
    st = _cif_case(oracle_lib)
    states, res = st.analyse_auto()
    res2 = st.analyse_replay(states)
    pan = np.array(seq.pan(1))
    mv = res2["mvs"][:, 0].astype(int)
    close = (np.abs(mv - pan) <= 4).all(axis=1)
    assert close.mean() > 0.8, close.mean()


def test_replay_equals_auto_on_its_own_decisions(oracle_lib):
    """Auto mode's macroblocks saw exactly their neighbours' final decisions, so replaying those
    decisions gives the same answers for every macroblock auto mode analysed."""
    st = _cif_case(oracle_lib, qp=22)
    states, res = st.analyse_auto()
    res2 = st.analyse_replay(states)
    inter = (res["flags"] & 1) == 1
    assert inter.any()
    assert np.array_equal(res[inter], res2[inter])
    assert np.array_equal(res["skip_sad"], res2["skip_sad"]) and np.array_equal(res["skip_mv"], res2["skip_mv"])


def test_oracle_matches_golden(oracle_lib):
    """The oracle reproduces the committed fixtures (tests/golden/make_golden.py)."""
    from tests.golden.make_golden import CASES, run_case

    data = np.load(os.path.join(GOLDEN, "oracle_cif.npz"))
    for name, case in CASES.items():
        luma_hash, states, res, rstates, rres = run_case(oracle_lib, **case)
        assert luma_hash == str(data[f"{name}_hash"]), f"{name}: synthetic input changed"
        assert np.array_equal(states, data[f"{name}_states"].view(MBSTATE_DTYPE)), name
        assert np.array_equal(res, data[f"{name}_results"].view(MBRESULT_DTYPE)), name
        assert np.array_equal(rres, data[f"{name}_replay"].view(MBRESULT_DTYPE)), name
