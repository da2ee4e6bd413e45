"""B pictures: the searches of a B macroblock (decide_b, crates/ironav-codec/src/h264/enc/frame.rs:1518-1572;
best_b_parts 1626-1687; spatial direct, direct_mvs 1715-1747), in replay mode.

CPU: the oracle on a panned synthetic sequence (I P B order: the B picture between its list-0 and list-1
pictures finds the pans to both), its internal consistency (the chosen direction is the cheapest, direct
vectors follow the rules of direct_mvs), and the ABI's argument checks. GPU: the sm_100a library against
the oracle, every field of every macroblock."""
from __future__ import annotations

import os

import numpy as np
import pytest

from ironav_b200.inter import MBSTATE_B_DTYPE, MBSTATE_DTYPE, InterStage, IronavError, b_decision_states
from ironav_b200.synth import Sequence


def assert_same(a, b, what):
    if np.array_equal(a, b):
        return
    bad = np.nonzero(a != b)[0]
    i = int(bad[0])
    fields = [f for f in a.dtype.names if not np.array_equal(a[i][f], b[i][f])]
    raise AssertionError(f"{what}: {len(bad)} macroblocks differ; first {i}, fields {fields}: "
                         f"got {a[i][fields[0]]} want {b[i][fields[0]]}")


def b_case(lib, cfg="cif", size=None, qp=28, nslices=2, seed=None, bd=8, fast=False, threads=True):
    """Frames 0 (list 0), 1 (the B picture) and 2 (list 1, coded before it as a P picture from frame 0).
    Returns the stage set up for the B picture, the list-1 picture's decisions and the frames."""
    seq = Sequence.config(cfg, 3, seed=seed, size=size)
    fr = [seq.frame10(t) if bd == 10 else seq.frame(t) for t in range(3)]
    qpp = qp + 6 * (bd - 8)
    st = InterStage(seq.width, seq.height, max_refs=2, nslices=nslices, lib=lib, bd=bd)
    if threads and hasattr(lib, "oracle_set_threads"):
        lib.oracle_set_threads(st.ctx, os.cpu_count() or 1)
    # the P picture (frame 2 from frame 0): its decisions are the list-1 picture's
    st.push_reference(fr[0])
    st.set_source(fr[2])
    st.begin_p_picture(qpp)
    col, _ = st.analyse_auto()
    st.push_reference(fr[2], col=col)   # reference 0 = frame 2 (list 1), reference 1 = frame 0 (list 0)
    st.set_source(fr[1])
    st.begin_b_picture(qpp + 2, ref_l0=1, ref_l1=0, col=col, tb=1, td=2, fast=fast)
    return st, col, seq


def b_replay_twice(st):
    """Results against all-intra neighbours, then against the decisions those results favour."""
    first = st.analyse_b_replay(np.zeros(st.nmb, dtype=MBSTATE_B_DTYPE))
    states = b_decision_states(first)
    return states, st.analyse_b_replay(states)


# ---- CPU: the oracle ------------------------------------------------------------------------------------

def test_oracle_b_finds_both_pans(oracle_lib):
    st, col, seq = b_case(oracle_lib)
    states, res = b_replay_twice(st)
    p1, p2 = np.array(seq.pan(1)), np.array(seq.pan(2))
    l0 = res["mv16"][:, 0].astype(int)
    l1 = res["mv16"][:, 1].astype(int)
    # pan(t) is frame t's offset from frame 0: the vector from frame 1 to frame t is pan(1) - pan(t)
    assert (np.abs(l0 - p1) <= 4).all(axis=1).mean() > 0.7
    assert (np.abs(l1 - (p1 - p2)) <= 4).all(axis=1).mean() > 0.7
    assert set(np.unique(res["dir16"])) <= {1, 2, 3} and (res["dir16"] == 3).any()


def test_oracle_b_choices_are_consistent(oracle_lib):
    st, col, seq = b_case(oracle_lib, qp=24)
    states, res = b_replay_twice(st)
    c0, c1, bi = res["cost16"][:, 0], res["cost16"][:, 1], res["cost_bi"]
    want = np.where(bi < np.minimum(c0, c1), 3, np.where(c0 <= c1, 1, 2))
    assert np.array_equal(res["dir16"], want)
    parts = res["has_parts"] == 1
    assert parts.any() and set(np.unique(res["part"][parts])) <= {1, 2, 3}
    # partitions use direct prediction only in P_8x8-like partitionings (part 3)
    assert not ((res["part"] != 3)[:, None] & (res["bdir"] == 0) & (np.arange(4)[None, :] < 2) & parts[:, None]).any()
    # a direct list that is used has the same vector in every 4x4 block of an 8x8 block
    dm = res["direct_mv"].reshape(-1, 2, 4, 4, 2)
    assert (dm[:, :, 0::2, 0::2] == dm[:, :, 1::2, 1::2]).all()
    assert (res["sad_px"] > 0).all() and (res["satd_px"] > 0).all()


def test_oracle_b_direct_zeroes_still_colocated_blocks(oracle_lib):
    """direct_mvs: in the 8x8 blocks whose co-located block (list-1 picture, reference 0) barely moves, the
    lists whose neighbours use reference 0 get zero vectors."""
    st, col, seq = b_case(oracle_lib)
    still = np.zeros(st.nmb, dtype=MBSTATE_DTYPE)
    still["inter"] = 1
    st.begin_b_picture(30, ref_l0=1, ref_l1=0, col=still, tb=1, td=2)
    states = np.zeros(st.nmb, dtype=MBSTATE_B_DTYPE)
    states["inter"] = 1
    states["mvs"] = 12  # neighbours move by 3 samples in both lists, reference 0
    res = st.analyse_b_replay(states)
    inner = np.arange(st.nmb) % st.mb_w > 0
    assert (res["direct_use"][inner] == 1).all()
    assert (res["direct_mv"][inner] == 0).all()
    st.begin_b_picture(30, ref_l0=1, ref_l1=0, col=None, tb=1, td=2)  # intra list-1 picture: no zeroing
    res = st.analyse_b_replay(states)
    assert (res["direct_mv"][inner] == 12).all()


def test_b_arguments_are_checked(oracle_lib):
    st = InterStage(64, 48, max_refs=2, lib=oracle_lib)
    with pytest.raises(IronavError):
        st.begin_b_picture(30, ref_l0=1, ref_l1=0, col=None, tb=1, td=2)  # no references held
    st.push_reference(np.zeros((48, 64), dtype=np.uint8))
    st.push_reference(np.zeros((48, 64), dtype=np.uint8))
    for bad in (dict(tb=0, td=2), dict(tb=1, td=0), dict(ref_l0=2)):
        kw = dict(ref_l0=1, ref_l1=0, col=None, tb=1, td=2)
        kw.update(bad)
        with pytest.raises(IronavError):
            st.begin_b_picture(30, **kw)


# ---- GPU: the sm_100a library against the oracle ------------------------------------------------------------

def _random_b_states(rng, nmb):
    st = np.zeros(nmb, dtype=MBSTATE_B_DTYPE)
    st["inter"] = rng.random(nmb) < 0.85
    for l in (0, 1):
        used = rng.random((nmb, 4)) < (0.8 if l == 0 else 0.5)
        st["refs"][:, l] = np.where(used & (st["inter"][:, None] == 1), 0, -1)
    mv = np.stack([rng.integers(-300, 300, size=(nmb, 2, 16)), rng.integers(-120, 120, size=(nmb, 2, 16))], axis=-1)
    st["mvs"] = np.where(rng.random((nmb, 1, 1, 1)) < 0.5, mv // 16, mv)
    return st


def _pair(oracle_lib, cuda_lib, **kw):
    o, col, seq = b_case(oracle_lib, **kw)
    c, col_c, _ = b_case(cuda_lib, threads=False, **kw)
    assert np.array_equal(col, col_c)
    return o, c, col


@pytest.mark.gpu
@pytest.mark.parametrize("kw", [dict(), dict(qp=22), dict(cfg="1080p", nslices=8), dict(cfg="1080p", size=(1280, 720), nslices=5, fast=True),
                                dict(bd=10, qp=30)])
def test_gpu_b_matches_oracle(oracle_lib, cuda_lib, kw):
    o, c, col = _pair(oracle_lib, cuda_lib, **kw)
    zero = np.zeros(o.nmb, dtype=MBSTATE_B_DTYPE)
    r0 = o.analyse_b_replay(zero)
    assert_same(c.analyse_b_replay(zero), r0, "B results against intra neighbours")
    states = b_decision_states(r0)
    assert_same(c.analyse_b_replay(states), o.analyse_b_replay(states), "B results against their own decisions")


@pytest.mark.gpu
def test_gpu_b_random_neighbours_and_intra_col(oracle_lib, cuda_lib):
    """Arbitrary two-list neighbour decisions (list-1-only, bi-predicted, intra, large vectors that reach the
    search clamps) and a list-1 picture that was intra coded (no co-located candidate, no direct zeroing)."""
    o, c, col = _pair(oracle_lib, cuda_lib, qp=26)
    rng = np.random.default_rng(7)
    states = _random_b_states(rng, o.nmb)
    assert_same(c.analyse_b_replay(states), o.analyse_b_replay(states), "B results, random neighbours")
    for st in (o, c):
        st.begin_b_picture(33, ref_l0=1, ref_l1=0, col=None, tb=2, td=3)
    assert_same(c.analyse_b_replay(states), o.analyse_b_replay(states), "B results, intra list-1 picture")


@pytest.mark.gpu
def test_gpu_b_device_form(oracle_lib, cuda_lib):
    import torch

    from ironav_b200.inter import BRESULT_DTYPE

    o, c, col = _pair(oracle_lib, cuda_lib)
    states = b_decision_states(o.analyse_b_replay(np.zeros(o.nmb, dtype=MBSTATE_B_DTYPE)))
    want = o.analyse_b_replay(states)
    c.set_stream(torch.cuda.current_stream().cuda_stream)
    tcol = torch.from_numpy(col.view(np.uint8)).cuda()
    c.lib.ironav_begin_b_picture_device(c.ctx, 30, c.lib.ironav_lambda(30), 1, 0, tcol.data_ptr(), 1, 2, 0)
    ts = torch.from_numpy(states.view(np.uint8)).cuda()
    tr = torch.zeros(c.nmb * 200, dtype=torch.uint8, device="cuda")
    assert c.lib.ironav_analyse_b_replay_device(c.ctx, ts.data_ptr(), tr.data_ptr()) == 0
    c.sync()
    assert_same(tr.cpu().numpy().view(BRESULT_DTYPE), want, "B device form")
