"""In-loop mode (the encoder's own macroblock loop drives the stage): the caller reads each
macroblock's result, makes the final decision itself and commits it (FrameCoder::encode / code_mb /
finish_mb, crates/ironav-codec/src/h264/enc/frame.rs:467-478, 715-790, 2281-2339).

CPU tests drive the oracle through the same C ABI; GPU tests compare the CUDA library with it."""
import threading

import numpy as np
import pytest

from ironav_b200.inter import MBRESULT_DTYPE, MBSTATE_DTYPE, InterStage, IronavError, decision_state
from ironav_b200.synth import Sequence


def _stage(lib, nslices=2, size=(352, 288), qp=26):
    seq = Sequence.config("cif", 2, size=size)
    st = InterStage(seq.width, seq.height, nslices=nslices, lib=lib)
    st.push_reference(seq.frame(0))
    st.set_source(seq.frame(1))
    st.begin_p_picture(qp)
    return st


def _policy(lib, qp):
    thr = lib.ironav_skip_threshold(qp)

    def decide(mb, res):
        if mb % 7 == 3:  # an intra decision the stage's own policy would never make
            st = np.zeros(1, dtype=MBSTATE_DTYPE)[0]
            st["refs"][:] = -1
            return st
        return decision_state(res, bool(res["skip_sad"] < thr))

    return decide


def run_raster(st, decide):
    st.inloop_begin(InterStage.INLOOP_RASTER)
    results = np.zeros(st.nmb, dtype=MBRESULT_DTYPE)
    states = np.zeros(st.nmb, dtype=MBSTATE_DTYPE)
    for mb in range(st.nmb):
        results[mb] = st.inloop_result(mb)
        states[mb] = decide(mb, results[mb])
        st.inloop_commit(mb, states[mb])
    st.inloop_end()
    return states, results


def run_bands(st, decide, bands):
    st.inloop_begin(InterStage.INLOOP_BANDS)
    results = np.zeros(st.nmb, dtype=MBRESULT_DTYPE)
    states = np.zeros(st.nmb, dtype=MBSTATE_DTYPE)
    errors = []

    def band(b):
        try:
            for mb in range(bands[b] * st.mb_w, bands[b + 1] * st.mb_w):
                results[mb] = st.inloop_result(mb)
                states[mb] = decide(mb, results[mb])
                st.inloop_commit(mb, states[mb])
        except Exception as e:  # reported after the join
            errors.append(e)

    threads = [threading.Thread(target=band, args=(b,)) for b in range(len(bands) - 1)]
    for t in threads:
        t.start()
    for t in threads:
        t.join()
    st.inloop_end()
    assert not errors, errors
    return states, results


def test_inloop_equals_replay_of_the_committed_decisions(oracle_lib):
    st = _stage(oracle_lib)
    states, results = run_raster(st, _policy(oracle_lib, 26))
    assert (states["inter"] == 0).sum() > 0
    assert np.array_equal(results, st.analyse_replay(states))


def test_inloop_with_the_analysis_policy_equals_auto_mode(oracle_lib):
    st = _stage(oracle_lib, qp=22)
    thr = oracle_lib.ironav_skip_threshold(22)
    states, results = run_raster(st, lambda mb, r: decision_state(r, bool(r["skip_sad"] < thr)))
    auto_states, auto_results = st.analyse_auto()
    assert np.array_equal(states, auto_states)
    inter = (auto_results["flags"] & 1) == 1
    assert np.array_equal(results[inter], auto_results[inter])


@pytest.mark.gpu
@pytest.mark.parametrize("order", ["raster", "bands"])
def test_inloop_gpu_matches_oracle(oracle_lib, cuda_lib, order):
    o, c = _stage(oracle_lib, nslices=3, size=(640, 360)), _stage(cuda_lib, nslices=3, size=(640, 360))
    decide = _policy(cuda_lib, 26)
    bands = [i * c.mb_h // 3 for i in range(4)]
    sc, rc = run_raster(c, decide) if order == "raster" else run_bands(c, decide, bands)
    so, ro = run_raster(o, decide)
    assert np.array_equal(sc, so)
    assert np.array_equal(rc, ro)
    # and the GPU can run the same picture again in the other modes
    assert np.array_equal(c.analyse_replay(sc), ro)


@pytest.mark.gpu
def test_inloop_wait_for_a_commit_that_never_comes_times_out(cuda_lib):
    c = _stage(cuda_lib)
    c.inloop_set_wait(300)
    c.inloop_begin(InterStage.INLOOP_RASTER)
    c.inloop_result(0)  # macroblock 0 has no neighbours to wait for; its decision is never committed
    with pytest.raises(IronavError) as e:
        c.inloop_result(1, timeout_ms=2000)
    assert e.value.status == 100
    with pytest.raises(IronavError) as e:
        c.inloop_end()
    assert e.value.status == 100
    # the context is usable afterwards
    states, results = c.analyse_auto()
    assert results["skip_sad"].sum() > 0


@pytest.mark.gpu
def test_native_band_threads_drive_the_picture(oracle_lib, cuda_lib):
    """The native caller (libironav_inloop_caller.so: one C++ thread per slice band, as the encoder's slice
    threads) under the analysis policy: its decisions equal the oracle's auto mode and its results the
    oracle's replay of them, at 1080p with eight bands."""
    from ironav_b200.inter import default_bands, inloop_caller

    seq = Sequence.config("1080p", 2)
    c = InterStage(1920, 1080, nslices=8, lib=cuda_lib)
    o = InterStage(1920, 1080, nslices=8, lib=oracle_lib)
    for st in (c, o):
        st.push_reference(seq.frame(0))
        st.set_source(seq.frame(1))
        st.begin_p_picture(27)
    bands = np.asarray(default_bands(c.mb_h, 8), dtype=np.int32)
    states = np.zeros(c.nmb, dtype=MBSTATE_DTYPE)
    results = np.zeros(c.nmb, dtype=MBRESULT_DTYPE)
    s = inloop_caller().ironav_inloop_drive_bands(c.ctx, c.mb_w, 8, bands.ctypes.data, cuda_lib.ironav_skip_threshold(27),
                                                  states.ctypes.data, results.ctypes.data)
    assert s == 0
    auto_states, _ = o.analyse_auto()
    assert np.array_equal(states, auto_states)
    assert np.array_equal(results, o.analyse_replay(states))
