"""ironav_analyse_auto_noalloc, the entry point for callers that cannot allocate device memory.

Such callers (a host callback or real-time thread with a fixed memory budget, a custom allocator that
owns all device memory, a plugin host that only hands out its own buffers) cannot create an ironav_ctx,
because creating one allocates its planes, flags and staging buffers. This entry point takes every input
and output as the caller's device pointers and keeps its scratch in a fixed array inside the library.

The test calls it through the C ABI twice in a row, on two consecutive P pictures (the second uses the
first one's decisions as its co-located vectors, so the second call also runs on the scratch the first
one left behind), and checks each call's half-sample planes, decisions and results against the context
entry points' on the same inputs and against the oracle (the CPU restatement of the reference), so its
parity does not rest on the other CUDA path alone. The work is integer, so the tolerance is zero: every
byte must match. A second test makes one wavefront wait run out (a macroblock's decision withheld by a
host-side test hook, with a short poll limit): the call returns IRONAV_TIMEOUT, and the next call, on
the same scratch, again matches the oracle.
This file is collected last (test_zz_*) so that a run stopping at its first failure has already run
every other test.
"""
import numpy as np
import pytest

from ironav_b200.inter import MBRESULT_DTYPE, MBSTATE_DTYPE, InterStage
from ironav_b200.synth import Sequence

pytestmark = pytest.mark.gpu

W, H, NSLICES, QP = 854, 480, 3, 27  # not a whole number of macroblocks wide: the source is padded


def _padded(luma, pw, ph):
    h, w = luma.shape
    return np.pad(luma, ((0, ph - h), (0, pw - w)), mode="edge")


def _context_outputs(lib, frames):
    """Planes, decisions and results of pictures 1 and 2 through a context of `lib` (each picture's
    reference is the one before it, with that picture's decisions as its co-located vectors)."""
    st = InterStage(W, H, nslices=NSLICES, lib=lib)
    want = []
    col = None
    for t in (1, 2):
        st.clear_references()
        st.push_reference(frames[t - 1], col=col)
        st.set_source(frames[t])
        st.begin_p_picture(QP)
        states, res = st.analyse_auto()
        want.append((st.planes(0), states, res))
        col = states
    dims = (st.mb_w, st.mb_h, st.sw, st.sh, st.nmb)
    st.close()
    return want, dims


def _noalloc(lib, frames, t, d_col, d_planes, d_states, d_results):
    import torch

    mb_w, mb_h = (W + 15) // 16, (H + 15) // 16
    pw, ph = mb_w * 16, mb_h * 16
    lam, thr = lib.ironav_lambda(QP), lib.ironav_skip_threshold(QP)
    d_src = torch.from_numpy(_padded(frames[t], pw, ph)).cuda()
    d_ref = torch.from_numpy(frames[t - 1]).cuda()
    status = lib.ironav_analyse_auto_noalloc(
        d_src.data_ptr(), pw, d_ref.data_ptr(), W, W, H, d_col, W, H, NSLICES, QP, lam, thr, 0, 0,
        d_planes.data_ptr(), d_states.data_ptr(), d_results.data_ptr(), torch.cuda.current_stream().cuda_stream)
    torch.cuda.synchronize()
    return status


def test_noalloc_matches_the_context_entry_points_and_the_oracle(cuda_lib, oracle_lib):
    import torch

    seq = Sequence.config("1080p", 3, size=(W, H))
    frames = [seq.frame(t) for t in range(3)]

    # the existing entry points (a context, which allocates its own buffers), and the oracle's
    want, (mb_w, mb_h, sw, sh, nmb) = _context_outputs(cuda_lib, frames)
    oracle, _ = _context_outputs(oracle_lib, frames)

    # the entry point that allocates nothing: every buffer is the caller's
    d_planes = torch.zeros(4 * sw * sh, dtype=torch.uint8, device="cuda")
    d_states = [torch.zeros(nmb * 72, dtype=torch.uint8, device="cuda") for _ in range(2)]
    d_results = torch.zeros(nmb * 104, dtype=torch.uint8, device="cuda")
    d_col = None
    for i, t in enumerate((1, 2)):
        status = _noalloc(cuda_lib, frames, t, d_col, d_planes, d_states[i], d_results)
        assert status == 0, f"call {i + 1}: status {status}"
        got_planes = d_planes.cpu().numpy().reshape(4, sh, sw)
        got_states = d_states[i].cpu().numpy().view(MBSTATE_DTYPE)
        got_res = d_results.cpu().numpy().view(MBRESULT_DTYPE)
        for name, (planes, states, res) in (("the context entry points", want[i]), ("the oracle", oracle[i])):
            assert np.array_equal(got_planes, planes), f"call {i + 1}: half-sample planes differ from {name}"
            assert np.array_equal(got_states, states), f"call {i + 1}: decisions differ from {name}"
            assert np.array_equal(got_res, res), f"call {i + 1}: results differ from {name}"
        d_col = d_states[i].data_ptr()


def test_noalloc_wait_times_out_and_the_next_call_recovers(cuda_lib, oracle_lib):
    """A macroblock whose decision is never published (withheld by the library's host-side test hook)
    makes the waits behind it run out after a short poll limit: the call returns IRONAV_TIMEOUT (100)
    instead of hanging. The next call, with the hook off, runs on the scratch the failed call left
    behind and matches the oracle."""
    import torch

    seq = Sequence.config("1080p", 2, seed=0x1A2B0011, size=(W, H))
    frames = [seq.frame(t) for t in range(2)]
    oracle_st = InterStage(W, H, nslices=NSLICES, lib=oracle_lib)
    oracle_st.push_reference(frames[0])
    oracle_st.set_source(frames[1])
    oracle_st.begin_p_picture(QP)
    o_states, o_res = oracle_st.analyse_auto()
    oracle_st.close()
    nmb = o_states.shape[0]
    sw, sh = ((W + 15) // 16) * 16 + 96, ((H + 15) // 16) * 16 + 96
    d_planes = torch.zeros(4 * sw * sh, dtype=torch.uint8, device="cuda")
    d_states = torch.zeros(nmb * 72, dtype=torch.uint8, device="cuda")
    d_results = torch.zeros(nmb * 104, dtype=torch.uint8, device="cuda")
    assert cuda_lib.ironav_debug_noalloc_wait(5, 20000) == 0
    try:
        status = _noalloc(cuda_lib, frames, 1, None, d_planes, d_states, d_results)
    finally:
        assert cuda_lib.ironav_debug_noalloc_wait(-1, 0) == 0
    assert status == 100, f"a withheld decision gave status {status}, not IRONAV_TIMEOUT"
    status = _noalloc(cuda_lib, frames, 1, None, d_planes, d_states, d_results)
    assert status == 0, f"the call after the timeout: status {status}"
    assert np.array_equal(d_states.cpu().numpy().view(MBSTATE_DTYPE), o_states)
    assert np.array_equal(d_results.cpu().numpy().view(MBRESULT_DTYPE), o_res)


def test_noalloc_rejects_pictures_beyond_its_scratch(cuda_lib):
    import torch

    d = torch.zeros(64, dtype=torch.uint8, device="cuda")
    # 8192 x 4608 is 147456 macroblocks, more than IRONAV_NOALLOC_MAX_MBS (36864)
    status = cuda_lib.ironav_analyse_auto_noalloc(
        d.data_ptr(), 8192, d.data_ptr(), 8192, 8192, 4608, None, 8192, 4608, 1, 27, 6, 100, 0, 0,
        d.data_ptr(), d.data_ptr(), d.data_ptr(), None)
    assert status == 3
