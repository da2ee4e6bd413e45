"""The batched form (ironav_batch_*): several streams of different sizes stepped together, one launch
per stage, must give every stream exactly the results of its own single-stream auto mode."""
import numpy as np
import pytest

from ironav_b200.inter import MBRESULT_DTYPE, MBSTATE_DTYPE, InterBatch, InterStage
from ironav_b200.synth import Sequence

pytestmark = pytest.mark.gpu

# (width, height, slice bands): the batched configuration's resolutions and their pinned band counts
STREAMS = [(640, 360, 2), (854, 480, 3), (352, 288, 2), (1280, 720, 5), (1920, 1080, 8), (176, 144, 1)]


def _frames(i, w, h, n=3, bd=8):
    seq = Sequence.config("1080p", n, seed=0x1A2B0300 + i, size=(w, h))
    return [seq.frame10(t) if bd == 10 else seq.frame(t) for t in range(n)]


@pytest.mark.parametrize("bd", [8, 10])
def test_batch_equals_single_stream_auto_mode(cuda_lib, bd):
    import torch

    qpp = 27 + 6 * (bd - 8)
    stream = torch.cuda.Stream()
    frames = [_frames(i, w, h, bd=bd) for i, (w, h, _) in enumerate(STREAMS)]
    # each stream alone (host-buffer calls)
    want = []
    for (w, h, ns), f in zip(STREAMS, frames):
        st = InterStage(w, h, nslices=ns, lib=cuda_lib, bd=bd)
        per = []
        col = None
        for t in (1, 2):
            st.clear_references()
            st.push_reference(f[t - 1], col=col)
            st.set_source(f[t])
            st.begin_p_picture(qpp)
            states, res = st.analyse_auto()
            per.append((states, res))
            col = states
        st.close()
        want.append(per)
    # all streams together: each context primed with a reference so its picture parameters are valid
    stages = []
    dev = [[torch.from_numpy(x.view(np.int16) if bd == 10 else x).cuda() for x in f] for f in frames]
    for (w, h, ns), f in zip(STREAMS, dev):
        st = InterStage(w, h, nslices=ns, lib=cuda_lib, bd=bd)
        st.set_stream(stream.cuda_stream)
        st.push_reference_device(f[0].data_ptr(), w, w, h, None)
        st.begin_p_picture(qpp)
        stages.append(st)
    n = len(stages)
    d_states = [[torch.zeros(s.nmb * 72, dtype=torch.uint8, device="cuda") for _ in range(2)] for s in stages]
    d_res = [[torch.zeros(s.nmb * 104, dtype=torch.uint8, device="cuda") for _ in range(2)] for s in stages]
    torch.cuda.synchronize()
    batch = InterBatch(stages)
    for k, t in enumerate((1, 2)):
        col = [None] * n if k == 0 else [d_states[i][0].data_ptr() for i in range(n)]
        batch.step([f[t].data_ptr() for f in dev], [f[t - 1].data_ptr() for f in dev], col,
                   [d_states[i][k].data_ptr() for i in range(n)], [d_res[i][k].data_ptr() for i in range(n)])
        batch.sync()
        for i in range(n):
            got_s = d_states[i][k].cpu().numpy().view(MBSTATE_DTYPE)
            got_r = d_res[i][k].cpu().numpy().view(MBRESULT_DTYPE)
            assert np.array_equal(got_s, want[i][k][0]), f"stream {i} step {k}: decisions"
            assert np.array_equal(got_r, want[i][k][1]), f"stream {i} step {k}: results"
    # the batched planes kernel built each stream's newest reference as a single stream builds it
    for i, ((w, h, ns), f) in enumerate(zip(STREAMS, frames)):
        one = InterStage(w, h, nslices=ns, lib=cuda_lib, bd=bd)
        one.push_reference(f[1])
        assert np.array_equal(stages[i].planes(0), one.planes(0)), f"stream {i}: planes"
        one.close()

    # a frame step captured in a CUDA graph replays to the same results
    for i in range(n):
        d_res[i][1].zero_()
    torch.cuda.synchronize()
    g = torch.cuda.CUDAGraph()
    with torch.cuda.graph(g, stream=stream):
        batch.step([f[2].data_ptr() for f in dev], [f[1].data_ptr() for f in dev], [d_states[i][0].data_ptr() for i in range(n)],
                   [d_states[i][1].data_ptr() for i in range(n)], [d_res[i][1].data_ptr() for i in range(n)])
    g.replay()
    torch.cuda.synchronize()
    batch.sync()
    for i in range(n):
        assert np.array_equal(d_res[i][1].cpu().numpy().view(MBRESULT_DTYPE), want[i][1][1]), f"stream {i}: graph replay"
    del g
    batch.close()


def test_config3_64_streams_four_steps(cuda_lib, oracle_lib):
    """The batched configuration itself: its 64 streams (seeded resolutions from {640x360, 854x480, 1280x720,
    1920x1080}, QP 27, one reference, the pinned slice bands) stepped together for four frame steps, each step
    one batch step over all streams; every stream's decisions and results at every step equal its own
    single-stream auto mode, and the first streams' equal the oracle's."""
    import torch

    from ironav_b200.synth import batch_streams

    streams = batch_streams(64)
    steps = 4
    stream = torch.cuda.Stream()
    stages, dev, want = [], [], []
    for i, (w, h, ns, seed) in enumerate(streams):
        seq = Sequence.config("1080p", steps + 1, seed=seed, size=(w, h))
        f = [seq.frame(t) for t in range(steps + 1)]
        one = InterStage(w, h, nslices=ns, lib=cuda_lib)
        per, col = [], None
        for t in range(1, steps + 1):
            one.clear_references()
            one.push_reference(f[t - 1], col=col)
            one.set_source(f[t])
            one.begin_p_picture(27)
            s, r = one.analyse_auto()
            per.append((s, r))
            col = s
        one.close()
        if i < 2:  # the single-stream path itself against the oracle on the first streams
            o = InterStage(w, h, nslices=ns, lib=oracle_lib)
            col = None
            for t in range(1, steps + 1):
                o.clear_references()
                o.push_reference(f[t - 1], col=col)
                o.set_source(f[t])
                o.begin_p_picture(27)
                s, r = o.analyse_auto()
                assert np.array_equal(s, per[t - 1][0]) and np.array_equal(r, per[t - 1][1]), f"stream {i} step {t}: oracle"
                col = s
            o.close()
        want.append(per)
        d = [torch.from_numpy(x).cuda() for x in f]
        st = InterStage(w, h, nslices=ns, lib=cuda_lib)
        st.set_stream(stream.cuda_stream)
        st.push_reference_device(d[0].data_ptr(), w, w, h, None)
        st.begin_p_picture(27)
        stages.append(st)
        dev.append(d)
    n = len(stages)
    d_states = [[torch.zeros(s.nmb * 72, dtype=torch.uint8, device="cuda") for _ in range(steps)] for s in stages]
    d_res = [torch.zeros(s.nmb * 104, dtype=torch.uint8, device="cuda") for s in stages]
    torch.cuda.synchronize()
    batch = InterBatch(stages)
    for k in range(steps):
        t = k + 1
        col = [None] * n if k == 0 else [d_states[i][k - 1].data_ptr() for i in range(n)]
        batch.step([f[t].data_ptr() for f in dev], [f[t - 1].data_ptr() for f in dev], col,
                   [d_states[i][k].data_ptr() for i in range(n)], [d.data_ptr() for d in d_res])
        batch.sync()
        for i in range(n):
            assert np.array_equal(d_states[i][k].cpu().numpy().view(MBSTATE_DTYPE), want[i][k][0]), f"stream {i} step {t}: decisions"
            assert np.array_equal(d_res[i].cpu().numpy().view(MBRESULT_DTYPE), want[i][k][1]), f"stream {i} step {t}: results"
    batch.close()
    for st in stages:
        st.close()


def test_every_tuning_gives_the_same_results_and_the_tuner_picks_one(cuda_lib, tmp_path):
    """The batched step's knobs (CTAs per SM of the analysis, the planes' tile rows, the ticket order) change
    only its time: every one of the 12 settings gives each stream its single-stream results. The tuner times
    them all, keeps the fastest, ends as one step of its inputs would, and a second call finds the setting in
    its cache."""
    import torch

    streams = STREAMS[:4]
    frames = [_frames(i, w, h) for i, (w, h, _) in enumerate(streams)]
    want = []
    for (w, h, ns), f in zip(streams, frames):
        one = InterStage(w, h, nslices=ns, lib=cuda_lib)
        one.push_reference(f[0])
        one.set_source(f[1])
        one.begin_p_picture(27)
        want.append(one.analyse_auto())
        one.close()
    stream = torch.cuda.Stream()
    dev = [[torch.from_numpy(x).cuda() for x in f] for f in frames]
    stages = []
    for (w, h, ns), f in zip(streams, dev):
        st = InterStage(w, h, nslices=ns, lib=cuda_lib)
        st.set_stream(stream.cuda_stream)
        st.push_reference_device(f[0].data_ptr(), w, w, h, None)
        st.begin_p_picture(27)
        stages.append(st)
    n = len(stages)
    d_states = [torch.zeros(s.nmb * 72, dtype=torch.uint8, device="cuda") for s in stages]
    d_res = [torch.zeros(s.nmb * 104, dtype=torch.uint8, device="cuda") for s in stages]
    torch.cuda.synchronize()
    batch = InterBatch(stages)
    args = ([f[1].data_ptr() for f in dev], [f[0].data_ptr() for f in dev], [None] * n, [d.data_ptr() for d in d_states],
            [d.data_ptr() for d in d_res])

    def check(what):
        for i in range(n):
            assert np.array_equal(d_states[i].cpu().numpy().view(MBSTATE_DTYPE), want[i][0]), f"{what}: stream {i} decisions"
            assert np.array_equal(d_res[i].cpu().numpy().view(MBRESULT_DTYPE), want[i][1]), f"{what}: stream {i} results"
            d_res[i].zero_()

    for k2, group in ((4, 0), (5, 0), (6, 0), (4, 8)):
        for th in (16, 8):
            for order in (0, 1):
                for st in stages:  # the step pushes the reference again: start from the ring as it was
                    st.clear_references()
                    st.push_reference_device(dev[stages.index(st)][0].data_ptr(), st.width, st.width, st.height, None)
                    st.begin_p_picture(27)
                batch.set_tuning(k2, th, order, group)
                assert batch.tuning() == {"k2_ctas_per_sm": k2, "k1_tile_rows": th, "order": order, "k2_group": group}
                batch.step(*args)
                batch.sync()
                check(f"setting {k2}/{th}/{order}/{group}")
    for st, f in zip(stages, dev):
        st.clear_references()
        st.push_reference_device(f[0].data_ptr(), st.width, st.width, st.height, None)
        st.begin_p_picture(27)
    cache = str(tmp_path / "tuning.json")
    out = batch.autotune(*args, reps=3, cache=cache)
    assert not out["cached"] and len(out["all"]) == 16 and out["best"]["ms"] > 0
    assert min(a["ms"] for a in out["all"]) == out["best"]["ms"]
    check("after the tuner")
    assert all(st.lib.ironav_ctx_sync(st.ctx) == 0 for st in stages)
    # one reference pushed, as by one step: a step with the same inputs again gives the same results
    for st, f in zip(stages, dev):
        st.clear_references()
        st.push_reference_device(f[0].data_ptr(), st.width, st.width, st.height, None)
        st.begin_p_picture(27)
    again = batch.autotune(*args, reps=3, cache=cache)
    assert again["cached"] and again["best"]["k2_ctas_per_sm"] == out["best"]["k2_ctas_per_sm"]
    check("the cached setting")
    batch.close()
    for st in stages:
        st.close()
