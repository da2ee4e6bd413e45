"""GPU parity: the sm_100a library (libironav_inter_cuda.so) against the oracle, through the C ABI.

Everything here is integer work, so the bar is bit-exactness: planes byte for byte, and every field
of every macroblock's result (vectors, costs, partitions, sub-partitions, references, P_Skip vector
and SAD, evaluation counts) and decision.
"""
import os

import numpy as np
import pytest

from ironav_b200.inter import MBRESULT_DTYPE, MBSTATE_DTYPE, InterStage, IronavError
from ironav_b200.synth import Sequence

pytestmark = pytest.mark.gpu

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def assert_same(a, b, what):
    if np.array_equal(a, b):
        return
    bad = np.nonzero(a != b)[0]
    i = int(bad[0])
    fields = [f for f in a.dtype.names if not np.array_equal(a[i][f], b[i][f])]
    raise AssertionError(f"{what}: {len(bad)} macroblocks differ; first {i}, fields {fields}: "
                         f"got {a[i][fields[0]]} want {b[i][fields[0]]}")


def stage_pair(oracle_lib, cuda_lib, w, h, **kw):
    return InterStage(w, h, lib=oracle_lib, **kw), InterStage(w, h, lib=cuda_lib, **kw)


def run_both(pair, fn):
    return fn(pair[0]), fn(pair[1])


@pytest.mark.parametrize("size", [(352, 288), (34, 18), (64, 48), (1920, 1080)])
def test_planes_byte_exact(oracle_lib, cuda_lib, size):
    w, h = size
    rng = np.random.default_rng(w * 7 + h)
    luma = rng.integers(0, 256, size=(h, w), dtype=np.uint8)
    o, c = stage_pair(oracle_lib, cuda_lib, w, h)
    o.push_reference(luma)
    c.push_reference(luma)
    po, pc = o.planes(0), c.planes(0)
    for k, name in enumerate("Gbhj"):
        assert np.array_equal(po[k], pc[k]), f"plane {name} of {w}x{h} differs at {np.argwhere(po[k] != pc[k])[:3]}"


def test_planes_rebuilt_in_a_reused_slot(oracle_lib, cuda_lib):
    """the_threaded_half_sample_planes_equal_the_single_threaded_ones (crates/ironav-codec/src/h264/enc/
    mod.rs:1302-1330), on its picture (80x112, the 32-bit LCG from seed 5) and its inverse: with one
    reference held, every push rebuilds the planes in the slot the previous picture used, and each
    rebuild equals a fresh context's planes of the same picture and the oracle's."""
    pw, ph = 80, 112
    seed, vals = 5, []
    for _ in range(pw * ph):
        seed = (seed * 1103515245 + 12345) & 0xFFFFFFFF
        vals.append((seed >> 16) % 256)
    luma = np.array(vals, np.uint8).reshape(ph, pw)
    luma2 = (255 - luma).astype(np.uint8)
    o = InterStage(pw, ph, max_refs=1, lib=oracle_lib)
    c = InterStage(pw, ph, max_refs=1, lib=cuda_lib)
    for k, pic in enumerate([luma, luma2, luma, luma2]):
        o.push_reference(pic)
        c.push_reference(pic)
        fresh = InterStage(pw, ph, max_refs=1, lib=cuda_lib)
        fresh.push_reference(pic)
        got = c.planes(0)
        assert np.array_equal(got, fresh.planes(0)), f"push {k}: the reused slot's planes differ from a fresh build"
        assert np.array_equal(got, o.planes(0)), f"push {k}: planes differ from the oracle's"


@pytest.mark.parametrize("bd", [8, 10])
def test_planes_from_a_misaligned_device_picture(oracle_lib, cuda_lib, bd):
    """A reference handed over in device memory at an unaligned address, rows an odd number of samples
    apart, takes the planes kernel's sample-by-sample staging on every tile: its planes equal the
    oracle's."""
    import torch

    w, h = 352, 288
    maxv = (1 << bd) - 1
    dt = np.uint8 if bd == 8 else np.uint16
    luma = np.random.default_rng(17 + bd).integers(0, maxv + 1, size=(h, w)).astype(dt)
    stride, off = w + 3, 1
    buf = np.zeros(h * stride + 8, dt)
    buf[off:off + h * stride].reshape(h, stride)[:, :w] = luma
    tbuf = torch.from_numpy(buf.view(np.int16) if bd == 10 else buf).cuda()
    c = InterStage(w, h, lib=cuda_lib, bd=bd)
    c.set_stream(torch.cuda.current_stream().cuda_stream)
    c.push_reference_device(tbuf.data_ptr() + off * buf.itemsize, stride, w, h, None)
    c.sync()
    o = InterStage(w, h, lib=oracle_lib, bd=bd)
    o.push_reference(luma)
    assert np.array_equal(c.planes(0), o.planes(0))


def test_planes_of_a_macroblock_aligned_reconstruction(oracle_lib, cuda_lib):
    """A reconstruction is 16*mb_w x 16*mb_h and is used as is (no edge repetition inside it)."""
    w, h = 40, 20  # mb 3 x 2
    rng = np.random.default_rng(5)
    recon = rng.integers(0, 256, size=(32, 48), dtype=np.uint8)
    o, c = stage_pair(oracle_lib, cuda_lib, w, h)
    o.push_reference(recon)
    c.push_reference(recon)
    assert np.array_equal(o.planes(0), c.planes(0))


def test_golden_cases(cuda_lib):
    """The CUDA library reproduces the committed oracle fixtures (tests/golden/oracle_cif.npz)."""
    from tests.golden.make_golden import CASES, run_case

    data = np.load(os.path.join(GOLDEN, "oracle_cif.npz"))
    for name, case in CASES.items():
        luma_hash, states, res, rstates, rres = run_case(cuda_lib, **case)
        assert luma_hash == str(data[f"{name}_hash"]), f"{name}: synthetic input changed"
        assert_same(states, data[f"{name}_states"].view(MBSTATE_DTYPE), f"{name} decisions")
        assert_same(res, data[f"{name}_results"].view(MBRESULT_DTYPE), f"{name} auto results")
        assert_same(rres, data[f"{name}_replay"].view(MBRESULT_DTYPE), f"{name} replay results")


def _sequence_case(oracle_lib, cuda_lib, cfg, qp, nslices, src=2, size=None, **pic):
    seq = Sequence.config(cfg, src + 1, size=size)
    f = [seq.frame(t) for t in range(src + 1)]
    o, c = stage_pair(oracle_lib, cuda_lib, seq.width, seq.height, nslices=nslices)
    oracle_lib.oracle_set_threads(o.ctx, os.cpu_count() or 1)
    # the reference picture's own decisions give the co-located candidates
    for st in (o, c):
        st.push_reference(f[src - 2])
        st.set_source(f[src - 1])
        st.begin_p_picture(qp)
    col_o, _ = o.analyse_auto()
    col_c, _ = c.analyse_auto()
    assert_same(col_c, col_o, "decisions of the reference picture")
    for st in (o, c):
        st.clear_references()
        st.push_reference(f[src - 1], col=col_o)
        st.set_source(f[src])
        st.begin_p_picture(qp, **pic)
    return o, c


@pytest.mark.parametrize("qp", [22, 27, 32])
def test_1080p_auto_and_replay(oracle_lib, cuda_lib, qp):
    o, c = _sequence_case(oracle_lib, cuda_lib, "1080p", qp, nslices=8)
    so, ro = o.analyse_auto()
    sc, rc = c.analyse_auto()
    assert_same(sc, so, f"1080p qp{qp} auto decisions")
    assert_same(rc, ro, f"1080p qp{qp} auto results")
    assert_same(c.analyse_replay(so), o.analyse_replay(so), f"1080p qp{qp} replay")


def test_4k_replay(oracle_lib, cuda_lib):
    o, c = _sequence_case(oracle_lib, cuda_lib, "4k", 27, nslices=16)
    so, ro = o.analyse_auto()
    sc, rc = c.analyse_auto()
    assert_same(sc, so, "4k auto decisions")
    assert_same(c.analyse_replay(so), o.analyse_replay(so), "4k replay")


@pytest.mark.parametrize("mode", [dict(fast=True), dict(sub8=True), dict(fast=False)])
def test_modes_720p(oracle_lib, cuda_lib, mode):
    o, c = _sequence_case(oracle_lib, cuda_lib, "1080p", 20 if mode.get("sub8") else 27, nslices=5, size=(1280, 720),
                          **mode)
    so, ro = o.analyse_auto()
    sc, rc = c.analyse_auto()
    assert_same(sc, so, f"{mode} decisions")
    assert_same(rc, ro, f"{mode} results")
    assert_same(c.analyse_replay(so), o.analyse_replay(so), f"{mode} replay")


@pytest.mark.parametrize("mode", [dict(), dict(fast=True), dict(sub8=True)])
def test_replay_forms_agree_on_random_decisions(oracle_lib, cuda_lib, mode):
    """Replay mode's two kernels (one macroblock per 8-lane group, the default; one per warp) and the oracle on
    three references with arbitrary neighbour decisions up to the level limits, so that predictors, candidates
    and diamond moves land on the clamps and the rounded candidates just outside them."""
    seq = Sequence.config("cif", 4)
    o, c = stage_pair(oracle_lib, cuda_lib, 352, 288, nslices=3, max_refs=3)
    rng = np.random.default_rng(17 + len(mode))
    nmb = o.nmb
    col = np.zeros(nmb, dtype=MBSTATE_DTYPE)
    col["inter"] = rng.integers(0, 2, nmb)
    col["mvs"] = rng.integers(-2100, 2100, size=(nmb, 16, 2))
    for st in (o, c):
        st.push_reference(seq.frame(0))
        st.push_reference(seq.frame(1))
        st.push_reference(seq.frame(2), col=col)
        st.set_source(seq.frame(3))
        st.begin_p_picture(18 if mode.get("sub8") else 28, nrefs_active=3, **mode)
    states = np.zeros(nmb, dtype=MBSTATE_DTYPE)
    states["inter"] = rng.integers(0, 4, nmb) > 0
    states["refs"] = np.where(states["inter"][:, None] == 1, rng.integers(-1, 3, size=(nmb, 4)), -1)
    mv = np.stack([rng.integers(-2048, 2048, size=(nmb, 16)), rng.integers(-512, 512, size=(nmb, 16))], axis=-1)
    near = rng.integers(0, 3, size=(nmb, 1, 1))
    edge = np.where(mv >= 0, 1, -1) * np.array([2047, 511]) - rng.integers(0, 3, size=mv.shape)  # at the limits
    states["mvs"] = np.where(near == 0, mv // 64, np.where(near == 1, edge, mv))
    want = o.analyse_replay(states)
    for form, name in ((0, "8-lane group"), (1, "warp"), (2, "16-lane group"), (3, "4-lane group")):
        assert cuda_lib.ironav_set_replay_form(c.ctx, form) == 0
        assert_same(c.analyse_replay(states), want, f"{mode} {name} form")
    assert cuda_lib.ironav_set_replay_form(c.ctx, 0) == 0


def test_random_decisions_exercise_the_clamps(oracle_lib, cuda_lib):
    """Replay against arbitrary neighbour vectors, up to the level limits (+-2048 x +-512 quarter samples):
    the predictors and candidates land on the search bounds, where clamped diamond moves are scored on
    demand."""
    seq = Sequence.config("cif", 3)
    o, c = stage_pair(oracle_lib, cuda_lib, 352, 288, nslices=2)
    rng = np.random.default_rng(11)
    nmb = o.nmb
    col = np.zeros(nmb, dtype=MBSTATE_DTYPE)
    col["inter"] = rng.integers(0, 2, nmb)
    col["mvs"] = rng.integers(-600, 600, size=(nmb, 16, 2))
    for st in (o, c):
        st.push_reference(seq.frame(0), col=col)
        st.set_source(seq.frame(1))
        st.begin_p_picture(26)
    states = np.zeros(nmb, dtype=MBSTATE_DTYPE)
    states["inter"] = rng.integers(0, 4, nmb) > 0
    states["refs"] = np.where(states["inter"][:, None] == 1, 0, -1)
    mv = np.stack([rng.integers(-2048, 2048, size=(nmb, 16)), rng.integers(-512, 512, size=(nmb, 16))], axis=-1)
    small = rng.integers(0, 2, size=(nmb, 1, 1)) == 1
    states["mvs"] = np.where(small, mv // 64, mv)
    assert_same(c.analyse_replay(states), o.analyse_replay(states), "replay on random decisions")


@pytest.mark.parametrize("size", [(16, 16), (32, 16), (48, 32), (80, 64)])
def test_small_pictures(oracle_lib, cuda_lib, size):
    w, h = size
    rng = np.random.default_rng(w + 100 * h)
    base = rng.integers(0, 256, size=(h + 40, w + 40), dtype=np.uint8)
    ref, src = base[:h, :w].copy(), base[3:h + 3, 5:w + 5].copy()
    o, c = stage_pair(oracle_lib, cuda_lib, w, h, max_refs=2, nslices=min(2, (h + 15) // 16))
    for st in (o, c):
        st.push_reference(base[7:h + 7, 2:w + 2].copy())
        st.push_reference(ref)
        st.set_source(src)
        st.begin_p_picture(24, nrefs_active=2)
    so, ro = o.analyse_auto()
    sc, rc = c.analyse_auto()
    assert_same(sc, so, f"{size} decisions")
    assert_same(rc, ro, f"{size} results")
    assert_same(c.analyse_replay(so), o.analyse_replay(so), f"{size} replay")


def test_device_forms_match_host_forms(cuda_lib):
    import torch

    seq = Sequence.config("cif", 2)
    f0, f1 = seq.frame(0), seq.frame(1)
    st = InterStage(352, 288, nslices=2, lib=cuda_lib)
    st.push_reference(f0)
    st.set_source(f1)
    st.begin_p_picture(26)
    states, res = st.analyse_auto()
    rep = st.analyse_replay(states)

    d = InterStage(352, 288, nslices=2, lib=cuda_lib)
    stream = torch.cuda.current_stream()
    d.set_stream(stream.cuda_stream)
    t0 = torch.from_numpy(f0).cuda()
    t1 = torch.from_numpy(f1).cuda()
    d.push_reference_device(t0.data_ptr(), 352, 352, 288, None)
    d.set_source_device(t1.data_ptr(), 352)
    d.begin_p_picture(26)
    ds = torch.zeros(d.nmb * 72, dtype=torch.uint8, device="cuda")
    dr = torch.zeros(d.nmb * 104, dtype=torch.uint8, device="cuda")
    d.analyse_auto_device(ds.data_ptr(), dr.data_ptr())
    d.sync()
    assert_same(ds.cpu().numpy().view(MBSTATE_DTYPE), states, "device auto decisions")
    assert_same(dr.cpu().numpy().view(MBRESULT_DTYPE), res, "device auto results")
    d.analyse_replay_device(ds.data_ptr(), dr.data_ptr())
    d.sync()
    assert_same(dr.cpu().numpy().view(MBRESULT_DTYPE), rep, "device replay results")


@pytest.mark.parametrize("bd", [8, 10])
def test_device_source_with_odd_stride_and_size(cuda_lib, bd):
    """A source handed over in device memory, rows an odd number of samples apart and a size that is not a
    whole number of macroblocks, is padded as the host form pads it: the same decisions and results."""
    import torch

    w, h = 200, 120
    seq = Sequence.config("cif", 2, size=(w, h))
    f0, f1 = (seq.frame10(t) if bd == 10 else seq.frame(t) for t in (0, 1))
    qp = 26 + 6 * (bd - 8)
    st = InterStage(w, h, nslices=2, lib=cuda_lib, bd=bd)
    st.push_reference(f0)
    st.set_source(f1)
    st.begin_p_picture(qp)
    states, res = st.analyse_auto()
    d = InterStage(w, h, nslices=2, lib=cuda_lib, bd=bd)
    d.set_stream(torch.cuda.current_stream().cuda_stream)
    d.push_reference(f0)
    stride = w + 5
    buf = np.zeros((h, stride), f1.dtype)
    buf[:, :w] = f1
    t1 = torch.from_numpy(buf.view(np.int16) if bd == 10 else buf).cuda()
    d.set_source_device(t1.data_ptr(), stride)
    d.begin_p_picture(qp)
    ds = torch.zeros(d.nmb * 72, dtype=torch.uint8, device="cuda")
    dr = torch.zeros(d.nmb * 104, dtype=torch.uint8, device="cuda")
    d.analyse_auto_device(ds.data_ptr(), dr.data_ptr())
    d.sync()
    assert_same(ds.cpu().numpy().view(MBSTATE_DTYPE), states, "device-source decisions")
    assert_same(dr.cpu().numpy().view(MBRESULT_DTYPE), res, "device-source results")


def test_wavefront_wait_times_out_and_the_context_recovers(oracle_lib, cuda_lib):
    """A macroblock whose decision is never published (the test withholds it) makes the waits behind it
    give up after a bounded number of polls; the call reports a timeout and the next call works."""
    seq = Sequence.config("cif", 2)
    c = InterStage(352, 288, nslices=2, lib=cuda_lib)
    o = InterStage(352, 288, nslices=2, lib=oracle_lib)
    for st in (o, c):
        st.push_reference(seq.frame(0))
        st.set_source(seq.frame(1))
        st.begin_p_picture(26)
    assert cuda_lib.ironav_debug_wait_limit(c.ctx, 20000) == 0
    assert cuda_lib.ironav_debug_withhold(c.ctx, 5) == 0
    with pytest.raises(IronavError) as e:
        c.analyse_auto()
    assert e.value.status == 100
    assert cuda_lib.ironav_debug_withhold(c.ctx, -1) == 0
    sc, rc = c.analyse_auto()
    so, ro = o.analyse_auto()
    assert_same(sc, so, "decisions after a timeout")
    assert_same(rc, ro, "results after a timeout")


def test_bad_arguments_are_rejected(cuda_lib):
    with pytest.raises(IronavError) as e:
        InterStage(351, 288, lib=cuda_lib)
    assert e.value.status == 3
    st = InterStage(64, 48, lib=cuda_lib)
    with pytest.raises(IronavError) as e:
        st.begin_p_picture(26)  # no reference yet
    assert e.value.status == 3
    with pytest.raises(IronavError):
        st.analyse_replay(np.zeros(st.nmb, dtype=MBSTATE_DTYPE))
