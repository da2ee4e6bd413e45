"""10-bit pictures (the encoder's Yuv420p10 input, bd = 10, enc/mod.rs:140-143, 481-529): HalfPel::new
at bd 10 (enc/subpel.rs:57-115, half samples clipped to 1023), the analysis over 16-bit samples
(enc/frame.rs:641-671, 722-1019), and the scene-cut measure on 10-bit low-resolution luma
(crates/ironav-codec/src/change.rs:16-90, enc/mod.rs:689-693).

CPU tests pin the oracle's 10-bit boundary: a context's planes equal those of the interpolation entry that
the known-answer test checks against the decoder's luma_mc_ref at bd 10 (tests/test_oracle.py), its scene
totals equal the numpy statement, and it still finds the synthetic pan. GPU tests compare the sm_100a
library with the oracle, bit for bit, through the C ABI.

QP' = QP + 6 * (bd - 8) for 10-bit pictures (FrameCoder::new, enc/frame.rs:381-412), so lambda and the
P_Skip threshold come from QP + 12."""
import ctypes
import os

import numpy as np
import pytest

from ironav_b200.inter import MBSTATE_DTYPE, InterStage, IronavError
from ironav_b200.synth import Sequence
from tests.test_scene import numpy_change


def assert_same(a, b, what):
    if np.array_equal(a, b):
        return
    bad = np.nonzero(a != b)[0]
    i = int(bad[0])
    fields = [f for f in a.dtype.names if not np.array_equal(a[i][f], b[i][f])]
    raise AssertionError(f"{what}: {len(bad)} macroblocks differ; first {i}, fields {fields}: "
                         f"got {a[i][fields[0]]} want {b[i][fields[0]]}")


def full_range(rng, h, w):
    """10-bit noise over the whole range: the 6-tap filters overshoot both ends, so the clips to 0 and
    1023 are exercised."""
    return rng.integers(0, 1024, size=(h, w), dtype=np.uint16)


# ---- CPU: the oracle's 10-bit boundary -----------------------------------------------------------------

@pytest.mark.parametrize("size", [(64, 48), (40, 20)])
def test_oracle_context_planes_equal_the_known_answer_entry(oracle_lib, size):
    w, h = size
    pw, ph = (w + 15) // 16 * 16, (h + 15) // 16 * 16
    rng = np.random.default_rng(w * 31 + h)
    luma = full_range(rng, ph, pw)
    st = InterStage(w, h, lib=oracle_lib, bd=10)
    st.push_reference(luma)  # a macroblock-aligned reconstruction, used as is
    got = st.planes(0)
    assert got.dtype == np.uint16 and got.max() == 1023
    hp = oracle_lib.oracle_halfpel_new(luma.ctypes.data, pw, ph, 10)
    try:
        want = np.zeros_like(got)
        for k in range(4):
            oracle_lib.oracle_halfpel_plane(hp, k, want[k].ctypes.data)
    finally:
        oracle_lib.oracle_halfpel_free(hp)
    assert np.array_equal(got, want)


def test_oracle_10bit_finds_the_pan(oracle_lib):
    seq = Sequence.config("cif", 2)
    st = InterStage(352, 288, nslices=2, lib=oracle_lib, bd=10)
    st.push_reference(seq.frame10(0))
    st.set_source(seq.frame10(1))
    st.begin_p_picture(26 + 12)
    states, res = st.analyse_auto()
    res2 = st.analyse_replay(states)
    pan = np.array(seq.pan(1))
    mv = res2["mvs"][:, 0].astype(int)
    assert (np.abs(mv - pan) <= 4).all(axis=1).mean() > 0.8


@pytest.mark.parametrize("size,cut", [((176, 144), False), ((198, 102), True)])
def test_oracle_10bit_scene_totals(oracle_lib, size, cut):
    w, h = size
    a = Sequence.config("1080p", 3, seed=11, size=size)
    b = Sequence.config("1080p", 3, seed=12, size=size) if cut else a
    prev, cur = a.frame10(1), b.frame10(2)
    st = InterStage(w, h, lib=oracle_lib, bd=10)
    assert st.scene_change(prev, cur) == numpy_change(prev, cur, st.mb_w, st.mb_h)


def test_depths_and_sample_types_are_checked(oracle_lib):
    for bd in (9, 12, 16):
        with pytest.raises(IronavError) as e:
            InterStage(64, 48, lib=oracle_lib, bd=bd)
        assert e.value.status == 3
    st = InterStage(64, 48, lib=oracle_lib, bd=10)
    with pytest.raises(TypeError):
        st.set_source(np.zeros((48, 64), dtype=np.uint8))


# ---- GPU: the sm_100a library against the oracle -----------------------------------------------------

def _pair(oracle_lib, cuda_lib, w, h, **kw):
    return InterStage(w, h, lib=oracle_lib, bd=10, **kw), InterStage(w, h, lib=cuda_lib, bd=10, **kw)


@pytest.mark.gpu
@pytest.mark.parametrize("size", [(352, 288), (34, 18), (1920, 1080)])
def test_gpu_10bit_planes(oracle_lib, cuda_lib, size):
    w, h = size
    luma = full_range(np.random.default_rng(w + 3 * h), h, w)
    o, c = _pair(oracle_lib, cuda_lib, w, h)
    o.push_reference(luma)
    c.push_reference(luma)
    po, pc = o.planes(0), c.planes(0)
    for k, name in enumerate("Gbhj"):
        assert np.array_equal(po[k], pc[k]), f"plane {name} differs at {np.argwhere(po[k] != pc[k])[:3]}"


def _sequence(oracle_lib, cuda_lib, cfg, qp, nslices, size=None, **pic):
    seq = Sequence.config(cfg, 3, size=size)
    f = [seq.frame10(t) for t in range(3)]
    o, c = _pair(oracle_lib, cuda_lib, seq.width, seq.height, nslices=nslices)
    oracle_lib.oracle_set_threads(o.ctx, os.cpu_count() or 1)
    for st in (o, c):
        st.push_reference(f[0])
        st.set_source(f[1])
        st.begin_p_picture(qp)
    col_o, _ = o.analyse_auto()
    col_c, _ = c.analyse_auto()
    assert_same(col_c, col_o, "decisions of the reference picture")
    for st in (o, c):
        st.clear_references()
        st.push_reference(f[1], col=col_o)
        st.set_source(f[2])
        st.begin_p_picture(qp, **pic)
    return o, c


@pytest.mark.gpu
@pytest.mark.parametrize("cfg,size,qp,nslices,pic", [
    ("cif", None, 26 + 12, 2, {}),
    ("1080p", None, 27 + 12, 8, {}),
    ("1080p", (1280, 720), 27 + 12, 5, dict(fast=True)),
    ("1080p", (1280, 720), 20 + 12, 5, dict(sub8=True)),
])
def test_gpu_10bit_auto_and_replay(oracle_lib, cuda_lib, cfg, size, qp, nslices, pic):
    o, c = _sequence(oracle_lib, cuda_lib, cfg, qp, nslices, size=size, **pic)
    so, ro = o.analyse_auto()
    sc, rc = c.analyse_auto()
    assert_same(sc, so, "10-bit auto decisions")
    assert_same(rc, ro, "10-bit auto results")
    assert_same(c.analyse_replay(so), o.analyse_replay(so), "10-bit replay")


@pytest.mark.gpu
def test_gpu_10bit_random_decisions_and_two_references(oracle_lib, cuda_lib):
    """Full-range 10-bit noise (every clip taken) and arbitrary neighbour vectors up to the level limits,
    over two reference pictures."""
    w, h = 96, 64
    rng = np.random.default_rng(23)
    base = full_range(rng, h + 40, w + 40)
    o, c = _pair(oracle_lib, cuda_lib, w, h, max_refs=2, nslices=2)
    nmb = o.nmb
    col = np.zeros(nmb, dtype=MBSTATE_DTYPE)
    col["inter"] = 1
    col["mvs"] = rng.integers(-300, 300, size=(nmb, 16, 2))
    for st in (o, c):
        st.push_reference(base[7:h + 7, 2:w + 2].copy())
        st.push_reference(base[:h, :w].copy(), col=col)
        st.set_source(base[3:h + 3, 5:w + 5].copy())
        st.begin_p_picture(24 + 12, nrefs_active=2)
    states = np.zeros(nmb, dtype=MBSTATE_DTYPE)
    states["inter"] = rng.integers(0, 4, nmb) > 0
    states["refs"] = np.where(states["inter"][:, None] == 1, rng.integers(0, 2, size=(nmb, 4)), -1)
    states["mvs"] = np.stack([rng.integers(-2048, 2048, size=(nmb, 16)), rng.integers(-512, 512, size=(nmb, 16))],
                             axis=-1)
    want = o.analyse_replay(states)
    for form in (1, 0, 2):  # replay mode's kernels: the warp form (the 10-bit default), 8- and 16-lane groups
        assert cuda_lib.ironav_set_replay_form(c.ctx, form) == 0
        assert_same(c.analyse_replay(states), want, f"10-bit replay on random decisions, form {form}")
    so, ro = o.analyse_auto()
    sc, rc = c.analyse_auto()
    assert_same(sc, so, "10-bit two-reference decisions")
    assert_same(rc, ro, "10-bit two-reference results")


@pytest.mark.gpu
@pytest.mark.parametrize("size,cut", [((352, 288), False), ((1920, 1080), True), ((198, 102), False)])
def test_gpu_10bit_scene_totals(oracle_lib, cuda_lib, size, cut):
    w, h = size
    a = Sequence.config("1080p", 3, seed=11, size=size)
    b = Sequence.config("1080p", 3, seed=12, size=size) if cut else a
    prev, cur = a.frame10(1), b.frame10(2)
    o, c = _pair(oracle_lib, cuda_lib, w, h)
    assert c.scene_change(prev, cur) == o.scene_change(prev, cur)


@pytest.mark.gpu
def test_gpu_10bit_device_forms_and_inloop(oracle_lib, cuda_lib):
    import torch

    from tests.test_inloop import _policy, run_raster

    seq = Sequence.config("cif", 2)
    f0, f1 = seq.frame10(0), seq.frame10(1)
    o = InterStage(352, 288, nslices=2, lib=oracle_lib, bd=10)
    o.push_reference(f0)
    o.set_source(f1)
    o.begin_p_picture(38)
    so, ro = o.analyse_auto()

    d = InterStage(352, 288, nslices=2, lib=cuda_lib, bd=10)
    d.set_stream(torch.cuda.current_stream().cuda_stream)
    t0 = torch.from_numpy(f0.view(np.int16)).cuda()
    t1 = torch.from_numpy(f1.view(np.int16)).cuda()
    d.push_reference_device(t0.data_ptr(), 352, 352, 288, None)
    d.set_source_device(t1.data_ptr(), 352)
    d.begin_p_picture(38)
    ds = torch.zeros(d.nmb * 72, dtype=torch.uint8, device="cuda")
    dr = torch.zeros(d.nmb * 104, dtype=torch.uint8, device="cuda")
    d.analyse_auto_device(ds.data_ptr(), dr.data_ptr())
    d.sync()
    from ironav_b200.inter import MBRESULT_DTYPE

    assert_same(ds.cpu().numpy().view(MBSTATE_DTYPE), so, "10-bit device decisions")
    assert_same(dr.cpu().numpy().view(MBRESULT_DTYPE), ro, "10-bit device results")

    decide = _policy(oracle_lib, 38)
    s_o, r_o = run_raster(o, decide)
    s_c, r_c = run_raster(d, decide)
    assert_same(s_c, s_o, "10-bit in-loop decisions")
    assert_same(r_c, r_o, "10-bit in-loop results")
