"""Scene-cut measure (change_threads, crates/ironav-codec/src/change.rs:56-90, on the low-resolution luma of
LowRes::new, change.rs:16-24, taken of the padded source as H264Encoder::low_res does, enc/mod.rs:689-693).

CPU: the oracle against an independent numpy statement of the same arithmetic, and its behaviour on
still, panned and cut pictures. GPU: the CUDA library against the oracle, totals equal."""
import numpy as np
import pytest

from ironav_b200.inter import InterStage
from ironav_b200.synth import Sequence


def numpy_change(prev, cur, mb_w, mb_h):
    def low(y):
        h, w = y.shape
        pad = np.pad(y.astype(np.int64), ((0, mb_h * 16 - h), (0, mb_w * 16 - w)), mode="edge")
        return pad.reshape(mb_h * 4, 4, mb_w * 4, 4).sum(axis=(1, 3)) >> 4
    lp, lc = low(prev), low(cur)
    lh, lw = lc.shape
    inter = intra = 0
    for by in range(0, lh - 7, 8):
        for bx in range(0, lw - 7, 8):
            blk = lc[by:by + 8, bx:bx + 8]
            mean = int(blk.sum()) // 64
            intra += int(np.abs(blk - mean).sum())
            best = None
            for dy in range(-4, 5):
                for dx in range(-4, 5):
                    ox, oy = bx + dx, by + dy
                    if ox < 0 or oy < 0 or ox + 8 > lw or oy + 8 > lh:
                        continue
                    sad = int(np.abs(blk - lp[oy:oy + 8, ox:ox + 8]).sum())
                    best = sad if best is None else min(best, sad)
            inter += best
    return inter, intra


def _pair(size, cut):
    w, h = size
    a = Sequence.config("1080p", 3, seed=11, size=(w, h))
    b = Sequence.config("1080p", 3, seed=12, size=(w, h)) if cut else a
    return a.frame(1), b.frame(2)


@pytest.mark.parametrize("size,cut", [((176, 144), False), ((352, 288), True), ((198, 102), False)])
def test_oracle_matches_numpy_statement(oracle_lib, size, cut):
    prev, cur = _pair(size, cut)
    st = InterStage(size[0], size[1], lib=oracle_lib)
    assert st.scene_change(prev, cur) == numpy_change(prev, cur, st.mb_w, st.mb_h)


def test_still_pan_and_cut(oracle_lib):
    seq = Sequence.config("cif", 3)
    st = InterStage(352, 288, lib=oracle_lib)
    f1, f2 = seq.frame(1), seq.frame(2)
    inter, intra = st.scene_change(f1, f1)
    assert inter == 0 and intra > 0
    assert not st.scene_cut(f1, f2)  # a pan of a few samples is well predicted
    other = Sequence.config("cif", 3, seed=99).frame(1)
    assert st.scene_cut(f1, other)


def _cut_sequence():
    """a_scene_cut_starts_an_idr_picture's pictures (crates/ironav-codec/src/h264/enc/mod.rs:1071-1086):
    96x64 `scene` for pictures 0-4, a vertical gradient (255 - 3 * row) from picture 5 on."""
    from tests.test_decode_inter import scene

    w, h = 96, 64
    grad = (255 - np.arange(w * h) // w * 3).astype(np.uint8).reshape(h, w)
    return w, h, [scene(w, h, t)[0] if t < 5 else grad for t in range(10)]


def _idr_pictures(lib):
    """The pictures the encoder starts as IDR (enc/mod.rs:706-714): the first, and each whose scene-cut
    measure against the picture before it says cut (the key-picture interval, KEYINT = 250 at
    enc/mod.rs:27, is not reached in 10 pictures)."""
    w, h, pics = _cut_sequence()
    st = InterStage(w, h, lib=lib)
    return [0] + [t for t in range(1, len(pics)) if st.scene_cut(pics[t - 1], pics[t])]


def test_a_scene_cut_starts_an_idr_picture(oracle_lib):
    assert _idr_pictures(oracle_lib) == [0, 5]


@pytest.mark.gpu
def test_gpu_a_scene_cut_starts_an_idr_picture(oracle_lib, cuda_lib):
    assert _idr_pictures(cuda_lib) == [0, 5]
    w, h, pics = _cut_sequence()
    o, c = InterStage(w, h, lib=oracle_lib), InterStage(w, h, lib=cuda_lib)
    for t in range(1, len(pics)):
        assert c.scene_change(pics[t - 1], pics[t]) == o.scene_change(pics[t - 1], pics[t]), t


@pytest.mark.gpu
@pytest.mark.parametrize("size", [(352, 288), (1920, 1080), (3840, 2160), (40, 24)])
def test_scene_change_gpu_matches_oracle(oracle_lib, cuda_lib, size):
    for cut in (False, True):
        prev, cur = _pair(size, cut)
        o = InterStage(size[0], size[1], lib=oracle_lib)
        c = InterStage(size[0], size[1], lib=cuda_lib)
        assert c.scene_change(prev, cur) == o.scene_change(prev, cur), (size, cut)
