"""The learned form's judge (ironav_set_learned): with proposals set, the P analysis scores every integer vector
within +-2 samples of each of a macroblock's 4 proposed vectors by the exact integer cost, refines the best by
the plain search's sub-sample steps, and falls back to the plain search on the other partitioning classes or
when no proposal is as cheap as the predictor's start plus the margin.

CPU: the oracle's judge — the class fallback reproduces the plain stream byte for byte, the judged streams
decode under FFmpeg to the encoder's reconstruction, and every searched macroblock lands in exactly one
counter. GPU: the sm_100a library's judge against the oracle's with the same proposals, bit for bit (codes,
states, reconstructions, stream bytes and counters), in decide mode and in auto mode; and the trained
proposer network inside the device encoder.
"""
from __future__ import annotations


import numpy as np
import pytest

from ironav_b200.encoder import DeviceEncoder, Encoder
from ironav_b200.synth import Sequence
from tests.stream_util import check_stream_decodes_to


def make_proposals(seq: Sequence, t: int, mb_w: int, mb_h: int, seed: int, classes=(0, 1, 1, 1, 2, 3, 4)):
    """Seeded proposals for picture t: vectors around the sequence's pan (quarter samples), some near it, some
    off by up to 24 samples, with classes drawn from `classes` (so that every path of the judge is taken)."""
    rng = np.random.default_rng([seed, t])
    n = mb_w * mb_h
    px, py = seq.pan(t)
    qx, qy = seq.pan(t - 1) if t > 0 else (px, py)
    base = np.array([qx - px, qy - py], dtype=np.int32)
    spread = np.where(rng.random((n, 4, 1)) < 0.6, 6, 96)
    v = base[None, None, :] + rng.integers(-1, 2, size=(n, 4, 2)) * rng.integers(0, spread + 1, size=(n, 4, 2))
    cands = np.clip(v, [-2048, -512], [2047, 511]).astype(np.int16).reshape(n, 8)
    cls = np.asarray(classes, dtype=np.uint8)[rng.integers(0, len(classes), size=n)]
    return cands, cls


class HostProposals:
    """Proposals in host memory (the oracle reads them when it analyses), refreshed before each P picture."""

    def __init__(self, enc: Encoder, seq: Sequence, seed: int, margin: int = 0, **kw):
        st = enc.st
        self.seq, self.seed, self.kw, self.t = seq, seed, kw, 0
        self.cands = np.zeros((st.nmb, 8), dtype=np.int16)
        self.cls = np.zeros(st.nmb, dtype=np.uint8)
        self.stats = np.zeros(3, dtype=np.uint32)
        st._check(enc.lib.ironav_set_learned(st.ctx, self.cands.ctypes.data, self.cls.ctypes.data, margin, self.stats.ctypes.data),
                  "ironav_set_learned")
        enc.before_p = self

    def __call__(self, enc, *args) -> None:
        self.t = enc.loop.count - 1
        c, k = make_proposals(self.seq, self.t, enc.st.mb_w, enc.st.mb_h, self.seed, **self.kw)
        self.cands[:] = c
        self.cls[:] = k


class DeviceProposals:
    """The same proposals in device memory, copied up on the encoder's stream before each P picture."""

    def __init__(self, enc: DeviceEncoder, seq: Sequence, seed: int, margin: int = 0, **kw):
        import torch

        self.torch = torch
        st = enc.st
        self.seq, self.seed, self.kw = seq, seed, kw
        dev = enc.d_rec.device
        self.cands = torch.zeros((st.nmb, 8), dtype=torch.int16, device=dev)
        self.cls = torch.zeros(st.nmb, dtype=torch.uint8, device=dev)
        self.stats = torch.zeros(3, dtype=torch.int32, device=dev)
        st._check(enc.lib.ironav_set_learned(st.ctx, self.cands.data_ptr(), self.cls.data_ptr(), margin, self.stats.data_ptr()),
                  "ironav_set_learned")
        enc.before_p = self

    def __call__(self, enc, *args) -> None:
        t = enc.loop.count - 1
        c, k = make_proposals(self.seq, t, enc.st.mb_w, enc.st.mb_h, self.seed, **self.kw)
        with self.torch.cuda.stream(enc.stream):
            self.cands.copy_(self.torch.from_numpy(c))
            self.cls.copy_(self.torch.from_numpy(k))

    def counters(self) -> np.ndarray:
        return self.stats.cpu().numpy().astype(np.uint32)


def _encode_host(lib, seq, frames, proposals=None, margin=0, **kw):
    enc = Encoder(seq.width, seq.height, lib=lib, **kw)
    hp = HostProposals(enc, seq, seed=7, margin=margin, **(proposals or {})) if proposals is not None else None
    out, recons = [], []
    try:
        for t in range(frames):
            cb, cr = seq.chroma(t)
            out.append(enc.encode(seq.frame(t), cb, cr))
            recons.append(tuple(a.copy() for a in enc.recon))
    finally:
        enc.close()
    return out, recons, (hp.stats.copy() if hp is not None else None)


# ---- CPU: the oracle's judge -------------------------------------------------------------------------------

def test_set_learned_checks_its_arguments(oracle_lib):
    from ironav_b200.inter import InterStage

    st = InterStage(64, 48, lib=oracle_lib)
    try:
        a = np.zeros(96, dtype=np.int16)
        assert oracle_lib.ironav_set_learned(st.ctx, a.ctypes.data, None, 0, None) != 0
        assert oracle_lib.ironav_set_learned(st.ctx, None, None, -1, None) != 0
        assert oracle_lib.ironav_set_learned(None, None, None, 0, None) != 0
        assert oracle_lib.ironav_set_learned(st.ctx, None, None, 0, None) == 0
    finally:
        st.close()


def test_class_fallback_is_the_plain_search(oracle_lib):
    """Proposals whose class is never P_Skip or 16x16 hand every macroblock to the plain search: the stream is
    the plain stream, byte for byte, and only the class-fallback counter moves."""
    seq = Sequence.config("cif", 4)
    plain, _, _ = _encode_host(oracle_lib, seq, 4, qp=27)
    got, _, stats = _encode_host(oracle_lib, seq, 4, proposals={"classes": (2, 3, 4)}, qp=27)
    assert got == plain
    assert stats[0] == 0 and stats[2] == 0 and stats[1] > 0


@pytest.mark.parametrize("margin", [0, 64])
def test_judged_streams_decode(oracle_lib, margin, tmp_path):
    """Judged macroblocks are coded like searched ones: FFmpeg decodes the stream to the reconstruction; every
    searched macroblock falls in one counter, and the judge takes a share of them."""
    seq = Sequence.config("cif", 5)
    plain, _, _ = _encode_host(oracle_lib, seq, 5, qp=27)
    got, recons, stats = _encode_host(oracle_lib, seq, 5, proposals={}, margin=margin, qp=27)
    check_stream_decodes_to(str(tmp_path), f"learned_m{margin}", b"".join(got), recons, 352, 288)
    assert stats[0] > 0 and stats[1] > 0
    assert got[0] == plain[0]  # the IDR picture has no P analysis
    print(f"margin {margin}: judged {stats[0]}, class fallbacks {stats[1]}, cost fallbacks {stats[2]}; "
          f"{sum(map(len, got))} bytes against the plain {sum(map(len, plain))}")


# ---- GPU: the library's judge against the oracle's -----------------------------------------------------

def _run_pair(oracle_lib, name, frames, size=None, margin=0, classes=(0, 1, 1, 1, 2, 3, 4), **kw):
    import os

    seq = Sequence.config(name, frames, size=size)
    w, h = seq.width, seq.height
    ref = Encoder(w, h, lib=oracle_lib, **kw)
    oracle_lib.oracle_set_threads(ref.st.ctx, os.cpu_count() or 1)
    gpu = DeviceEncoder(w, h, **kw)
    hp = HostProposals(ref, seq, seed=11, margin=margin, classes=classes)
    dp = DeviceProposals(gpu, seq, seed=11, margin=margin, classes=classes)
    stream, recons = [], []
    try:
        for t in range(frames):
            y = seq.frame(t)
            cb, cr = seq.chroma(t)
            want = ref.encode(y, cb, cr)
            got = gpu.encode(y, cb, cr)
            if got != want:
                codes = gpu.codes()
                bad = [k for k in range(len(codes)) if codes[k].tobytes() != ref.codes[k].tobytes()]
                raise AssertionError(f"{name} picture {t}: {len(bad)} macroblock codes differ from the oracle's, first {bad[:5]}")
            stream.append(got)
            recons.append(tuple(a.copy() for a in ref.recon))
        assert np.array_equal(gpu.states(), ref.states)
        for a, b in zip(gpu.recon(), ref.recon):
            assert np.array_equal(a, b)
        assert np.array_equal(dp.counters(), hp.stats), (dp.counters(), hp.stats)
    finally:
        gpu.close()
        ref.close()
    return b"".join(stream), recons, hp.stats.copy()


@pytest.mark.gpu
@pytest.mark.parametrize("margin", [0, 48])
def test_decide_mode_judge_matches_the_oracle_cif(oracle_lib, margin, tmp_path):
    """CIF, 8 pictures, QP 27, two slice bands: the device encoder with proposals against the oracle's."""
    stream, recons, stats = _run_pair(oracle_lib, "cif", 8, margin=margin, qp=27, keyint=30, nslices=2)
    check_stream_decodes_to(str(tmp_path), f"learned_gpu_m{margin}", stream, recons, 352, 288)
    assert stats[0] > 0 and stats[1] > 0
    print(f"margin {margin}: judged {stats[0]}, class fallbacks {stats[1]}, cost fallbacks {stats[2]}")


@pytest.mark.gpu
def test_decide_mode_judge_matches_the_oracle_1080p(oracle_lib):
    """1920x1080, an IDR picture and 3 P pictures at QP 22 with eight bands; fast mode on a cropped picture."""
    _run_pair(oracle_lib, "1080p", 4, qp=22, keyint=60, nslices=8)
    _run_pair(oracle_lib, "1080p", 4, size=(170, 102), qp=34, keyint=60, nslices=2, fast=True)


@pytest.mark.gpu
def test_auto_mode_judge_matches_the_oracle(oracle_lib, cuda_lib):
    """Auto mode (the analysis alone, ironav_analyse_auto) with proposals: every result record and counter."""
    import torch

    from ironav_b200.inter import InterStage

    seq = Sequence.config("1080p", 3, size=(640, 368))
    a = InterStage(640, 368, lib=oracle_lib)
    b = InterStage(640, 368, lib=cuda_lib)
    try:
        cands, cls = make_proposals(seq, 1, a.mb_w, a.mb_h, seed=3)
        sa = np.zeros(3, dtype=np.uint32)
        assert oracle_lib.ironav_set_learned(a.ctx, cands.ctypes.data, cls.ctypes.data, 16, sa.ctypes.data) == 0
        dc, dk = torch.from_numpy(cands).cuda(), torch.from_numpy(cls).cuda()
        sb = torch.zeros(3, dtype=torch.int32, device="cuda")
        assert cuda_lib.ironav_set_learned(b.ctx, dc.data_ptr(), dk.data_ptr(), 16, sb.data_ptr()) == 0
        for st in (a, b):
            st.push_reference(seq.frame(0))
            st.set_source(seq.frame(1))
            st.begin_p_picture(27 + 0, nrefs_active=1)
        ra, _ = a.analyse_auto()
        rb, _ = b.analyse_auto()
        assert ra.tobytes() == rb.tobytes()
        torch.cuda.synchronize()
        assert np.array_equal(sb.cpu().numpy().astype(np.uint32), sa)
        assert sa[0] > 0
    finally:
        a.close()
        b.close()


@pytest.mark.gpu
def test_trained_proposer_inside_the_encoder(tmp_path):
    """The network end to end on a small case: training data from the plain search, a few hundred Adam steps,
    then the device encoder with the learned form: its stream decodes under FFmpeg to its reconstruction, the
    judge takes macroblocks, and the training loss went down."""
    from ironav_b200 import learned
    from ironav_b200.proposer import Proposer

    data = learned.TrainingSet().collect(sequences=1, frames=5, qps=(27,), size=(320, 192))
    assert len(data) > 500
    prop = Proposer(max_batch=256)
    hist = learned.train(prop, data, samples=256 * 200, batch=256, lr=1e-3, log_every=50)
    assert hist[0]["step"] == 1
    assert hist[-1]["mv_loss"] + hist[-1]["part_loss"] < 0.7 * (hist[0]["mv_loss"] + hist[0]["part_loss"]), hist
    seq = Sequence.config("1080p", 5, seed=learned.TRAIN_SEED + 99, size=(320, 192))
    enc = DeviceEncoder(320, 192, 27)
    judge = learned.LearnedJudge(prop, enc, margin=0)
    stream, recons = [], []
    try:
        for t in range(5):
            cb, cr = seq.chroma(t)
            stream.append(enc.encode(seq.frame(t), cb, cr))
            recons.append(tuple(a.copy() for a in enc.recon()))
        c = judge.counters()
    finally:
        enc.close()
    check_stream_decodes_to(str(tmp_path), "learned_net", b"".join(stream), recons, 320, 192)
    assert c["judged"] + c["class_fallback"] + c["cost_fallback"] > 0
    print(hist[0], hist[-1], c)
