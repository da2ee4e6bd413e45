"""High profile with CABAC on the device against the oracle, bit for bit: whole sequences through the device
pipeline (decide mode's rate-distortion decision, decide_rd_kernel, for the IDR and P pictures; the CABAC
slices written from the codes in device memory, cabac_write_kernel; the filter's records, the deblocking
filter and the new reference), each picture's Annex B bytes, codes, states and reconstruction equal to the
oracle's chain (decide_rd, enc/frame.rs:1462-1513; write_mb_cabac, 2020-2279; CabacWriter / CabacCost,
enc/cabac.rs:42-192), and the GPU's streams decoded by FFmpeg to its reconstructions."""
from __future__ import annotations

import pytest

from ironav_b200.encoder import Encoder
from ironav_b200.synth import Sequence
from tests.stream_util import check_stream_decodes_to
from tests.test_chain_gpu import _run_pair

pytestmark = pytest.mark.gpu


def test_cif_high_chain(oracle_lib, tmp_path):
    """CIF, an IDR picture and 11 P pictures at QP 26, one reference, two slice bands, CABAC with the 8x8
    transform (Intra8x8 and inter 8x8 candidates)."""
    stream, recons, _ = _run_pair(oracle_lib, "cif", 12, qp=26, keyint=30, refs=1, nslices=2, cabac=True)
    check_stream_decodes_to(str(tmp_path), "cif_high_gpu", stream, recons, 352, 288)


@pytest.mark.parametrize("qp", [22, 27, 32])
def test_1080p_high_pictures(oracle_lib, qp, tmp_path):
    """1920x1080, an IDR picture and 2 P pictures at QP 22, 27 and 32, eight slice bands."""
    stream, recons, _ = _run_pair(oracle_lib, "1080p", 3, qp=qp, keyint=120, refs=1, nslices=8, check_every=False, cabac=True)
    check_stream_decodes_to(str(tmp_path), f"1080p_high_qp{qp}", stream, recons, 1920, 1080)


def test_references_sub_partitions_and_idr_pictures_under_cabac(oracle_lib, tmp_path):
    """Three references at QP 18 with sub-partitions (ref_idx and sub_mb_type bins, no 8x8 transform on split
    blocks), an IDR picture every four pictures, three bands."""
    stream, recons, _ = _run_pair(oracle_lib, "cif", 10, size=(176, 144), qp=18, keyint=4, refs=3, nslices=3, sub8=True, cabac=True)
    check_stream_decodes_to(str(tmp_path), "qcif_cabac_gpu", stream, recons, 176, 144)


def test_main_profile_and_live_coding_under_cabac(oracle_lib, tmp_path):
    """CABAC without the 8x8 transform (Main) with live coding's P_Skip test, on a cropped picture."""
    stream, recons, _ = _run_pair(oracle_lib, "1080p", 6, size=(170, 102), qp=34, keyint=30, refs=1, nslices=2, fast=True, cabac=True,
                                  transform8=False)
    check_stream_decodes_to(str(tmp_path), "main_fast_gpu", stream, recons, 170, 102)


def test_ten_bit_high10_cabac_chain(oracle_lib):
    """High 10 with CABAC and the 8x8 transform: 10-bit pictures (the stream's bytes against the oracle's)."""
    _run_pair(oracle_lib, "cif", 5, qp=26, keyint=30, refs=2, nslices=2, bd=10, cabac=True)


def test_host_forms_write_the_same_cabac_stream(oracle_lib, cuda_lib):
    """The host-buffer entry points (ironav_decide_*_picture, ironav_write_slices) under CABAC."""
    seq = Sequence.config("cif", 4)
    a = Encoder(352, 288, qp=30, keyint=30, nslices=3, refs=2, lib=oracle_lib, cabac=True)
    b = Encoder(352, 288, qp=30, keyint=30, nslices=3, refs=2, lib=cuda_lib, cabac=True)
    for t in range(4):
        f = (seq.frame(t), *seq.chroma(t))
        assert a.encode(*f) == b.encode(*f), f"picture {t}"
    a.close()
    b.close()


@pytest.mark.parametrize("bd", [8, 10])
def test_batched_cabac_decide_matches_single_streams_and_the_oracle(oracle_lib, cuda_lib, bd):
    """Four streams of different sizes, slice layouts, references and content decided under CABAC in one launch
    (every stream's slice bands as chains, decide_rd_batch_kernel): each stream's codes, states and
    reconstruction are those of its own decide call, and the oracle's."""
    import numpy as np
    import torch

    from ironav_b200.inter import MBCODE_DTYPE, MBSTATE_DTYPE, InterBatch
    from tests.test_decide import _same_decisions, decide_case

    cases = [dict(), dict(new_content=True, qp=30), dict(size=(320, 176), nslices=3, fast=True, refs=2), dict(cfg="1080p", nslices=8, qp=27)]
    cases = [dict(kw, bd=bd) for kw in cases]
    stages = []
    for kw in cases:
        st = decide_case(cuda_lib, threads=False, **kw)[0]
        st.set_entropy(True, True)
        stages.append(st)
    want = [st.decide_p_picture() for st in stages]
    for k in (1, 2):
        o = decide_case(oracle_lib, **cases[k])[0]
        o.set_entropy(True, True)
        _same_decisions(want[k], o.decide_p_picture(), f"single stream {cases[k]} against the oracle")
        o.close()
    stream = torch.cuda.Stream()
    for st in stages:
        st.set_stream(stream.cuda_stream)
    dt = torch.uint8 if bd == 8 else torch.int16
    bufs = [(torch.zeros(st.nmb * 72, dtype=torch.uint8, device="cuda"), torch.full((st.nmb * 1516,), 0x5A, dtype=torch.uint8, device="cuda"),
             torch.zeros((st.mb_h * 16, st.mb_w * 16), dtype=dt, device="cuda"), torch.zeros((2, st.mb_h * 8, st.mb_w * 8), dtype=dt, device="cuda"))
            for st in stages]
    batch = InterBatch(stages)
    for _ in range(2):
        batch.decide([b[0].data_ptr() for b in bufs], [b[1].data_ptr() for b in bufs], [b[2].data_ptr() for b in bufs],
                     [b[2].shape[1] for b in bufs], [b[3][0].data_ptr() for b in bufs], [b[3][1].data_ptr() for b in bufs],
                     [b[3].shape[2] for b in bufs])
        batch.sync()
    view = (lambda t: t.cpu().numpy().view(np.uint16)) if bd == 10 else (lambda t: t.cpu().numpy())
    for k, (st, b) in enumerate(zip(stages, bufs)):
        got = (b[0].cpu().numpy().view(MBSTATE_DTYPE), b[1].cpu().numpy().view(MBCODE_DTYPE), (view(b[2]), view(b[3][0]), view(b[3][1])))
        _same_decisions(got, want[k], f"stream {k} {cases[k]}")
    batch.close()
    for st in stages:
        st.close()
