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
