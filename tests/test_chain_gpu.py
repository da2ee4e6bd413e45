"""Whole sequences through the device pipeline against the oracle's chain, bit for bit, on the configurations
the stage is specified on: every picture goes scene-cut measure -> decide mode (ironav_decide_i_picture_device
for the IDR picture, ironav_decide_p_picture_device after it) -> the slices written on the device from the
codes (ironav_write_slices_device) -> ironav_decide_dbk_records_device -> ironav_deblock_picture_device ->
ironav_push_reference_device / ironav_push_reference_chroma_device of the filtered reconstruction, which the
next picture predicts from (code_picture and the reference list, crates/ironav-codec/src/h264/enc/mod.rs:
539-670; run_refs, 787-827). Each picture's Annex B bytes, codes, states and filtered reconstruction must
equal the oracle's; errors would accumulate through the chain, so equality at the last picture covers the
whole pipeline. The GPU's streams also decode under FFmpeg to its reconstructions (stream_util)."""
from __future__ import annotations

import os

import numpy as np
import pytest

from ironav_b200.encoder import DeviceEncoder, Encoder
from ironav_b200.synth import Sequence
from tests.stream_util import check_stream_decodes_to

pytestmark = pytest.mark.gpu


def _run_pair(oracle_lib, name, frames, size=None, check_every=True, **kw):
    """Codes the sequence with the oracle (host forms) and with the device pipeline; asserts equality picture
    by picture. Returns the GPU's stream and its reconstructions."""
    seq = Sequence.config(name, frames, size=size)
    w, h = seq.width, seq.height
    ref = Encoder(w, h, lib=oracle_lib, **kw)
    oracle_lib.oracle_set_threads(ref.st.ctx, os.cpu_count() or 1)
    gpu = DeviceEncoder(w, h, **kw)
    stream, recons = [], []
    try:
        for t in range(frames):
            bd = kw.get("bd", 8)
            y = seq.frame10(t) if bd > 8 else seq.frame(t)
            cb, cr = seq.chroma(t, bd=bd)
            want = ref.encode(y, cb, cr)
            got = gpu.encode(y, cb, cr)
            kind = ref.loop.kinds[-1]
            if check_every or t == frames - 1 or got != want:
                codes = gpu.codes()
                for k in range(len(codes)):
                    if codes[k].tobytes() != ref.codes[k].tobytes():
                        raise AssertionError(f"{name} picture {t} ({kind}): macroblock {k}'s code differs from the oracle's")
                assert np.array_equal(gpu.states(), ref.states), f"{name} picture {t} ({kind}): states"
                for c, (a, b) in enumerate(zip(gpu.recon(), ref.recon)):
                    assert np.array_equal(a, b), f"{name} picture {t} ({kind}): reconstruction plane {c}"
            assert got == want, f"{name} picture {t} ({kind}): {len(got)} bytes, the oracle's {len(want)}"
            stream.append(got)
            recons.append(tuple(a.copy() for a in ref.recon))
        assert gpu.loop.kinds == ref.loop.kinds
    finally:
        gpu.close()
        ref.close()
    return b"".join(stream), recons, seq


def test_config0_cif_30_pictures(oracle_lib, tmp_path):
    """CIF 352x288, 30 pictures IPPP, QP 26, one reference, two slice bands."""
    stream, recons, seq = _run_pair(oracle_lib, "cif", 30, qp=26, keyint=30, refs=1, nslices=2)
    check_stream_decodes_to(str(tmp_path), "cif_gpu", stream, recons, 352, 288)
    print(f"config 0: {len(stream)} bytes, FFmpeg decodes the GPU's stream to its reconstruction")


@pytest.mark.parametrize("qp", [22, 27, 32])
def test_config1_1080p_ten_p_pictures(oracle_lib, qp, tmp_path):
    """1920x1080, an IDR picture and 10 P pictures at each of QP 22, 27 and 32, eight slice bands."""
    stream, recons, _ = _run_pair(oracle_lib, "1080p", 11, qp=qp, keyint=120, refs=1, nslices=8, check_every=False)
    check_stream_decodes_to(str(tmp_path), f"1080p_qp{qp}", stream, recons, 1920, 1080)


def test_config2_4k_pictures(oracle_lib, tmp_path):
    """3840x2160, an IDR picture and 4 P pictures at QP 27, sixteen slice bands."""
    stream, recons, _ = _run_pair(oracle_lib, "4k", 5, qp=27, keyint=60, refs=1, nslices=16, check_every=False)
    check_stream_decodes_to(str(tmp_path), "4k_qp27", stream, recons, 3840, 2160)


def test_several_references_and_idr_pictures(oracle_lib, tmp_path):
    """Three references at QP 18 with sub-partitions, an IDR picture every four pictures, three bands."""
    stream, recons, _ = _run_pair(oracle_lib, "cif", 10, size=(176, 144), qp=18, keyint=4, refs=3, nslices=3, sub8=True)
    check_stream_decodes_to(str(tmp_path), "qcif_3refs_gpu", stream, recons, 176, 144)


def test_fast_mode_on_a_cropped_picture(oracle_lib, tmp_path):
    stream, recons, _ = _run_pair(oracle_lib, "1080p", 6, size=(170, 102), qp=34, keyint=30, refs=1, nslices=2, fast=True)
    check_stream_decodes_to(str(tmp_path), "fast_gpu", stream, recons, 170, 102)


def test_ten_bit_chain(oracle_lib):
    """High 10 with CAVLC: 10-bit pictures through the same pipeline (the stream's bytes against the oracle's)."""
    _run_pair(oracle_lib, "cif", 6, qp=26, keyint=30, refs=1, nslices=2, bd=10)


def test_host_forms_write_the_same_stream(oracle_lib, cuda_lib):
    """The host-buffer entry points of the CUDA library (ironav_decide_i_picture, ironav_write_slices, ...)
    through the same encoder loop as the oracle."""
    seq = Sequence.config("cif", 5)
    a = Encoder(352, 288, qp=26, keyint=30, nslices=2, lib=oracle_lib)
    b = Encoder(352, 288, qp=26, keyint=30, nslices=2, lib=cuda_lib)
    for t in range(5):
        f = (seq.frame(t), *seq.chroma(t))
        assert a.encode(*f) == b.encode(*f), f"picture {t}"
    a.close()
    b.close()
