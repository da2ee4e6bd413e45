"""The bitstream: the oracle's CAVLC writer, parameter sets and whole encoded sequences, on the CPU.

- write_block reads back through a CAVLC reader written from the standard, on the reference's own
  random blocks (blocks_read_back_through_the_decoder, crates/ironav-codec/src/h264/enc/cavlc.rs:141-178);
- put_nal inserts emulation prevention bytes as the reference's test vector says
  (emulation_prevention_is_inserted, enc/bitw.rs:137-142);
- the SPS declares Constrained Baseline and the level the reference's tests expect
  (constrained_baseline_live_streams_declare_it_and_decode, the_sps_level_follows_the_picture_size_and_rate,
  enc/mod.rs:1033-1069), from the oracle and from the CUDA library (host code: no GPU needed);
- whole IPPP sequences coded by the oracle decode, under FFmpeg (a decoder that is not this project's), to
  the oracle's reconstruction: the reference's contract "decoder(stream) == encoder reconstruction"
  (decoder_rebuilds_the_encoders_reference and its family, enc/mod.rs:787-967), here on the stage's own
  configurations. This is what pins the oracle's decisions (modes, vectors, partitions, levels) to a third
  party: a wrong decision still decodes, but a decision coded differently from how it was reconstructed
  does not decode to the reconstruction.
"""
from __future__ import annotations

import ctypes
import json
import os
import re

import numpy as np
import pytest

from tests.cavlc_reader import BitReader, residual_block, tables
from tests.stream_util import check_stream_decodes_to

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _header_arrays(path: str) -> dict:
    text = open(path).read()
    out = {}
    for m in re.finditer(r"uint8_t CAVLC_(\w+)((?:\[\d+\])+) = (\{.*?\});", text):
        out[m.group(1)] = json.loads(m.group(3).replace("{", "[").replace("}", "]"))
    return out


def test_both_writers_hold_the_fixture_tables():
    want = tables()
    for path in ("oracle/cavlc_tables.h", "ironav_b200/csrc/cavlc_tables.cuh"):
        got = _header_arrays(os.path.join(ROOT, path))
        for name, v in want.items():
            if name == "source":
                continue
            assert got[name] == v, f"{path}: {name} differs from tests/golden/cavlc_tables.json"


def _write_block(lib, nc, levels):
    lv = np.asarray(levels + [0] * (16 - len(levels)), dtype=np.int32)
    out = np.zeros(4096, dtype=np.uint8)
    nbits = ctypes.c_int(0)
    n = lib.oracle_write_block(nc, lv.ctypes.data, len(levels), out.ctypes.data, len(out), ctypes.byref(nbits))
    return n, bytes(out), nbits.value


def test_blocks_read_back_through_a_reader_of_the_standard(oracle_lib):
    """The reference's writer test on the oracle: its seeded generator (an LCG from 12345), nC in
    {0, 1, 2, 3, 5, 7, 8, 16}, blocks of 16 and 15 levels at every density and four magnitude ranges, chroma DC
    blocks, and its two fixed cases; each block reads back to its levels and leaves the reader where the writer
    stopped."""
    T = tables()
    seed = [12345]

    def rnd(m):
        seed[0] = (seed[0] * 1103515245 + 12345) & 0xFFFFFFFF
        return (seed[0] >> 16) % m

    def round_trip(nc, levels):
        n, data, nbits = _write_block(oracle_lib, nc, levels)
        r = BitReader(data)
        got = residual_block(r, nc, len(levels), T)
        assert got == list(levels), (nc, levels)
        assert r.pos == nbits, f"{levels}: the reader stopped at {r.pos}, the writer at {nbits}"
        assert n == sum(1 for v in levels if v)

    cases = 0
    for nc in (0, 1, 2, 3, 5, 7, 8, 16):
        for ln in (16, 15):
            round_trip(nc, [0] * ln)
            for _ in range(300):
                density = 1 + rnd(16)
                big = rnd(4)
                levels = []
                for _ in range(ln):
                    if rnd(16) >= density:
                        levels.append(0)
                        continue
                    m = (2, 8, 100, 9000)[big]
                    v = 1 + rnd(m)
                    levels.append(v if rnd(2) == 0 else -v)
                round_trip(nc, levels)
                cases += 1
    for _ in range(500):
        round_trip(-1, [rnd(7) - 3 for _ in range(4)])
    round_trip(0, [1, -1, 1] + [0] * 12 + [1])
    round_trip(0, [30000] * 16)
    assert cases == 8 * 2 * 300


def test_emulation_prevention_is_inserted(oracle_lib):
    rbsp = np.array([0, 0, 0, 0, 0, 1, 0, 0, 3, 7], dtype=np.uint8)
    out = np.zeros(64, dtype=np.uint8)
    n = oracle_lib.oracle_put_nal(3, 5, rbsp.ctypes.data, len(rbsp), out.ctypes.data, len(out))
    assert list(out[:n]) == [0, 0, 0, 1, 0x65, 0, 0, 3, 0, 0, 3, 0, 1, 0, 0, 3, 3, 7]


def _sps_head(data: bytes):
    at = next(i for i in range(len(data) - 3) if data[i:i + 3] == b"\0\0\1" and data[i + 3] & 31 == 7)
    return data[at + 4], data[at + 5], data[at + 6]


@pytest.mark.parametrize("which", ["oracle", "cuda"])
def test_sps_declares_constrained_baseline_and_the_level(which, oracle_lib):
    from ironav_b200.inter import cuda_library, write_parameter_sets

    lib = oracle_lib if which == "oracle" else cuda_library()
    head = _sps_head(write_parameter_sets(64, 48, 8, (25, 1), 1, lib=lib))
    assert (head[0], head[1] & 0xC0) == (66, 0xC0)
    for (w, h, fps), level in (((1280, 720, 30), 31), ((1920, 1080, 30), 40), ((1920, 1080, 60), 42), ((2560, 1440, 30), 50),
                               ((3840, 2160, 30), 51)):
        assert _sps_head(write_parameter_sets(w, h, 8, (fps, 1), 1, lib=lib))[2] == level, (w, h, fps)
    assert _sps_head(write_parameter_sets(352, 288, 10, (30, 1), 1, lib=lib))[0] == 110  # High 10 at 10 bits


def test_the_cuda_library_writes_the_oracles_parameter_sets(oracle_lib):
    from ironav_b200.inter import cuda_library, write_parameter_sets

    cuda = cuda_library()
    for args in ((352, 288, 8, (30, 1), 1), (1920, 1080, 8, (30, 1), 1), (3840, 2160, 8, (30, 1), 1), (854, 480, 8, (25, 1), 3),
                 (200, 120, 10, (30000, 1001), 16), (64, 48, 8, (0, 0), 2)):
        assert write_parameter_sets(*args, lib=cuda) == write_parameter_sets(*args, lib=oracle_lib), args


def encode_sequence(lib, name: str, frames: int, width: int | None = None, height: int | None = None, **kw):
    """Codes `frames` pictures of a synthetic configuration with the Encoder over `lib`: (stream, recons)."""
    from ironav_b200.encoder import Encoder
    from ironav_b200.synth import Sequence

    seq = Sequence.config(name, frames, size=(width, height) if width else None)
    enc = Encoder(seq.width, seq.height, lib=lib, **kw)
    if hasattr(lib, "oracle_set_threads"):
        lib.oracle_set_threads(enc.st.ctx, os.cpu_count() or 1)
    data, recons = [], []
    for t in range(frames):
        data.append(enc.encode(seq.frame(t), *seq.chroma(t)))
        recons.append(tuple(a.copy() for a in enc.recon))
    kinds = "".join(enc.loop.kinds)
    enc.close()
    return b"".join(data), recons, kinds, data


def test_config0_stream_from_the_oracle_decodes_to_its_reconstruction(oracle_lib, tmp_path):
    """CIF, 30 pictures IPPP, QP 26 (the IDR picture at 23), one reference, two slice bands: FFmpeg decodes
    every picture to the oracle's reconstruction."""
    stream, recons, kinds, _ = encode_sequence(oracle_lib, "cif", 30, qp=26, keyint=30, refs=1, nslices=2)
    assert kinds == "I" + "P" * 29
    check_stream_decodes_to(str(tmp_path), "cif_qp26", stream, recons, 352, 288)


def test_several_references_sub_partitions_and_idr_pictures_decode(oracle_lib, tmp_path):
    """176x144 at QP 18 (sub-partitions searched), three references (ref_idx coded as ue), an IDR picture every
    four (frame_num and idr_pic_id start again), three slice bands; then two references (ref_idx as one
    inverted bit) at QP 30."""
    stream, recons, kinds, _ = encode_sequence(oracle_lib, "cif", 10, 176, 144, qp=18, keyint=4, refs=3, nslices=3, sub8=True)
    assert kinds == "IPPPIPPPIP"
    check_stream_decodes_to(str(tmp_path), "qcif_3refs", stream, recons, 176, 144)
    stream, recons, kinds, _ = encode_sequence(oracle_lib, "1080p", 6, 208, 112, qp=30, keyint=30, refs=2, nslices=2)
    check_stream_decodes_to(str(tmp_path), "small_2refs", stream, recons, 208, 112)


def test_fast_mode_and_odd_sizes_decode(oracle_lib, tmp_path):
    """Live coding (H264Encoder::realtime's decisions: the fast P_Skip test, flat intra macroblocks left to
    Intra16x16) on a picture that is not a whole number of macroblocks (cropped in the SPS)."""
    stream, recons, _, _ = encode_sequence(oracle_lib, "1080p", 6, 170, 102, qp=34, keyint=30, refs=1, nslices=2, fast=True)
    check_stream_decodes_to(str(tmp_path), "fast_odd", stream, recons, 170, 102)


def test_a_planted_chroma_error_is_seen(oracle_lib, tmp_path):
    """The chroma check through BGR is not blind: one chroma sample of one reconstruction off by one fails it."""
    stream, recons, _, _ = encode_sequence(oracle_lib, "cif", 3, 96, 64, qp=26, keyint=30, refs=1, nslices=1)
    y, cb, cr = (a.copy() for a in recons[1])
    cb[10, 20] = (int(cb[10, 20]) + 1) % 256
    recons[1] = (y, cb, cr)
    with pytest.raises(AssertionError, match="chroma differs"):
        check_stream_decodes_to(str(tmp_path), "planted", stream, recons, 96, 64)
