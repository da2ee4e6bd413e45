"""High profile with CABAC (the reference encoder's default entropy coding) in the oracle, on the CPU.

- both copies of the CABAC tables (oracle and CUDA headers) hold the fixture extracted from the reference;
- the arithmetic coder reads back through a decoder written from the standard (tests/cabac_reader.py) on
  the reference's own test recipe (bins_read_back_through_the_decoder, crates/ironav-codec/src/h264/enc/
  cabac.rs:252-291: 20000 seeded decisions, bypass bins and terminating zeros), and the decoder's last bit
  read is the rbsp_stop_one_bit of the flush;
- the bit counter (CabacCost, enc/cabac.rs:150-192) charges what the entropy of each context state says;
- the SPS and PPS declare Main or High with CABAC and the 8x8 transform (enc/mod.rs:296-400);
- whole IPPP sequences decided by rate-distortion cost (decide_rd, enc/frame.rs:1462-1513) and written with
  CABAC (write_mb_cabac, enc/frame.rs:2020-2279) decode under FFmpeg to the oracle's reconstruction, as the
  reference's decoder_rebuilds_the_encoders_reference family asserts for its CABAC modes (enc/mod.rs:860-873):
  every macroblock type the decision reaches (Intra4x4, Intra8x8, Intra16x16, P_Skip, the four
  partitionings with either transform, sub-partitions, several references) coded as it was reconstructed.
"""
from __future__ import annotations

import ctypes
import json
import math
import os
import re
from collections import Counter

import numpy as np
import pytest

from tests.cabac_reader import Decoder, tables
from tests.stream_util import check_stream_decodes_to
from tests.test_stream import _sps_head, encode_sequence

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _hooks(lib):
    lib.oracle_cabac_ops.argtypes = [ctypes.c_void_p] * 3 + [ctypes.c_int] * 4 + [ctypes.c_void_p, ctypes.c_int]
    lib.oracle_cabac_cost.argtypes = [ctypes.c_void_p] * 3 + [ctypes.c_int] * 4
    lib.oracle_cabac_cost.restype = ctypes.c_uint32
    return lib


def _reference_ops(n: int = 20000):
    """The reference test's bins: an LCG from seed 4321, kinds [decision x3, bypass, terminate 0], contexts
    multiples of 37, values skewed by context parity so that the contexts adapt (enc/cabac.rs:256-270)."""
    seed = 4321

    def rnd(m: int) -> int:
        nonlocal seed
        seed = (seed * 1103515245 + 12345) & 0xFFFFFFFF
        return (seed >> 16) % m

    ops = []
    for _ in range(n):
        kind = [0, 0, 0, 1, 2][rnd(5)]
        ctx = rnd(8) * 37
        ops.append((kind, ctx, int(rnd(10) < (2 if ctx % 2 == 0 else 8))))
    return ops


def _arrays(ops):
    return [np.ascontiguousarray([o[i] for o in ops], dtype=np.int32) for i in range(3)]


def test_both_headers_hold_the_fixture_tables():
    fixture = tables()
    for path in ("oracle/cabac_tables.h", "ironav_b200/csrc/cabac_tables.cuh"):
        text = open(os.path.join(ROOT, path)).read()
        got = {m.group(1): json.loads(m.group(2).replace("{", "[").replace("}", "]"))
               for m in re.finditer(r"int\d+_t (\w+)(?:\[\d+\])+ = (\{.*?\});", text)}
        for name, v in fixture.items():
            if name != "source":
                assert got[name] == v, f"{path}: {name} differs from tests/golden/cabac_tables.json"
    assert len(fixture["CABAC_INIT_I"]) == 1024 and len(fixture["CABAC_INIT_PB"]) == 3


def test_bins_read_back_through_a_decoder_of_the_standard(oracle_lib):
    lib = _hooks(oracle_lib)
    ops = _reference_ops()
    k, c, v = _arrays(ops)
    out = np.zeros(1 << 16, dtype=np.uint8)
    n = lib.oracle_cabac_ops(k.ctypes.data, c.ctypes.data, v.ctypes.data, len(ops), 0, 1, 30, out.ctypes.data, len(out))
    assert n > 0
    data = bytes(out[:n])
    assert data[0] == 0b10110111  # the header bits and cabac_alignment_one_bit
    d = Decoder(data, 1, tables(), False, 1, 30)
    for i, (kind, ctx, val) in enumerate(ops):
        got = d.decision(ctx) if kind == 0 else d.bypass() if kind == 1 else d.terminate()
        assert got == (0 if kind == 2 else val), f"bin {i}"
    assert d.terminate() == 1
    bits = "".join(f"{b:08b}" for b in data)
    # the flush ends the data: the last bit the decoder reads is the rbsp_stop_one_bit, zeros follow
    assert d.pos == bits.rindex("1") + 1 and len(bits) - d.pos < 8


def test_the_counter_charges_the_entropy_of_each_state(oracle_lib):
    """CabacCost: -log2 of the MPS / LPS probability of the context's state (pLPS = 0.5 * (0.01875/0.5)^(p/63),
    9.3.1.1), rounded to 1/256 bit, 1 bit a bypass bin, 1/256 bit a terminating 0; the contexts adapt as the
    coder's do."""
    lib = _hooks(oracle_lib)
    T = tables()
    ops = _reference_ops(3000)
    k, c, v = _arrays(ops)
    got = lib.oracle_cabac_cost(k.ctypes.data, c.ctypes.data, v.ctypes.data, len(ops), 0, 1, 30)
    from tests.cabac_reader import init_states

    st = init_states(T, False, 1, 30)
    want = 0
    for kind, ctx, val in ops:
        if kind == 1:
            want += 256
        elif kind == 2:
            want += 1
        else:
            p, mps = st[ctx]
            lps = 0.5 * (0.01875 / 0.5) ** (p / 63.0)
            want += round(-math.log2(lps if val != mps else 1.0 - lps) * 256.0)
            st[ctx] = ((T["TRANS_LPS"][p], 1 - mps if p == 0 else mps) if val != mps else (min(p + 1, 62), mps))
    assert got == want


@pytest.mark.parametrize("cabac,t8,profile", [(True, True, 100), (True, False, 77)])
def test_parameter_sets_declare_the_profile_and_the_8x8_transform(oracle_lib, cabac, t8, profile):
    from ironav_b200.inter import write_parameter_sets

    data = write_parameter_sets(1920, 1080, 8, (30, 1), 3, lib=oracle_lib, cabac=cabac, transform8=t8)
    assert _sps_head(data)[0] == profile and _sps_head(data)[2] == 40
    from tests.cavlc_reader import BitReader

    at = next(i for i in range(len(data) - 3) if data[i:i + 3] == b"\0\0\1" and data[i + 3] & 31 == 8)
    r = BitReader(data[at + 4:])
    assert (r.ue(), r.ue(), r.bit()) == (0, 0, 1)  # pps id, sps id, entropy_coding_mode_flag
    r.bit(), r.ue(), r.ue(), r.ue(), r.bit(), r.bits(2), r.se(), r.se(), r.se(), r.bit(), r.bit(), r.bit()
    if t8:
        assert (r.bit(), r.bit(), r.se()) == (1, 0, 0)  # transform_8x8_mode_flag, no scaling matrix, offset 0
    assert r.bit() == 1  # rbsp_stop_one_bit
    # 10-bit streams stay High 10 whatever the entropy coding
    assert _sps_head(write_parameter_sets(352, 288, 10, (30, 1), 1, lib=oracle_lib, cabac=True, transform8=t8))[0] == 110


def _kinds(codes) -> Counter:
    h = Counter()
    for k, skip, t8, part, sub, refs in zip(codes["kind"], codes["skip"], codes["res"]["t8x8"], codes["part"], codes["sub"],
                                             codes["refs"]):
        if k != 5:
            h[{1: "I4", 2: "I8", 3: "I16"}[int(k)]] += 1
        elif skip:
            h["skip"] += 1
        else:
            h[f"P{part}" + ("t8" if t8 else "")] += 1
            h["sub"] += int(part == 3 and sub.any())
            h["ref>0"] += int(refs.any())
    return h


def _encode(lib, name, frames, w, h, **kw):
    from ironav_b200.encoder import Encoder
    from ironav_b200.synth import Sequence

    seq = Sequence.config(name, frames, size=(w, h))
    enc = Encoder(seq.width, seq.height, lib=lib, cabac=True, **kw)
    lib.oracle_set_threads(enc.st.ctx, os.cpu_count() or 1)
    data, recons, hist, psnr = [], [], Counter(), []
    for t in range(frames):
        y = seq.frame(t)
        data.append(enc.encode(y, *seq.chroma(t)))
        recons.append(tuple(a.copy() for a in enc.recon))
        hist += _kinds(enc.codes)
        mse = np.mean((enc.recon[0][:h, :w].astype(np.float64) - y.astype(np.float64)) ** 2)
        psnr.append(10 * math.log10(255.0 ** 2 / max(mse, 1e-9)))
    kinds = "".join(enc.loop.kinds)
    enc.close()
    return b"".join(data), recons, kinds, hist, psnr


def test_config0_in_high_decodes_to_the_oracles_reconstruction(oracle_lib, tmp_path):
    """CIF, 30 pictures IPPP at QP 26 (the IDR picture at 23), one reference, two slice bands, CABAC with the
    8x8 transform: FFmpeg decodes every picture to the oracle's reconstruction."""
    stream, recons, kinds, hist, psnr = _encode(oracle_lib, "cif", 30, 352, 288, qp=26, keyint=30, refs=1, nslices=2)
    assert kinds == "I" + "P" * 29
    for k in ("I8", "I16", "skip", "P0", "P0t8"):
        assert hist[k] > 0, (k, hist)
    assert min(psnr) > 30.0, psnr
    check_stream_decodes_to(str(tmp_path), "cif_high", stream, recons, 352, 288)


def test_references_sub_partitions_and_idr_pictures_under_cabac(oracle_lib, tmp_path):
    """176x144 at QP 18: three references (ref_idx with its unary contexts), sub-partitions (sub_mb_type, no
    8x8 transform on split blocks), every partitioning with both transforms, Intra4x4 and Intra8x8, an IDR
    picture every four, three slice bands."""
    stream, recons, kinds, hist, _ = _encode(oracle_lib, "cif", 10, 176, 144, qp=18, keyint=4, refs=3, nslices=3, sub8=True)
    assert kinds == "IPPPIPPPIP"
    for k in ("I8", "I16", "skip", "P0", "P0t8", "P1", "P1t8", "P2", "P2t8", "sub", "ref>0"):
        assert hist[k] > 0, (k, hist)
    check_stream_decodes_to(str(tmp_path), "qcif_cabac_3refs", stream, recons, 176, 144)


def test_main_profile_live_coding_and_odd_sizes_under_cabac(oracle_lib, tmp_path):
    """CABAC without the 8x8 transform (Main), live coding's P_Skip test, a picture that is not a whole
    number of macroblocks, and a coarse quantiser."""
    stream, recons, _, hist, _ = _encode(oracle_lib, "1080p", 6, 170, 102, qp=34, keyint=30, refs=1, nslices=2, fast=True,
                                         transform8=False)
    assert hist["I8"] == 0 and hist["P0t8"] == 0
    check_stream_decodes_to(str(tmp_path), "main_fast_odd", stream, recons, 170, 102)
    stream, recons, _, hist, _ = _encode(oracle_lib, "1080p", 8, 320, 176, qp=32, keyint=30, refs=2, nslices=2)
    assert hist["I4"] > 0 and hist["I8"] > 0
    check_stream_decodes_to(str(tmp_path), "high_2refs", stream, recons, 320, 176)


def test_a_planted_decision_error_is_seen(oracle_lib, tmp_path):
    """The check is not blind to the decisions: a reconstruction whose one macroblock is predicted from another
    vector than the one coded (here: one luma sample changed) no longer matches what FFmpeg decodes."""
    stream, recons, _, _, _ = _encode(oracle_lib, "cif", 3, 96, 64, qp=26, keyint=30, refs=1, nslices=1)
    y, cb, cr = (a.copy() for a in recons[2])
    y[17, 33] = (int(y[17, 33]) + 1) % 256
    recons[2] = (y, cb, cr)
    with pytest.raises(AssertionError, match="luma differs"):
        check_stream_decodes_to(str(tmp_path), "planted_cabac", stream, recons, 96, 64)


def test_the_cuda_library_writes_the_oracles_high_parameter_sets(oracle_lib):
    from ironav_b200.inter import cuda_library, write_parameter_sets

    cuda = cuda_library()
    for args in ((352, 288, 8, (30, 1), 1), (1920, 1080, 8, (30, 1), 3), (200, 120, 10, (30000, 1001), 2)):
        for cabac, t8 in ((True, True), (True, False)):
            assert write_parameter_sets(*args, lib=cuda, cabac=cabac, transform8=t8) == \
                write_parameter_sets(*args, lib=oracle_lib, cabac=cabac, transform8=t8), (args, cabac, t8)
