"""A reader of CAVLC residual blocks and Exp-Golomb codes written from ITU-T H.264 9.1 and 9.2 (test
infrastructure): it parses what the oracle's writer writes, as the reference's writer tests parse theirs with
the reference decoder's residual_block (crates/ironav-codec/src/h264/enc/cavlc.rs:124-179)."""
from __future__ import annotations

import json
import os

HERE = os.path.dirname(os.path.abspath(__file__))


def tables() -> dict:
    with open(os.path.join(HERE, "golden", "cavlc_tables.json")) as f:
        return json.load(f)


class BitReader:
    def __init__(self, data: bytes):
        self.data, self.pos = data, 0

    def bit(self) -> int:
        b = (self.data[self.pos >> 3] >> (7 - (self.pos & 7))) & 1
        self.pos += 1
        return b

    def bits(self, n: int) -> int:
        v = 0
        for _ in range(n):
            v = (v << 1) | self.bit()
        return v

    def ue(self) -> int:
        z = 0
        while self.bit() == 0:
            z += 1
        return (1 << z) - 1 + self.bits(z)

    def se(self) -> int:
        k = self.ue()
        return (k + 1) // 2 if k & 1 else -(k // 2)


def _vlc(r: BitReader, lens, codes) -> int:
    """The index of the variable-length code (lens[i] bits, value codes[i]) that the next bits hold."""
    table = {(n, c): i for i, (n, c) in enumerate(zip(lens, codes)) if n > 0}
    n = code = 0
    while n < 17:
        code = (code << 1) | r.bit()
        n += 1
        if (n, code) in table:
            return table[(n, code)]
    raise ValueError("no code matches")


def residual_block(r: BitReader, nc: int, max_coeff: int, T: dict) -> list[int]:
    """residual_block_cavlc (7.3.5.3.2) with the coeff_token, level, total_zeros and run_before semantics of
    9.2.1-9.2.3: the block's levels in scan order."""
    if nc == -1:
        tok = _vlc(r, T["CHROMA_DC_COEFF_TOKEN_LEN"], T["CHROMA_DC_COEFF_TOKEN_BITS"])
    else:
        cls = 0 if nc < 2 else 1 if nc < 4 else 2 if nc < 8 else 3
        tok = _vlc(r, T["COEFF_TOKEN_LEN"][cls], T["COEFF_TOKEN_BITS"][cls])
    total, ones = tok // 4, tok % 4
    out = [0] * max_coeff
    if total == 0:
        return out
    levels = []
    for _ in range(ones):
        levels.append(-1 if r.bit() else 1)
    suffix_len = 1 if total > 10 and ones < 3 else 0
    for i in range(ones, total):
        prefix = 0
        while r.bit() == 0:
            prefix += 1
        size = 4 if (prefix == 14 and suffix_len == 0) else (prefix - 3 if prefix >= 15 else suffix_len)
        code = (min(15, prefix) << suffix_len) + (r.bits(size) if size > 0 else 0)
        if prefix >= 15 and suffix_len == 0:
            code += 15
        if prefix >= 16:
            code += (1 << (prefix - 3)) - 4096
        if i == ones and ones < 3:
            code += 2
        val = (code + 2) >> 1 if code % 2 == 0 else (-code - 1) >> 1
        levels.append(val)
        if suffix_len == 0:
            suffix_len = 1
        if abs(val) > (3 << (suffix_len - 1)) and suffix_len < 6:
            suffix_len += 1
    zeros_left = 0
    if total < max_coeff:
        if nc == -1:
            zeros_left = _vlc(r, T["CHROMA_DC_TOTAL_ZEROS_LEN"][total - 1], T["CHROMA_DC_TOTAL_ZEROS_BITS"][total - 1])
        else:
            zeros_left = _vlc(r, T["TOTAL_ZEROS_LEN"][total - 1], T["TOTAL_ZEROS_BITS"][total - 1])
    runs = []
    for i in range(total - 1):
        run = 0
        if zeros_left > 0:
            zl = min(zeros_left, 7)
            run = _vlc(r, T["RUN_LEN"][zl - 1], T["RUN_BITS"][zl - 1])
        runs.append(run)
        zeros_left -= run
    runs.append(zeros_left)
    pos = -1
    for i in range(total - 1, -1, -1):
        pos += runs[i] + 1
        out[pos] = levels[i]
    return out
