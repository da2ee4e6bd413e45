"""A CABAC arithmetic decoder written from ITU-T H.264 9.3.1.2 and 9.3.3.2 (test infrastructure): it reads
back what the oracle's coder writes, as the reference's coder test reads its own with the reference
decoder (bins_read_back_through_the_decoder, crates/ironav-codec/src/h264/enc/cabac.rs:252-291). The
tables come from tests/golden/cabac_tables.json."""
from __future__ import annotations

import json
import os

HERE = os.path.dirname(os.path.abspath(__file__))


def tables() -> dict:
    with open(os.path.join(HERE, "golden", "cabac_tables.json")) as f:
        return json.load(f)


def init_states(T: dict, intra: bool, idc: int, qp: int) -> list[tuple[int, int]]:
    """(pStateIdx, valMPS) per ctxIdx (9.3.1.1)."""
    qp = min(max(qp, 0), 51)
    mn = T["CABAC_INIT_I"] if intra else T["CABAC_INIT_PB"][idc]
    out = []
    for m, n in mn:
        pre = min(max(((m * qp) >> 4) + n, 1), 126)
        out.append((63 - pre, 0) if pre <= 63 else (pre - 64, 1))
    return out


class Decoder:
    """The arithmetic decoding engine on slice data starting at byte `start`."""

    def __init__(self, data: bytes, start: int, T: dict, intra: bool, idc: int, qp: int):
        self.data, self.pos, self.T = data, start * 8, T
        self.st = init_states(T, intra, idc, qp)
        self.range = 510
        self.offset = self.bits(9)

    def bit(self) -> int:
        i = self.pos >> 3
        b = (self.data[i] >> (7 - (self.pos & 7))) & 1 if i < len(self.data) else 0
        self.pos += 1
        return b

    def bits(self, n: int) -> int:
        v = 0
        for _ in range(n):
            v = (v << 1) | self.bit()
        return v

    def _renorm(self) -> None:
        while self.range < 256:
            self.range <<= 1
            self.offset = (self.offset << 1) | self.bit()

    def decision(self, ctx: int) -> int:
        p, mps = self.st[ctx]
        lps = self.T["LPS_RANGE"][p][(self.range >> 6) & 3]
        self.range -= lps
        if self.offset >= self.range:
            b = 1 - mps
            self.offset -= self.range
            self.range = lps
            self.st[ctx] = (self.T["TRANS_LPS"][p], 1 - mps if p == 0 else mps)
        else:
            b = mps
            self.st[ctx] = (min(p + 1, 62), mps)
        self._renorm()
        return b

    def bypass(self) -> int:
        self.offset = (self.offset << 1) | self.bit()
        if self.offset >= self.range:
            self.offset -= self.range
            return 1
        return 0

    def terminate(self) -> int:
        self.range -= 2
        if self.offset >= self.range:
            return 1
        self._renorm()
        return 0
