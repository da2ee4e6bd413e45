"""Extracts the deblocking filter's tables from the reference into tests/golden/deblock_tables.json (run
from the repository root with the root of a checkout of the reference as the argument:
`python -m tests.golden.make_deblock_tables <reference-root>`).

The tables are the standard's (ITU-T H.264 Tables 8-15 to 8-17) as the reference holds them: ALPHA, BETA
and TC0 of crates/ironav-codec/src/h264/tables.rs (indexed by indexA / indexB, and indexA x bS), and
CHROMA_QP of crates/ironav-codec/src/h264/mb.rs:211 (QPc for qPi 30..51). The fixture lets the tests pin
the oracle's copies without the reference present.
"""
from __future__ import annotations

import ast
import json
import os
import re
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
# the H.264 module within the reference's tree
H264 = os.path.join("crates", "ironav-codec", "src", "h264")


def _const(text: str, name: str):
    m = re.search(r"const " + name + r": \[[^=]*= (\[.*?\]);", text, re.S)
    if not m:
        raise ValueError(f"{name} not found")
    return ast.literal_eval(m.group(1))


def main(reference_root: str) -> None:
    src = os.path.join(reference_root, H264)
    tables = open(os.path.join(src, "tables.rs")).read()
    mb = open(os.path.join(src, "mb.rs")).read()
    out = {
        "alpha": _const(tables, "ALPHA"),
        "beta": _const(tables, "BETA"),
        "tc0": _const(tables, "TC0"),
        "chroma_qp": _const(mb, "CHROMA_QP"),
        "source": "crates/ironav-codec/src/h264/tables.rs (ALPHA, BETA, TC0), crates/ironav-codec/src/h264/mb.rs:211 (CHROMA_QP)",
    }
    with open(os.path.join(HERE, "deblock_tables.json"), "w") as f:
        json.dump(out, f)
        f.write("\n")


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit("usage: python -m tests.golden.make_deblock_tables <reference-root>")
    main(sys.argv[1])
