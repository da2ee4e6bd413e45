"""Extracts the CAVLC code tables from the reference and writes them three ways (run from the repository
root with the root of a checkout of the reference as the argument:
`python -m tests.golden.make_cavlc_tables <reference-root>`):

- tests/golden/cavlc_tables.json: the fixture the CPU tests pin both headers against;
- oracle/cavlc_tables.h: the oracle's copy (plain C arrays);
- ironav_b200/csrc/cavlc_tables.cuh: the CUDA writer's copy (__constant__ arrays).

The tables are the standard's (ITU-T H.264 Table 9-4 codeNum <-> coded_block_pattern for Intra_4x4 and
Inter macroblocks, Table 9-5 coeff_token, Tables 9-7 to 9-9 total_zeros, Table 9-10 run_before) as the
reference holds them in crates/ironav-codec/src/h264/tables.rs: code lengths (*_LEN) and code values
(*_BITS) indexed by the writer's own keys (coeff_token by nC class and 4 * TotalCoeff + TrailingOnes;
total_zeros by TotalCoeff - 1 and total_zeros; run_before by min(zerosLeft, 7) - 1 and run_before).
"""
from __future__ import annotations

import ast
import json
import os
import re
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
H264 = os.path.join("crates", "ironav-codec", "src", "h264")

NAMES = [
    "COEFF_TOKEN_LEN", "COEFF_TOKEN_BITS", "CHROMA_DC_COEFF_TOKEN_LEN", "CHROMA_DC_COEFF_TOKEN_BITS",
    "TOTAL_ZEROS_LEN", "TOTAL_ZEROS_BITS", "CHROMA_DC_TOTAL_ZEROS_LEN", "CHROMA_DC_TOTAL_ZEROS_BITS",
    "RUN_LEN", "RUN_BITS", "GOLOMB_TO_INTRA4X4_CBP", "GOLOMB_TO_INTER_CBP",
]


def _const(text: str, name: str):
    m = re.search(r"const " + name + r": \[[^=]*= (\[.*?\]);", text, re.S)
    if not m:
        raise ValueError(f"{name} not found")
    return ast.literal_eval(m.group(1))


def _dims(v):
    return [len(v)] + (_dims(v[0]) if isinstance(v[0], list) else [])


def _c_init(v) -> str:
    if isinstance(v[0], list):
        return "{" + ", ".join(_c_init(x) for x in v) + "}"
    return "{" + ", ".join(str(x) for x in v) + "}"


def _header(tables: dict, qualifier: str, guard: str, what: str) -> str:
    lines = [
        f"// {what}",
        "// Generated by tests/golden/make_cavlc_tables.py: the CAVLC code tables of ITU-T H.264 (Table 9-4",
        "// codeNum <-> coded_block_pattern, 9-5 coeff_token, 9-7 to 9-9 total_zeros, 9-10 run_before): code",
        "// lengths (*_LEN) and values (*_BITS). coeff_token: [nC class][4 * TotalCoeff + TrailingOnes];",
        "// total_zeros: [TotalCoeff - 1][total_zeros]; run_before: [min(zerosLeft, 7) - 1][run_before].",
        f"#ifndef {guard}",
        f"#define {guard}",
        "",
        "#include <stdint.h>",
        "",
    ]
    for name in NAMES:
        v = tables[name]
        dims = "".join(f"[{d}]" for d in _dims(v))
        lines.append(f"{qualifier} uint8_t CAVLC_{name}{dims} = {_c_init(v)};")
    lines += ["", f"#endif  // {guard}", ""]
    return "\n".join(lines)


def main(reference_root: str) -> None:
    text = open(os.path.join(reference_root, H264, "tables.rs")).read()
    tables = {name: _const(text, name) for name in NAMES}
    with open(os.path.join(HERE, "cavlc_tables.json"), "w") as f:
        json.dump(dict(tables, source="crates/ironav-codec/src/h264/tables.rs"), f)
        f.write("\n")
    with open(os.path.join(ROOT, "oracle", "cavlc_tables.h"), "w") as f:
        f.write(_header(tables, "static const", "IRONAV_ORACLE_CAVLC_TABLES_H",
                        "oracle/cavlc_tables.h — the oracle's CAVLC tables (test infrastructure)."))
    with open(os.path.join(ROOT, "ironav_b200", "csrc", "cavlc_tables.cuh"), "w") as f:
        f.write(_header(tables, "static __constant__", "IRONAV_CAVLC_TABLES_CUH",
                        "cavlc_tables.cuh — the CUDA CAVLC writer's tables, in constant memory."))


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit("usage: python -m tests.golden.make_cavlc_tables <reference-root>")
    main(sys.argv[1])
