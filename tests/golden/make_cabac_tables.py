"""Extracts the CABAC tables from the reference and writes them three ways (run from the repository root with
the root of a checkout of the reference as the argument:
`python -m tests.golden.make_cabac_tables <reference-root>`):

- tests/golden/cabac_tables.json: the fixture the CPU tests pin both headers against;
- oracle/cabac_tables.h: the oracle's copy (plain C arrays);
- ironav_b200/csrc/cabac_tables.cuh: the CUDA coder's copy (__constant__ arrays).

The tables are the standard's, as the reference holds them in crates/ironav-codec/src/h264/tables.rs and
cabac.rs: the context initialisation values (m, n) of ITU-T H.264 Tables 9-12 to 9-33 for I slices
(CABAC_INIT_I) and for P slices by cabac_init_idc (CABAC_INIT_PB), rangeTabLPS (Table 9-44, LPS_RANGE),
transIdxLPS (Table 9-45, TRANS_LPS), and the residual block context offsets of Tables 9-34 and 9-43
(SIG_OFF, LAST_OFF and ABS_OFF per ctxBlockCat; SIG_OFF_8X8 and LAST_OFF_8X8 per 8x8 scan position; row 0
of the two-row tables is the frame-coded one).
"""
from __future__ import annotations

import json
import os
import sys

from tests.golden.make_cavlc_tables import _c_init, _const, _dims

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
H264 = os.path.join("crates", "ironav-codec", "src", "h264")

# name -> (source file under h264/, C element type)
TABLES = {
    "CABAC_INIT_I": ("tables.rs", "int8_t"),
    "CABAC_INIT_PB": ("tables.rs", "int8_t"),
    "LPS_RANGE": ("tables.rs", "uint8_t"),
    "TRANS_LPS": ("cabac.rs", "uint8_t"),
    "SIG_OFF": ("tables.rs", "uint16_t"),
    "LAST_OFF": ("tables.rs", "uint16_t"),
    "ABS_OFF": ("tables.rs", "uint16_t"),
    "SIG_OFF_8X8": ("tables.rs", "uint8_t"),
    "LAST_OFF_8X8": ("tables.rs", "uint8_t"),
}


def _header(tables: dict, qualifier: str, guard: str, what: str) -> str:
    lines = [
        f"// {what}",
        "// Generated by tests/golden/make_cabac_tables.py: the CABAC tables of ITU-T H.264: context",
        "// initialisation (m, n) per ctxIdx for I slices (Tables 9-12 to 9-33, CABAC_INIT_I) and for P slices",
        "// by cabac_init_idc (CABAC_INIT_PB), rangeTabLPS[pStateIdx][qCodIRangeIdx] (Table 9-44), transIdxLPS",
        "// (Table 9-45), and the residual context offsets per ctxBlockCat (Table 9-34: significant_coeff_flag,",
        "// last_significant_coeff_flag, coeff_abs_level_minus1; row 0 frame coded) and per 8x8 scan position",
        "// (Table 9-43).",
        f"#ifndef {guard}",
        f"#define {guard}",
        "",
        "#include <stdint.h>",
        "",
    ]
    for name, (_, ctype) in TABLES.items():
        v = tables[name]
        dims = "".join(f"[{d}]" for d in _dims(v))
        lines.append(f"{qualifier} {ctype} {name}{dims} = {_c_init(v)};")
    lines += ["", f"#endif  // {guard}", ""]
    return "\n".join(lines)


def main(reference_root: str) -> None:
    texts = {}
    tables = {}
    for name, (src, _) in TABLES.items():
        if src not in texts:
            texts[src] = open(os.path.join(reference_root, H264, src)).read()
        tables[name] = _const(texts[src], name)
    with open(os.path.join(HERE, "cabac_tables.json"), "w") as f:
        json.dump(dict(tables, source="crates/ironav-codec/src/h264/tables.rs, cabac.rs"), f)
        f.write("\n")
    with open(os.path.join(ROOT, "oracle", "cabac_tables.h"), "w") as f:
        f.write(_header(tables, "static const", "IRONAV_ORACLE_CABAC_TABLES_H",
                        "oracle/cabac_tables.h — the oracle's CABAC tables (test infrastructure)."))
    with open(os.path.join(ROOT, "ironav_b200", "csrc", "cabac_tables.cuh"), "w") as f:
        f.write(_header(tables, "static __constant__", "IRONAV_CABAC_TABLES_CUH",
                        "cabac_tables.cuh — the CUDA CABAC coder's tables, in constant memory."))


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit("usage: python -m tests.golden.make_cabac_tables <reference-root>")
    main(sys.argv[1])
