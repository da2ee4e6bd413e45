"""Loads the oracle (oracle/_build/libironav_inter_cpu.so, the CPU restatement of the reference's
inter-analysis stage) for the tests. It implements include/ironav_inter.h, so the same binding drives
it and the CUDA library; it also exports oracle_* helpers for the interpolation known-answer test."""
from __future__ import annotations

import ctypes
import os
import subprocess

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
ORACLE_DIR = os.path.join(ROOT, "oracle")
ORACLE_LIB = os.path.join(ORACLE_DIR, "_build", "libironav_inter_cpu.so")

_LIB = None


def build_oracle() -> str:
    srcs = [os.path.join(ORACLE_DIR, f) for f in ("inter_oracle.c", "cavlc_tables.h", "cabac_tables.h")]
    if not os.path.exists(ORACLE_LIB) or any(os.path.getmtime(ORACLE_LIB) < os.path.getmtime(s) for s in srcs):
        subprocess.run(["make", "-s", "-C", ORACLE_DIR], check=True)
    return ORACLE_LIB


def oracle_library() -> ctypes.CDLL:
    global _LIB
    if _LIB is None:
        from ironav_b200.inter import load_library

        lib = load_library(build_oracle())
        u16p = ctypes.POINTER(ctypes.c_uint16)
        lib.oracle_luma_mc_ref.argtypes = [ctypes.c_void_p] + [ctypes.c_int] * 9 + [ctypes.c_void_p, ctypes.c_int]
        lib.oracle_halfpel_new.restype = ctypes.c_void_p
        lib.oracle_halfpel_new.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_int]
        lib.oracle_halfpel_free.argtypes = [ctypes.c_void_p]
        lib.oracle_halfpel_predict.argtypes = [ctypes.c_void_p] + [ctypes.c_int] * 6 + [ctypes.c_void_p]
        lib.oracle_halfpel_plane.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p]
        lib.oracle_satd4.argtypes = [ctypes.c_void_p]
        lib.oracle_decimate.argtypes = [ctypes.c_void_p, ctypes.c_int]
        lib.oracle_fdct4.argtypes = [ctypes.c_void_p, ctypes.c_void_p]
        lib.oracle_quant.argtypes = [ctypes.c_int] * 4
        lib.oracle_idct4_add.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int, ctypes.c_int]
        lib.oracle_quant8.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p]
        lib.oracle_idct8_add.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int, ctypes.c_int]
        lib.oracle_dbk_tables.argtypes = [ctypes.c_void_p] * 4
        lib.oracle_set_threads.argtypes = [ctypes.c_void_p, ctypes.c_int]
        lib.oracle_analyse_replay_subset.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
                                                     ctypes.c_int, ctypes.c_void_p]
        del u16p
        declare_stream_hooks(lib)
        _LIB = lib
    return _LIB


def declare_stream_hooks(lib) -> None:
    """The oracle's writer test hooks (not in the public header)."""
    lib.oracle_write_block.argtypes = [ctypes.c_int, ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p]
    lib.oracle_put_nal.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p, ctypes.c_int]
