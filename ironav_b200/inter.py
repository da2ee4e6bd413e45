"""Python binding of the inter-analysis C ABI (include/ironav_inter.h).

`InterStage` mirrors the calls the reference encoder makes into this stage for one stream
(crates/ironav-codec/src/h264/enc/):

- ``push_reference``   -> ``HalfPel::new`` of a new reference picture (mod.rs:660) and the
  reference list update (mod.rs:663-666);
- ``begin_p_picture``  -> ``FrameCoder::new`` / ``with_refs`` / ``with_fast`` / ``with_sub8x8``
  (frame.rs:381-440) for a P picture;
- ``analyse_replay``   -> for every macroblock, the P_Skip vector and SAD of ``code_mb``
  (frame.rs:722-729) and ``best_inter`` (frame.rs:839-849), given the final decisions of the
  neighbours;
- ``analyse_auto``     -> the same, with the stage deciding each macroblock itself (P_Skip below the
  threshold, else the best inter partitioning) in wavefront order.

The library is ``ironav_b200/lib/libironav_inter_cuda.so``; loading fails loudly when it is missing
or no CUDA device is present. Another library implementing the same header may be passed as ``lib``.
"""
from __future__ import annotations

import ctypes
import os
from dataclasses import dataclass

import numpy as np

from . import build as _build

MBSTATE_DTYPE = np.dtype(
    [("inter", "u1"), ("refs", "i1", (4,)), ("pad", "u1", (3,)), ("mvs", "<i2", (16, 2))]
)
MBRESULT_DTYPE = np.dtype(
    [
        ("skip_mv", "<i2", (2,)),
        ("skip_sad", "<i4"),
        ("part", "u1"),
        ("refs", "u1", (4,)),
        ("sub", "u1", (4,)),
        ("flags", "u1"),
        ("pad", "u1", (2,)),
        ("cost", "<i4"),
        ("mvs", "<i2", (16, 2)),
        ("cost16", "<i4"),
        ("sad_px", "<u4"),
        ("satd_px", "<u4"),
        ("pad2", "<u4"),
    ]
)
# One macroblock as the deblocking filter sees it (ironav_dbk_mb: the MbInfo fields of h264/mb.rs:34-68 that
# h264/deblock.rs reads) and a slice's filter parameters (ironav_dbk_slice, SliceParams, h264/mb.rs:115-120).
DBK_MB_DTYPE = np.dtype(
    [
        ("slice", "<u2"),
        ("inter", "u1"),
        ("qp", "i1"),
        ("t8x8", "u1"),
        ("keep", "u1"),
        ("pad", "u1", (2,)),
        ("nnz", "u1", (16,)),
        ("ref_idx", "i1", (2, 4)),
        ("ref_id", "<i4", (2, 4)),
        ("mv", "<i2", (2, 16, 2)),
    ]
)
DBK_SLICE_DTYPE = np.dtype(
    [("disable_deblocking", "<i4"), ("alpha_offset", "<i4"), ("beta_offset", "<i4"), ("chroma_qp_offset", "<i4", (2,))]
)
# B pictures: a macroblock's final decision with both lists (ironav_mbstate_b) and the B searches' results
# (ironav_bresult).
MBSTATE_B_DTYPE = np.dtype([("inter", "u1"), ("refs", "i1", (2, 4)), ("pad", "u1", (3,)), ("mvs", "<i2", (2, 16, 2))])
BRESULT_DTYPE = np.dtype(
    [
        ("direct_mv", "<i2", (2, 16, 2)),
        ("direct_use", "u1", (2,)),
        ("dir16", "u1"),
        ("has_parts", "u1"),
        ("part", "u1"),
        ("bdir", "u1", (4,)),
        ("pad", "u1", (3,)),
        ("mv16", "<i2", (2, 2)),
        ("cost16", "<i4", (2,)),
        ("cost_bi", "<i4"),
        ("pmv", "<i2", (2, 4, 2)),
        ("sad_px", "<u4"),
        ("satd_px", "<u4"),
    ]
)
assert MBSTATE_DTYPE.itemsize == 72 and MBRESULT_DTYPE.itemsize == 104
assert MBSTATE_B_DTYPE.itemsize == 140 and BRESULT_DTYPE.itemsize == 200
# Inter residual coding: a macroblock's decision (ironav_interdec) and its coded residual (ironav_intercode).
INTERDEC_DTYPE = np.dtype([("mode", "u1"), ("part", "u1"), ("sub", "u1", (4,)), ("refs", "u1", (4,)), ("t8", "u1"),
                           ("pad", "u1", (3,)), ("mvs", "<i2", (16, 2))])
INTERCODE_DTYPE = np.dtype([("luma", "<i2", (16, 16)), ("luma8", "<i2", (4, 64)), ("cdc", "<i2", (2, 4)),
                            ("cac", "<i2", (2, 4, 16)), ("nnz", "u1", (16,)), ("cnnz", "u1", (2, 4)), ("cbp", "u1"),
                            ("t8x8", "u1"), ("pad", "u1", (2,))])
assert INTERDEC_DTYPE.itemsize == 78 and INTERCODE_DTYPE.itemsize == 1324
# Decide mode: a macroblock's code (ironav_mbcode, MbCode) and the reference's Kind values it carries.
MBCODE_DTYPE = np.dtype([("res", INTERCODE_DTYPE), ("dc", "<i2", (16,)), ("mvs", "<i2", (16, 2)), ("mvds", "<i2", (16, 2)),
                         ("modes", "u1", (16,)), ("kind", "u1"), ("skip", "u1"), ("i16_mode", "u1"), ("chroma_mode", "u1"),
                         ("part", "u1"), ("sub", "u1", (4,)), ("refs", "u1", (4,)), ("pad", "u1", (3,))])
assert MBCODE_DTYPE.itemsize == 1516
KIND_I4X4, KIND_I16X16, KIND_INTER = 1, 3, 5
assert DBK_MB_DTYPE.itemsize == 192 and DBK_SLICE_DTYPE.itemsize == 20

RESULT_INTER = 1
RESULT_SKIP = 2

# ironav_status: 1 + the index of ironav_core::ErrorCode (crates/ironav-core/src/error.rs:9-27)
STATUS_NAMES = {
    0: "Ok",
    2: "InvalidInput",
    3: "InvalidArgument",
    8: "HardwareUnavailable",
    13: "Internal",
    100: "Timeout",
}

# Every entry point include/ironav_inter.h declares.
EXPORTS = (
    "ironav_lambda", "ironav_skip_threshold", "ironav_se_bits", "ironav_ue_bits", "ironav_version",
    "ironav_ctx_create", "ironav_ctx_destroy", "ironav_ctx_dims", "ironav_ctx_set_stream",
    "ironav_set_source", "ironav_push_reference", "ironav_clear_references", "ironav_get_planes",
    "ironav_begin_p_picture", "ironav_analyse_picture_replay", "ironav_analyse_picture_auto",
    "ironav_set_source_device", "ironav_push_reference_device",
    "ironav_analyse_picture_replay_device", "ironav_analyse_picture_auto_device", "ironav_ctx_sync",
    "ironav_inloop_begin", "ironav_inloop_result", "ironav_inloop_commit", "ironav_inloop_end",
    "ironav_inloop_set_wait", "ironav_batch_create", "ironav_batch_destroy", "ironav_batch_step",
    "ironav_batch_sync", "ironav_scene_change", "ironav_scene_change_device", "ironav_analyse_auto_noalloc",
    "ironav_deblock_picture", "ironav_deblock_picture_device",
    "ironav_begin_b_picture", "ironav_begin_b_picture_device", "ironav_analyse_b_replay", "ironav_analyse_b_replay_device",
    "ironav_set_source_chroma", "ironav_push_reference_chroma", "ironav_code_inter_picture", "ironav_code_inter_picture_device",
    "ironav_decide_p_picture", "ironav_decide_p_picture_device", "ironav_batch_decide", "ironav_decide_dbk_records",
    "ironav_decide_dbk_records_device", "ironav_batch_deblock",
    "ironav_begin_i_picture", "ironav_decide_i_picture", "ironav_decide_i_picture_device", "ironav_set_source_chroma_device",
    "ironav_push_reference_chroma_device",
    "ironav_write_parameter_sets", "ironav_write_slices", "ironav_write_slices_device",
    "ironav_batch_set_tuning", "ironav_batch_get_tuning", "ironav_batch_autotune",
    "ironav_prop_conv3x3", "ironav_prop_wgrad3x3", "ironav_prop_prep", "ironav_prop_head_fwd", "ironav_prop_loss",
    "ironav_prop_head_bwd", "ironav_prop_adam", "ironav_prop_weights", "ironav_set_learned",
    "ironav_prop_propose", "ironav_set_replay_form", "ironav_prop_head_pack", "ironav_prop_head_fwd_packed",
    "ironav_set_entropy",
)

# ironav_batch_tuning (include/ironav_inter.h): the batched step's knobs
BATCH_TUNING_DTYPE = np.dtype([("k2_ctas_per_sm", "<i4"), ("k1_tile_rows", "<i4"), ("order", "<i4"), ("k2_group", "<i4"), ("ms", "<f4")])

# ironav_stream_params (include/ironav_inter.h): what the SPS and PPS say
STREAM_PARAMS_DTYPE = np.dtype([("width", "<i4"), ("height", "<i4"), ("bd", "<i4"), ("fps_num", "<i4"), ("fps_den", "<i4"),
                                ("refs", "<i4"), ("cabac", "<i4"), ("transform8", "<i4")])

SCENE_CUT = 0.8  # codec/change.rs:6


class IronavError(RuntimeError):
    """A non-zero ironav_status; `.status` holds the code and `.name` the ErrorCode it maps to."""

    def __init__(self, status: int, what: str):
        self.status = status
        self.name = STATUS_NAMES.get(status, f"status {status}")
        super().__init__(f"{what}: {self.name} ({status})")


_VP = ctypes.c_void_p
_I = ctypes.c_int


def _declare(lib: ctypes.CDLL) -> ctypes.CDLL:
    lib.ironav_lambda.argtypes = [_I]
    lib.ironav_skip_threshold.argtypes = [_I]
    lib.ironav_se_bits.argtypes = [_I]
    lib.ironav_ue_bits.argtypes = [ctypes.c_uint]
    lib.ironav_version.restype = ctypes.c_char_p
    lib.ironav_ctx_create.argtypes = [ctypes.POINTER(_VP), _I, _I, _I, _I, _I, _VP]
    lib.ironav_ctx_destroy.argtypes = [_VP]
    lib.ironav_ctx_dims.argtypes = [_VP] + [ctypes.POINTER(_I)] * 4
    lib.ironav_ctx_set_stream.argtypes = [_VP, _VP]
    lib.ironav_set_source.argtypes = [_VP, _VP, _I]
    lib.ironav_push_reference.argtypes = [_VP, _VP, _I, _I, _I, _VP]
    lib.ironav_clear_references.argtypes = [_VP]
    lib.ironav_get_planes.argtypes = [_VP, _I, _VP]
    lib.ironav_begin_p_picture.argtypes = [_VP, _I, _I, _I, _I, _I, _I]
    lib.ironav_analyse_picture_replay.argtypes = [_VP, _VP, _VP]
    lib.ironav_analyse_picture_auto.argtypes = [_VP, _VP, _VP]
    lib.ironav_set_source_device.argtypes = [_VP, _VP, _I]
    lib.ironav_push_reference_device.argtypes = [_VP, _VP, _I, _I, _I, _VP]
    lib.ironav_analyse_picture_replay_device.argtypes = [_VP, _VP, _VP]
    lib.ironav_analyse_picture_auto_device.argtypes = [_VP, _VP, _VP]
    lib.ironav_ctx_sync.argtypes = [_VP]
    if hasattr(lib, "ironav_inloop_begin"):
        lib.ironav_inloop_begin.argtypes = [_VP, _I]
        lib.ironav_inloop_result.argtypes = [_VP, _I, _VP, _I]
        lib.ironav_inloop_commit.argtypes = [_VP, _I, _VP]
        lib.ironav_inloop_end.argtypes = [_VP]
        lib.ironav_inloop_set_wait.argtypes = [_VP, _I]
    if hasattr(lib, "ironav_scene_change"):
        lib.ironav_scene_change.argtypes = [_VP, _VP, _VP, _I, _VP]
        lib.ironav_scene_change_device.argtypes = [_VP, _VP, _VP, _I, _VP]
    if hasattr(lib, "ironav_begin_b_picture"):
        lib.ironav_begin_b_picture.argtypes = [_VP, _I, _I, _I, _I, _VP, _I, _I, _I]
        lib.ironav_begin_b_picture_device.argtypes = [_VP, _I, _I, _I, _I, _VP, _I, _I, _I]
        lib.ironav_analyse_b_replay.argtypes = [_VP, _VP, _VP]
        lib.ironav_analyse_b_replay_device.argtypes = [_VP, _VP, _VP]
    if hasattr(lib, "ironav_code_inter_picture"):
        lib.ironav_set_source_chroma.argtypes = [_VP, _VP, _VP, _I]
        lib.ironav_push_reference_chroma.argtypes = [_VP, _VP, _VP, _I, _I, _I]
        lib.ironav_code_inter_picture.argtypes = [_VP, _I, _VP, _VP, _VP, _I, _VP, _VP, _I]
        lib.ironav_code_inter_picture_device.argtypes = [_VP, _I, _VP, _VP, _VP, _I, _VP, _VP, _I]
    if hasattr(lib, "ironav_decide_p_picture"):
        lib.ironav_decide_p_picture.argtypes = [_VP, _VP, _VP, _VP, _I, _VP, _VP, _I]
        lib.ironav_decide_dbk_records.argtypes = [_VP, _VP, _VP, _VP]
        lib.ironav_decide_dbk_records_device.argtypes = [_VP, _VP, _VP, _VP]
        lib.ironav_decide_p_picture_device.argtypes = [_VP, _VP, _VP, _VP, _I, _VP, _VP, _I]
    if hasattr(lib, "ironav_deblock_picture"):
        lib.ironav_deblock_picture.argtypes = [_VP, _VP, _I, _VP, _VP, _I, _VP, _VP, _I]
        lib.ironav_deblock_picture_device.argtypes = [_VP, _VP, _I, _VP, _VP, _I, _VP, _VP, _I]
    if hasattr(lib, "ironav_batch_create"):
        lib.ironav_batch_create.argtypes = [ctypes.POINTER(_VP), ctypes.POINTER(_VP), _I]
        lib.ironav_batch_destroy.argtypes = [_VP]
        lib.ironav_batch_step.argtypes = [_VP] + [ctypes.POINTER(_VP)] * 5
        lib.ironav_batch_sync.argtypes = [_VP]
    if hasattr(lib, "ironav_prop_conv3x3"):
        _LL, _F = ctypes.c_longlong, ctypes.c_float
        lib.ironav_prop_conv3x3.argtypes = [_VP, _I, _LL, _VP, _VP, _I, _VP, _VP, _VP, _VP]
        lib.ironav_prop_wgrad3x3.argtypes = [_VP, _I, _VP, _LL, _VP, _VP, _VP, _VP]
        lib.ironav_prop_prep.argtypes = [_VP, _I, _VP, _VP]
        lib.ironav_prop_head_fwd.argtypes = [_VP, _I, _VP, _VP, _VP, _VP]
        lib.ironav_prop_loss.argtypes = [_VP, _VP, _VP, _I, _VP, _VP, _VP]
        lib.ironav_prop_head_bwd.argtypes = [_VP, _I, _VP, _VP, _VP, _VP, _VP, _VP]
        lib.ironav_prop_adam.argtypes = [_VP, _VP, _VP, _VP, _LL, _F, _F, _F, _I, _F, _VP]
        lib.ironav_prop_weights.argtypes = [_VP, _I, _VP, _VP, _VP]
    if hasattr(lib, "ironav_prop_head_pack"):
        lib.ironav_prop_head_pack.argtypes = [_VP, _VP, _VP]
        lib.ironav_prop_head_fwd_packed.argtypes = [_VP, _I, _VP, _VP, _VP, _VP]
    if hasattr(lib, "ironav_prop_propose"):
        lib.ironav_prop_propose.argtypes = [_VP, _I, _F, _VP, _VP, _VP]
    if hasattr(lib, "ironav_set_replay_form"):
        lib.ironav_set_replay_form.argtypes = [_VP, _I]
    if hasattr(lib, "ironav_set_learned"):
        lib.ironav_set_learned.argtypes = [_VP, _VP, _VP, _I, _VP]
    if hasattr(lib, "ironav_batch_autotune"):
        lib.ironav_batch_set_tuning.argtypes = [_VP, _VP]
        lib.ironav_batch_get_tuning.argtypes = [_VP, _VP]
        lib.ironav_batch_autotune.argtypes = [_VP] + [ctypes.POINTER(_VP)] * 5 + [_I, _VP, _VP, _I, ctypes.POINTER(_I)]
    if hasattr(lib, "ironav_batch_deblock"):
        lib.ironav_batch_deblock.argtypes = [_VP, ctypes.POINTER(_VP), ctypes.POINTER(_I), ctypes.POINTER(_VP), ctypes.POINTER(_VP),
                                             ctypes.POINTER(_I), ctypes.POINTER(_VP), ctypes.POINTER(_VP), ctypes.POINTER(_I)]
    if hasattr(lib, "ironav_batch_decide"):
        lib.ironav_batch_decide.argtypes = [_VP, ctypes.POINTER(_VP), ctypes.POINTER(_VP), ctypes.POINTER(_VP), ctypes.POINTER(_I),
                                            ctypes.POINTER(_VP), ctypes.POINTER(_VP), ctypes.POINTER(_I)]
    if hasattr(lib, "ironav_begin_i_picture"):
        lib.ironav_begin_i_picture.argtypes = [_VP, _I, _I, _I]
        lib.ironav_decide_i_picture.argtypes = [_VP, _VP, _VP, _VP, _I, _VP, _VP, _I]
        lib.ironav_decide_i_picture_device.argtypes = [_VP, _VP, _VP, _VP, _I, _VP, _VP, _I]
        lib.ironav_set_source_chroma_device.argtypes = [_VP, _VP, _VP, _I]
        lib.ironav_push_reference_chroma_device.argtypes = [_VP, _VP, _VP, _I, _I, _I]
        _SZ = ctypes.POINTER(ctypes.c_size_t)
        lib.ironav_write_parameter_sets.argtypes = [_VP, _VP, ctypes.c_size_t, _SZ]
        lib.ironav_write_slices.argtypes = [_VP, _I, _I, _I, _VP, _VP, ctypes.c_size_t, _SZ]
        lib.ironav_write_slices_device.argtypes = [_VP, _I, _I, _I, _VP, _VP, ctypes.c_size_t, _SZ]
    if hasattr(lib, "ironav_set_entropy"):
        lib.ironav_set_entropy.argtypes = [_VP, _I, _I]
    if hasattr(lib, "ironav_analyse_auto_noalloc"):
        # (d_src, src_stride, d_ref, ref_stride, ref_w, ref_h, d_col, width, height, nslices, qp_prime, lambda,
        #  skip_thresh, fast, sub8, d_planes, d_states, d_results, stream)
        lib.ironav_analyse_auto_noalloc.argtypes = [_VP, _I, _VP, _I, _I, _I, _VP, _I, _I, _I, _I, _I, _I, _I, _I,
                                                    _VP, _VP, _VP, _VP]
    for name in ("ironav_debug_withhold", "ironav_debug_wait_limit"):
        if hasattr(lib, name):
            getattr(lib, name).argtypes = [_VP, ctypes.c_int if name.endswith("withhold") else ctypes.c_uint]
    if hasattr(lib, "ironav_debug_noalloc_wait"):
        lib.ironav_debug_noalloc_wait.argtypes = [_I, ctypes.c_uint]
    return lib


_CUDA = None

# An open in-loop picture is a kernel that stays resident until the caller has committed every decision.
# A call that synchronises the whole device (cudaFree when a context is destroyed, among others) waits for
# it, so a context destroyed from a thread the picture needs — Python's garbage collector may run in any
# thread — would stall the picture until its wait bound. While in-loop pictures are open, contexts that go
# out of use are therefore destroyed only when the last of those pictures ends.
import threading as _threading

_INLOOP_LOCK = _threading.Lock()
_INLOOP_OPEN = 0
_DEFERRED: list = []


def _destroy_later_or_now(lib, ctx) -> None:
    with _INLOOP_LOCK:
        if _INLOOP_OPEN > 0:
            _DEFERRED.append((lib, ctx))
            return
    lib.ironav_ctx_destroy(ctx)


def _inloop_opened() -> None:
    global _INLOOP_OPEN
    with _INLOOP_LOCK:
        _INLOOP_OPEN += 1


def _inloop_closed() -> None:
    global _INLOOP_OPEN
    with _INLOOP_LOCK:
        _INLOOP_OPEN -= 1
        todo = []
        if _INLOOP_OPEN == 0:
            todo, _DEFERRED[:] = list(_DEFERRED), []
    for lib, ctx in todo:
        lib.ironav_ctx_destroy(ctx)


def cuda_library() -> ctypes.CDLL:
    """The sm_100a library, built in-tree. Raises when it is absent: there is no CPU fallback."""
    global _CUDA
    if _CUDA is None:
        path = _build.CUDA_LIB
        if not os.path.exists(path):
            raise RuntimeError(f"{path} is missing: build it with `python -m ironav_b200.build`")
        _CUDA = _declare(ctypes.CDLL(path))
    return _CUDA


_INLOOP_CALLER = None


def inloop_caller() -> ctypes.CDLL:
    """The native in-loop caller (libironav_inloop_caller.so): ironav_inloop_drive_bands(ctx, mb_w, nbands,
    band_rows, skip_thresh, states, results) runs one P picture with one host thread per slice band."""
    global _INLOOP_CALLER
    if _INLOOP_CALLER is None:
        from . import build

        cuda_library()
        lib = ctypes.CDLL(build.INLOOP_LIB)
        lib.ironav_inloop_drive_bands.argtypes = [_VP, _I, _I, _VP, _I, _VP, _VP]
        _INLOOP_CALLER = lib
    return _INLOOP_CALLER


def load_library(path: str) -> ctypes.CDLL:
    """Another implementation of include/ironav_inter.h (same entry points, same meaning)."""
    return _declare(ctypes.CDLL(path))


def _ptr(a: np.ndarray) -> int:
    return a.ctypes.data


def lambda_of(qp_prime: int, lib: ctypes.CDLL | None = None) -> int:
    return (lib or cuda_library()).ironav_lambda(qp_prime)


@dataclass
class PictureParams:
    qp_prime: int
    nrefs_active: int = 1
    fast: bool = False
    sub8: bool = False


class InterStage:
    """One stream's inter-analysis context (ironav_ctx). ``bd`` is the sample depth, 8 or 10 (the
    encoder's Yuv420p / Yuv420p10, enc/mod.rs:140-143): luma arrays are uint8 at 8 bits and uint16 at 10."""

    def __init__(self, width: int, height: int, max_refs: int = 1, nslices: int = 1,
                 band_rows: list[int] | None = None, lib: ctypes.CDLL | None = None, bd: int = 8):
        self.lib = lib if lib is not None else cuda_library()
        self.width, self.height, self.bd = width, height, bd
        self.dtype = np.uint8 if bd == 8 else np.uint16
        h = _VP()
        bands = None
        if band_rows is not None:
            self._bands = np.asarray(band_rows, dtype=np.int32)
            bands = _ptr(self._bands)
        self._check(self.lib.ironav_ctx_create(ctypes.byref(h), width, height, bd, max_refs, nslices, bands),
                    "ironav_ctx_create")
        self.ctx = h
        mw, mh, sw, sh = _I(), _I(), _I(), _I()
        self.lib.ironav_ctx_dims(self.ctx, ctypes.byref(mw), ctypes.byref(mh), ctypes.byref(sw), ctypes.byref(sh))
        self.mb_w, self.mb_h, self.sw, self.sh = mw.value, mh.value, sw.value, sh.value
        self.nmb = self.mb_w * self.mb_h

    @staticmethod
    def _check(status: int, what: str) -> None:
        if status != 0:
            raise IronavError(status, what)

    def close(self) -> None:
        if getattr(self, "ctx", None):
            if getattr(self, "_inloop_open", False):
                self.inloop_end_quietly()
            _destroy_later_or_now(self.lib, self.ctx)
            self.ctx = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    # -- pictures ------------------------------------------------------------------------------------

    def _luma(self, luma: np.ndarray) -> np.ndarray:
        if luma.dtype != self.dtype:
            raise TypeError(f"{self.bd}-bit context takes {np.dtype(self.dtype).name} luma, got {luma.dtype}")
        return np.ascontiguousarray(luma)

    def set_source(self, luma: np.ndarray) -> None:
        luma = self._luma(luma)
        assert luma.shape == (self.height, self.width)
        self._check(self.lib.ironav_set_source(self.ctx, _ptr(luma), self.width), "ironav_set_source")

    def push_reference(self, luma: np.ndarray, col: np.ndarray | None = None) -> None:
        luma = self._luma(luma)
        h, w = luma.shape
        colp = None
        if col is not None:
            col = np.ascontiguousarray(col, dtype=MBSTATE_DTYPE)
            assert col.shape == (self.nmb,)
            colp = _ptr(col)
        self._check(self.lib.ironav_push_reference(self.ctx, _ptr(luma), w, w, h, colp), "ironav_push_reference")

    def clear_references(self) -> None:
        self._check(self.lib.ironav_clear_references(self.ctx), "ironav_clear_references")

    def planes(self, idx: int = 0) -> np.ndarray:
        out = np.empty((4, self.sh, self.sw), dtype=self.dtype)
        self._check(self.lib.ironav_get_planes(self.ctx, idx, _ptr(out)), "ironav_get_planes")
        return out

    def begin_p_picture(self, qp_prime: int, nrefs_active: int = 1, fast: bool = False, sub8: bool = False) -> None:
        lam = self.lib.ironav_lambda(qp_prime)
        thr = self.lib.ironav_skip_threshold(qp_prime)
        self._check(self.lib.ironav_begin_p_picture(self.ctx, qp_prime, lam, thr, nrefs_active, int(fast), int(sub8)),
                    "ironav_begin_p_picture")

    def analyse_replay(self, states: np.ndarray) -> np.ndarray:
        states = np.ascontiguousarray(states, dtype=MBSTATE_DTYPE)
        assert states.shape == (self.nmb,)
        out = np.zeros(self.nmb, dtype=MBRESULT_DTYPE)
        self._check(self.lib.ironav_analyse_picture_replay(self.ctx, _ptr(states), _ptr(out)),
                    "ironav_analyse_picture_replay")
        return out

    def analyse_auto(self) -> tuple[np.ndarray, np.ndarray]:
        states = np.zeros(self.nmb, dtype=MBSTATE_DTYPE)
        out = np.zeros(self.nmb, dtype=MBRESULT_DTYPE)
        self._check(self.lib.ironav_analyse_picture_auto(self.ctx, _ptr(states), _ptr(out)),
                    "ironav_analyse_picture_auto")
        return states, out

    # -- scene-cut measure (change_threads, codec/change.rs:56-90) -----------------------------------------

    def scene_change(self, prev: np.ndarray, cur: np.ndarray) -> tuple[int, int]:
        """(inter, intra) totals of cur against prev on the low-resolution luma."""
        prev = self._luma(prev)
        cur = self._luma(cur)
        out = np.zeros(2, dtype=np.int64)
        self._check(self.lib.ironav_scene_change(self.ctx, _ptr(prev), _ptr(cur), self.width, _ptr(out)),
                    "ironav_scene_change")
        return int(out[0]), int(out[1])

    def scene_cut(self, prev: np.ndarray, cur: np.ndarray) -> bool:
        """Whether cur starts a new scene: inter > SCENE_CUT * intra, in f64 (enc/mod.rs:707-711)."""
        inter, intra = self.scene_change(prev, cur)
        return float(inter) > SCENE_CUT * float(intra)

    # -- B pictures (decide_b's searches, enc/frame.rs:1518-1572, 1626-1747) ------------------------------

    def begin_b_picture(self, qp_prime: int, ref_l0: int, ref_l1: int, col: np.ndarray | None, tb: int, td: int,
                        fast: bool = False) -> None:
        lam = self.lib.ironav_lambda(qp_prime)
        colp = None
        if col is not None:
            self._bcol = np.ascontiguousarray(col, dtype=MBSTATE_DTYPE)
            assert self._bcol.shape == (self.nmb,)
            colp = _ptr(self._bcol)
        self._check(self.lib.ironav_begin_b_picture(self.ctx, qp_prime, lam, ref_l0, ref_l1, colp, tb, td, int(fast)),
                    "ironav_begin_b_picture")

    def analyse_b_replay(self, states: np.ndarray) -> np.ndarray:
        states = np.ascontiguousarray(states, dtype=MBSTATE_B_DTYPE)
        assert states.shape == (self.nmb,)
        out = np.zeros(self.nmb, dtype=BRESULT_DTYPE)
        self._check(self.lib.ironav_analyse_b_replay(self.ctx, _ptr(states), _ptr(out)), "ironav_analyse_b_replay")
        return out

    # -- inter residual coding and reconstruction (enc/frame.rs:1202-1305, 1856-1915) -------------------------

    def set_source_chroma(self, cb: np.ndarray, cr: np.ndarray) -> None:
        cb, cr = self._luma(cb), self._luma(cr)
        self._check(self.lib.ironav_set_source_chroma(self.ctx, _ptr(cb), _ptr(cr), cb.shape[1]), "ironav_set_source_chroma")

    def push_reference_chroma(self, cb: np.ndarray, cr: np.ndarray) -> None:
        cb, cr = self._luma(cb), self._luma(cr)
        h, w = cb.shape
        self._check(self.lib.ironav_push_reference_chroma(self.ctx, _ptr(cb), _ptr(cr), w, w, h), "ironav_push_reference_chroma")

    def code_inter(self, qp: int, decs: np.ndarray, rec: tuple[np.ndarray, np.ndarray, np.ndarray]):
        """Codes the inter macroblocks of decs (INTERDEC_DTYPE) into copies of the reconstruction planes rec
        (luma 16*mb_w x 16*mb_h, chroma 8*mb_w x 8*mb_h); returns (codes, (y, cb, cr))."""
        decs = np.ascontiguousarray(decs, dtype=INTERDEC_DTYPE)
        assert decs.shape == (self.nmb,)
        y, cb, cr = (self._luma(a).copy() for a in rec)
        codes = np.zeros(self.nmb, dtype=INTERCODE_DTYPE)
        self._check(self.lib.ironav_code_inter_picture(self.ctx, qp, _ptr(decs), _ptr(codes), _ptr(y), y.shape[1], _ptr(cb),
                                                       _ptr(cr), cb.shape[1]), "ironav_code_inter_picture")
        return codes, (y, cb, cr)

    def decide_p_picture(self):
        """Decides and codes every macroblock of the current P picture (code_mb, CAVLC): returns (states,
        codes, (y, cb, cr)) with the unfiltered reconstruction."""
        dt = np.uint8 if self.bd == 8 else np.uint16
        y = np.zeros((self.mb_h * 16, self.mb_w * 16), dt)
        cb = np.zeros((self.mb_h * 8, self.mb_w * 8), dt)
        cr = np.zeros_like(cb)
        states = np.zeros(self.nmb, dtype=MBSTATE_DTYPE)
        codes = np.zeros(self.nmb, dtype=MBCODE_DTYPE)
        self._check(self.lib.ironav_decide_p_picture(self.ctx, _ptr(states), _ptr(codes), _ptr(y), y.shape[1], _ptr(cb), _ptr(cr),
                                                     cb.shape[1]), "ironav_decide_p_picture")
        return states, codes, (y, cb, cr)

    def set_entropy(self, cabac: bool, transform8: bool = True) -> None:
        """CABAC (with rate-distortion decisions, and the 8x8 transform when transform8) or CAVLC for the
        decide and write entry points (H264Encoder's cabac and transform8 settings)."""
        self._check(self.lib.ironav_set_entropy(self.ctx, int(cabac), int(transform8)), "ironav_set_entropy")

    def begin_i_picture(self, qp_prime: int, fast: bool = False) -> None:
        """Parameters of an IDR picture (FrameCoder::new without a reference, enc/frame.rs:381-412)."""
        lam = self.lib.ironav_lambda(qp_prime)
        self._check(self.lib.ironav_begin_i_picture(self.ctx, qp_prime, lam, int(fast)), "ironav_begin_i_picture")

    def decide_i_picture(self):
        """Decides and codes every macroblock of the current IDR picture (code_mb without a reference):
        returns (states, codes, (y, cb, cr)) with the unfiltered reconstruction."""
        dt = np.uint8 if self.bd == 8 else np.uint16
        y = np.zeros((self.mb_h * 16, self.mb_w * 16), dt)
        cb = np.zeros((self.mb_h * 8, self.mb_w * 8), dt)
        cr = np.zeros_like(cb)
        states = np.zeros(self.nmb, dtype=MBSTATE_DTYPE)
        codes = np.zeros(self.nmb, dtype=MBCODE_DTYPE)
        self._check(self.lib.ironav_decide_i_picture(self.ctx, _ptr(states), _ptr(codes), _ptr(y), y.shape[1], _ptr(cb), _ptr(cr),
                                                     cb.shape[1]), "ironav_decide_i_picture")
        return states, codes, (y, cb, cr)

    def write_slices(self, idr: bool, frame_num: int, idr_pic_id: int, codes: np.ndarray) -> bytes:
        """The current picture's slice NAL units (Annex B) from its codes (MBCODE_DTYPE, mb_w*mb_h)."""
        codes = np.ascontiguousarray(codes, dtype=MBCODE_DTYPE)
        assert codes.shape == (self.nmb,)
        return _sized_call(lambda buf, cap, n: self.lib.ironav_write_slices(self.ctx, int(idr), frame_num, idr_pic_id, _ptr(codes),
                                                                             buf, cap, n), "ironav_write_slices", self._stream_guess(idr))

    def write_slices_device(self, idr: bool, frame_num: int, idr_pic_id: int, d_codes: int) -> bytes:
        return _sized_call(lambda buf, cap, n: self.lib.ironav_write_slices_device(self.ctx, int(idr), frame_num, idr_pic_id, d_codes,
                                                                                    buf, cap, n), "ironav_write_slices_device",
                           self._stream_guess(idr))

    def _stream_guess(self, idr: bool) -> int:
        # a buffer most pictures fit, so that the writer rarely runs twice (a call that is short of room
        # reports the size it needs and is made again): 128 bytes a macroblock for an IDR picture, 16 for P
        return max(1 << 16, self.nmb * (128 if idr else 16))

    def decide_dbk_records(self, codes: np.ndarray, states: np.ndarray) -> np.ndarray:
        """The deblocking filter's macroblock records (DBK_MB_DTYPE) of a picture decide_p_picture coded."""
        codes = np.ascontiguousarray(codes, dtype=MBCODE_DTYPE)
        states = np.ascontiguousarray(states, dtype=MBSTATE_DTYPE)
        mbs = np.zeros(self.nmb, dtype=DBK_MB_DTYPE)
        self._check(self.lib.ironav_decide_dbk_records(self.ctx, _ptr(codes), _ptr(states), _ptr(mbs)), "ironav_decide_dbk_records")
        return mbs

    # -- deblocking of the reconstruction (h264/deblock.rs) ------------------------------------------------

    def deblock(self, y: np.ndarray, cb: np.ndarray, cr: np.ndarray, mbs: np.ndarray,
                slices: np.ndarray) -> tuple[np.ndarray, np.ndarray, np.ndarray]:
        """The filtered copies of a reconstructed 4:2:0 picture (luma 16*mb_w x 16*mb_h, chroma half that)
        given its macroblock records (DBK_MB_DTYPE, mb_w*mb_h) and slice table (DBK_SLICE_DTYPE)."""
        y, cb, cr = (self._luma(a).copy() for a in (y, cb, cr))
        assert y.shape == (self.mb_h * 16, self.mb_w * 16) and cb.shape == cr.shape == (self.mb_h * 8, self.mb_w * 8)
        mbs = np.ascontiguousarray(mbs, dtype=DBK_MB_DTYPE)
        slices = np.ascontiguousarray(slices, dtype=DBK_SLICE_DTYPE)
        assert mbs.shape == (self.nmb,)
        self._check(self.lib.ironav_deblock_picture(self.ctx, _ptr(y), y.shape[1], _ptr(cb), _ptr(cr), cb.shape[1],
                                                    _ptr(mbs), _ptr(slices), len(slices)), "ironav_deblock_picture")
        return y, cb, cr

    def deblock_device(self, d_y: int, ys: int, d_cb: int, d_cr: int, cs: int, d_mbs: int, slices: np.ndarray) -> None:
        slices = np.ascontiguousarray(slices, dtype=DBK_SLICE_DTYPE)
        self._check(self.lib.ironav_deblock_picture_device(self.ctx, d_y, ys, d_cb, d_cr, cs, d_mbs, _ptr(slices),
                                                           len(slices)), "ironav_deblock_picture_device")

    # -- in-loop mode: the caller decides each macroblock (the encoder's own loop) ---------------------

    INLOOP_RASTER = 0
    INLOOP_BANDS = 1

    def inloop_begin(self, order: int = 0) -> None:
        self._check(self.lib.ironav_inloop_begin(self.ctx, order), "ironav_inloop_begin")
        self._inloop_open = True
        _inloop_opened()

    def inloop_result(self, mb: int, timeout_ms: int = 10000) -> np.ndarray:
        out = np.zeros(1, dtype=MBRESULT_DTYPE)
        self._check(self.lib.ironav_inloop_result(self.ctx, mb, _ptr(out), timeout_ms), "ironav_inloop_result")
        return out[0]

    def inloop_commit(self, mb: int, state: np.ndarray) -> None:
        st = np.ascontiguousarray(np.asarray(state, dtype=MBSTATE_DTYPE).reshape(1))
        self._check(self.lib.ironav_inloop_commit(self.ctx, mb, _ptr(st)), "ironav_inloop_commit")

    def inloop_end(self) -> None:
        status = self.lib.ironav_inloop_end(self.ctx)
        if getattr(self, "_inloop_open", False):
            self._inloop_open = False
            _inloop_closed()
        self._check(status, "ironav_inloop_end")

    def inloop_end_quietly(self) -> None:
        try:
            self.inloop_end()
        except IronavError:
            pass

    def inloop_set_wait(self, ms: int) -> None:
        self._check(self.lib.ironav_inloop_set_wait(self.ctx, ms), "ironav_inloop_set_wait")

    # -- device-resident forms (integer device pointers, e.g. torch tensor.data_ptr()) ---------------

    def set_stream(self, stream_handle: int) -> None:
        self._check(self.lib.ironav_ctx_set_stream(self.ctx, stream_handle), "ironav_ctx_set_stream")

    def set_source_device(self, d_luma: int, stride: int) -> None:
        self._check(self.lib.ironav_set_source_device(self.ctx, d_luma, stride), "ironav_set_source_device")

    def push_reference_device(self, d_luma: int, stride: int, w: int, h: int, d_col: int | None) -> None:
        self._check(self.lib.ironav_push_reference_device(self.ctx, d_luma, stride, w, h, d_col),
                    "ironav_push_reference_device")

    def analyse_replay_device(self, d_states: int, d_out: int) -> None:
        self._check(self.lib.ironav_analyse_picture_replay_device(self.ctx, d_states, d_out),
                    "ironav_analyse_picture_replay_device")

    def analyse_auto_device(self, d_states: int, d_out: int) -> None:
        self._check(self.lib.ironav_analyse_picture_auto_device(self.ctx, d_states, d_out),
                    "ironav_analyse_picture_auto_device")

    def sync(self) -> None:
        self._check(self.lib.ironav_ctx_sync(self.ctx), "ironav_ctx_sync")


# Sub-partitions of P_8x8 (SUB, enc/frame.rs:204): (x, y, w, h) in 4x4 blocks.
_SUB = [[(0, 0, 2, 2)], [(0, 0, 2, 1), (0, 1, 2, 1)], [(0, 0, 1, 2), (1, 0, 1, 2)],
        [(0, 0, 1, 1), (1, 0, 1, 1), (0, 1, 1, 1), (1, 1, 1, 1)]]
_PARTS = [[(0, 0, 4, 4)], [(0, 0, 4, 2), (0, 2, 4, 2)], [(0, 0, 2, 4), (2, 0, 2, 4)],
          [(0, 0, 2, 2), (2, 0, 2, 2), (0, 2, 2, 2), (2, 2, 2, 2)]]


def inter_decisions(res: np.ndarray, t8: bool = False) -> np.ndarray:
    """The inter coding decision of each macroblock from P analysis results (auto mode): P_Skip where the
    policy skipped (its vector), else the best_inter partitioning with its vectors and reference."""
    d = np.zeros(len(res), dtype=INTERDEC_DTYPE)
    skip = (res["flags"] & RESULT_SKIP) != 0
    inter = (res["flags"] & RESULT_INTER) != 0
    d["mode"] = np.where(skip, 1, np.where(inter, 2, 0))
    d["part"] = np.where(skip, 0, res["part"])
    d["sub"] = np.where(skip[:, None], 0, res["sub"])
    d["refs"] = np.where(skip[:, None], 0, res["refs"])
    d["t8"] = 1 if t8 else 0
    d["mvs"] = res["mvs"]
    d["mvs"][skip, 0] = res["skip_mv"][skip]
    return d


def b_decision_states(res: np.ndarray) -> np.ndarray:
    """A plausible final decision per B macroblock from its search results (the 16x16 of the best
    direction), for replaying a picture against decisions the stage itself would favour."""
    st = np.zeros(len(res), dtype=MBSTATE_B_DTYPE)
    st["inter"] = 1
    for l in (0, 1):
        used = (res["dir16"] >> l) & 1
        st["refs"][:, l] = np.where(used[:, None] == 1, 0, -1)
        st["mvs"][:, l] = np.where(used[:, None, None] == 1, res["mv16"][:, l][:, None, :], 0)
    return st


def decision_state(res, skip: bool) -> np.ndarray:
    """The MbState a P macroblock leaves once decided (finish_mb, enc/frame.rs:2281-2321): P_Skip with
    the skip vector, or the best_inter partitioning's vectors painted over its 4x4 blocks."""
    st = np.zeros(1, dtype=MBSTATE_DTYPE)[0]
    st["inter"] = 1
    if skip:
        st["mvs"][:] = res["skip_mv"]
        st["refs"][:] = 0
        return st
    part = int(res["part"])
    if part == 3:
        rects = [((k & 1) * 2 + x, (k >> 1) * 2 + y, w, h) for k in range(4) for (x, y, w, h) in _SUB[int(res["sub"][k])]]
    else:
        rects = _PARTS[part]
    for n, (x, y, w, h) in enumerate(rects):
        for by in range(y, y + h):
            for bx in range(x, x + w):
                st["mvs"][by * 4 + bx] = res["mvs"][n]
    st["refs"][:] = res["refs"]
    return st


class InterBatch:
    """The batched form: several InterStage streams stepped together, one launch per stage (ironav_batch)."""

    def __init__(self, stages: list[InterStage]):
        self.stages = stages
        self.lib = stages[0].lib
        arr = (_VP * len(stages))(*[s.ctx.value for s in stages])
        h = _VP()
        InterStage._check(self.lib.ironav_batch_create(ctypes.byref(h), arr, len(stages)), "ironav_batch_create")
        self.h = h

    def step(self, d_src, d_ref, d_col, d_states, d_results) -> None:
        """Lists of device pointers (ints; None in d_col for a reference without decisions)."""
        n = len(self.stages)
        mk = lambda xs: (_VP * n)(*[x if x is not None else None for x in xs])
        InterStage._check(self.lib.ironav_batch_step(self.h, mk(d_src), mk(d_ref), mk(d_col), mk(d_states), mk(d_results)),
                          "ironav_batch_step")

    def decide(self, d_states, d_codes, d_y, y_strides, d_cb, d_cr, c_strides) -> None:
        """Decide mode for every stream's current P picture in one launch: lists of device pointers (ints)
        and strides, one entry per stream (ironav_batch_decide)."""
        n = len(self.stages)
        vp = lambda xs: (_VP * n)(*xs)
        ip = lambda xs: (ctypes.c_int * n)(*xs)
        InterStage._check(self.lib.ironav_batch_decide(self.h, vp(d_states), vp(d_codes), vp(d_y), ip(y_strides), vp(d_cb), vp(d_cr),
                                                       ip(c_strides)), "ironav_batch_decide")

    def deblock(self, d_y, y_strides, d_cb, d_cr, c_strides, d_mbs, slices) -> None:
        """The deblocking filter of every stream's picture in place: lists of device pointers (ints) and
        strides, each stream's device records and its slice table (DBK_SLICE_DTYPE arrays) (ironav_batch_deblock)."""
        n = len(self.stages)
        vp = lambda xs: (_VP * n)(*xs)
        ip = lambda xs: (ctypes.c_int * n)(*xs)
        tabs = [np.ascontiguousarray(t, dtype=DBK_SLICE_DTYPE) for t in slices]
        InterStage._check(self.lib.ironav_batch_deblock(self.h, vp(d_y), ip(y_strides), vp(d_cb), vp(d_cr), ip(c_strides), vp(d_mbs),
                                                        vp([_ptr(t) for t in tabs]), ip([len(t) for t in tabs])), "ironav_batch_deblock")

    def sync(self) -> None:
        InterStage._check(self.lib.ironav_batch_sync(self.h), "ironav_batch_sync")

    # -- the tuner: the batched step's knobs for this stream mix on this GPU ---------------------------------

    def signature(self) -> str:
        """What a tuning is valid for: the GPU and every stream's size, bands and depth."""
        import torch

        streams = ",".join(f"{s.width}x{s.height}/{s.mb_h}r/{s.bd}b" for s in self.stages)
        return f"{torch.cuda.get_device_name()}|{streams}"

    def tuning(self) -> dict:
        t = np.zeros(1, dtype=BATCH_TUNING_DTYPE)
        InterStage._check(self.lib.ironav_batch_get_tuning(self.h, _ptr(t)), "ironav_batch_get_tuning")
        return {k: t[0][k].item() for k in ("k2_ctas_per_sm", "k1_tile_rows", "order", "k2_group")}

    def set_tuning(self, k2_ctas_per_sm: int, k1_tile_rows: int, order: int, k2_group: int = 0) -> None:
        """k2_group: 0, the analysis with one macroblock a warp; 8, one per 8-lane group (k2_ctas_per_sm 4)."""
        t = np.zeros(1, dtype=BATCH_TUNING_DTYPE)
        t[0] = (k2_ctas_per_sm, k1_tile_rows, order, k2_group, 0.0)
        InterStage._check(self.lib.ironav_batch_set_tuning(self.h, _ptr(t)), "ironav_batch_set_tuning")

    def autotune(self, d_src, d_ref, d_col, d_states, d_results, reps: int = 5, cache: str | None = None) -> dict:
        """Times every setting on `reps` steps of these inputs (ironav_batch_autotune; the batch ends as after one
        step of them) and keeps the fastest. With `cache` (a JSON file), a setting found before for the same
        signature is applied without timing (the step still runs once), and a new one is stored there.
        Returns {"best": {...}, "all": [...], "cached": bool}."""
        import json

        sig = self.signature()
        table = {}
        if cache and os.path.exists(cache):
            with open(cache) as f:
                table = json.load(f)
        if sig in table:
            b = table[sig]
            self.set_tuning(b["k2_ctas_per_sm"], b["k1_tile_rows"], b["order"], b.get("k2_group", 0))
            self.step(d_src, d_ref, d_col, d_states, d_results)
            self.sync()
            return {"best": b, "all": [], "cached": True}
        n = len(self.stages)
        mk = lambda xs: (_VP * n)(*[x if x is not None else None for x in xs])
        best = np.zeros(1, dtype=BATCH_TUNING_DTYPE)
        allv = np.zeros(32, dtype=BATCH_TUNING_DTYPE)
        cnt = _I(0)
        InterStage._check(self.lib.ironav_batch_autotune(self.h, mk(d_src), mk(d_ref), mk(d_col), mk(d_states), mk(d_results), reps,
                                                         _ptr(best), _ptr(allv), len(allv), ctypes.byref(cnt)), "ironav_batch_autotune")
        as_dict = lambda r: {k: r[k].item() for k in ("k2_ctas_per_sm", "k1_tile_rows", "order", "k2_group", "ms")}
        out = {"best": as_dict(best[0]), "all": [as_dict(allv[i]) for i in range(cnt.value)], "cached": False}
        if cache:
            table[sig] = out["best"]
            os.makedirs(os.path.dirname(os.path.abspath(cache)), exist_ok=True)
            with open(cache, "w") as f:
                json.dump(table, f, indent=1)
        return out

    def close(self) -> None:
        if getattr(self, "h", None):
            self.lib.ironav_batch_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def _sized_call(fn, what: str, guess: int) -> bytes:
    """Calls a writer (buf, cap, len*) that reports the bytes it needs when cap is too small; retries once
    with that size."""
    n = ctypes.c_size_t(0)
    for cap in (guess, None):
        if cap is None:
            cap = n.value
        buf = ctypes.create_string_buffer(max(cap, 1))
        st = fn(buf, cap, ctypes.byref(n))
        if st == 0:
            return buf.raw[: n.value]
        if st != 3 or n.value <= cap:
            raise IronavError(st, what)
    raise IronavError(3, what)


def write_parameter_sets(width: int, height: int, bd: int = 8, fps: tuple[int, int] = (30, 1), refs: int = 1,
                         lib: ctypes.CDLL | None = None, cabac: bool = False, transform8: bool = False) -> bytes:
    """The SPS and PPS NAL units (Annex B) of a stream without B pictures (H264Encoder::sps / pps,
    enc/mod.rs:296-400): CAVLC, or CABAC with or without the 8x8 transform."""
    lib = lib if lib is not None else cuda_library()
    p = np.zeros(1, dtype=STREAM_PARAMS_DTYPE)
    p[0] = (width, height, bd, fps[0], fps[1], refs, int(cabac), int(transform8))
    return _sized_call(lambda buf, cap, n: lib.ironav_write_parameter_sets(_ptr(p), buf, cap, n), "ironav_write_parameter_sets", 256)


def default_bands(mb_h: int, nslices: int) -> list[int]:
    """Slice bands as the encoder cuts them: band i = [i*mb_h/n, (i+1)*mb_h/n) (enc/mod.rs:603)."""
    return [i * mb_h // nslices for i in range(nslices + 1)]


def reference_slices(mb_h: int, cores: int) -> int:
    """The encoder's slice count, min(cores, max(mb_h/8, 1)) (enc/mod.rs:192)."""
    return min(cores, max(mb_h // 8, 1))
