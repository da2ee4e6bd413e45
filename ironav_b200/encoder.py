"""An IPPP H.264 encoder built on the library's entry points: the encoder loop of ironav-codec's H264Encoder
(crates/ironav-codec/src/h264/enc/mod.rs) without B pictures, with CAVLC (`constrained_baseline`,
enc/mod.rs:236-243) or with CABAC, rate-distortion decisions and the 8x8 transform (the High stream of
`low_latency`, enc/mod.rs:210-215), IDR pictures every `keyint` pictures or at a scene cut
(encode, enc/mod.rs:700-724), a constant quantiser with the IDR picture's offset of -3 (QP_OFFSET and
next_qp, enc/mod.rs:33,403-417), `refs` reference pictures, and `nslices` slice bands.

Each picture goes: scene-cut measure -> decide mode (ironav_decide_i_picture / ironav_decide_p_picture:
code_mb of every macroblock) -> the slices written (ironav_write_slices: header, write_mb, trailing bits;
SPS and PPS ahead of an IDR picture) -> the filter's records and the deblocking filter of the
reconstruction -> the filtered picture pushed as the newest reference (code_picture, enc/mod.rs:539-670).

`Encoder` runs on host buffers through any library that implements include/ironav_inter.h (the CUDA
library, or the oracle as the parity checker). `DeviceEncoder` keeps the whole picture pipeline on the GPU
(the device-pointer entry points, the context's stream) and brings only the stream's bytes back.
"""
from __future__ import annotations

import ctypes

import numpy as np

from .inter import (DBK_MB_DTYPE, DBK_SLICE_DTYPE, MBCODE_DTYPE, MBSTATE_DTYPE, SCENE_CUT, InterStage, cuda_library,
                    write_parameter_sets)

QP_OFFSET_IDR = -3  # QP_OFFSET[0], enc/mod.rs:33


class _Loop:
    """The encoder's picture bookkeeping (enc/mod.rs:539-545,636-668,700-724)."""

    def __init__(self, width: int, height: int, qp: int, keyint: int, refs: int, bd: int, fps: tuple[int, int]):
        self.width, self.height, self.qp, self.keyint, self.nrefs, self.bd, self.fps = width, height, qp, max(1, keyint), refs, bd, fps
        self.count = 0
        self.idr_at = 0
        self.frame_num = 0
        self.idr_id = 0
        self.held = 0  # reference pictures held (the list P pictures predict from)
        self.kinds: list[str] = []

    def qp_prime(self, idr: bool) -> int:
        q = min(max(self.qp + (QP_OFFSET_IDR if idr else 0), 0), 51)
        return q + 6 * (self.bd - 8)

    def choose(self, cut: bool) -> bool:
        d = self.count
        self.count += 1
        idr = d == 0 or d - self.idr_at >= self.keyint or cut
        if idr:
            self.frame_num = 0
            self.held = 0
            self.idr_at = d
        self.kinds.append("I" if idr else "P")
        return idr

    def after(self, idr: bool) -> None:
        if idr:
            self.idr_id = (self.idr_id + 1) % 65536
        self.held = min(self.held + 1, self.nrefs)
        self.frame_num = (self.frame_num + 1) % 256


class Encoder:
    """encode(y, cb, cr) -> the picture's Annex B bytes (with SPS and PPS ahead of an IDR picture), on host
    buffers through `lib`. `recon` holds the last picture's filtered reconstruction (y, cb, cr)."""

    def __init__(self, width: int, height: int, qp: int, keyint: int = 250, refs: int = 1, nslices: int = 1,
                 fps: tuple[int, int] = (30, 1), bd: int = 8, fast: bool = False, sub8: bool = False, scene_cut: bool = True,
                 lib: ctypes.CDLL | None = None, cabac: bool = False, transform8: bool = True):
        self.lib = lib if lib is not None else cuda_library()
        self.st = InterStage(width, height, max_refs=refs, nslices=nslices, lib=self.lib, bd=bd)
        self.st.set_entropy(cabac, transform8)
        self.loop = _Loop(width, height, qp, keyint, refs, bd, fps)
        self.fast, self.sub8, self.scene_cut = fast, sub8, scene_cut
        self.slices = np.zeros(nslices, dtype=DBK_SLICE_DTYPE)  # every slice filtered, no offsets (enc/mod.rs:648)
        self.prev = None
        self.recon = None
        self.codes = None
        self.states = None
        self.params = write_parameter_sets(width, height, bd, fps, refs, lib=self.lib, cabac=cabac, transform8=transform8)
        # called as before_p(encoder, y) once a P picture's parameters are set and before it is decided
        self.before_p = None

    def close(self) -> None:
        self.st.close()

    def encode(self, y: np.ndarray, cb: np.ndarray, cr: np.ndarray) -> bytes:
        st, L = self.st, self.loop
        cut = self.scene_cut and self.prev is not None and st.scene_cut(self.prev, y)
        self.prev = y
        idr = L.choose(cut)
        st.set_source(y)  # padded to whole macroblocks by the library, as H264Encoder::source does
        st.set_source_chroma(cb, cr)
        qpp = L.qp_prime(idr)
        if idr:
            st.clear_references()
            st.begin_i_picture(qpp, fast=self.fast)
            states, codes, rec = st.decide_i_picture()
            data = self.params + st.write_slices(True, L.frame_num, L.idr_id, codes)
        else:
            st.begin_p_picture(qpp, nrefs_active=min(L.held, L.nrefs), fast=self.fast, sub8=self.sub8)
            if self.before_p is not None:
                self.before_p(self, y)
            states, codes, rec = st.decide_p_picture()
            data = st.write_slices(False, L.frame_num, 0, codes)
        mbs = st.decide_dbk_records(codes, states)
        y_f, cb_f, cr_f = st.deblock(*rec, mbs, self.slices)
        st.push_reference(y_f, col=None if idr else states)
        st.push_reference_chroma(cb_f, cr_f)
        L.after(idr)
        self.recon, self.codes, self.states = (y_f, cb_f, cr_f), codes, states
        return data


class DeviceEncoder:
    """The same encoder with every picture's work on the GPU: the source planes go up once, and the scene-cut
    measure, decide mode, the filter's records, the deblocking filter and the new reference's planes run on
    device buffers on the context's stream; the slices are written from the codes in device memory, and only
    the stream's bytes come back. Needs the CUDA library and torch for device buffers."""

    def __init__(self, width: int, height: int, qp: int, keyint: int = 250, refs: int = 1, nslices: int = 1,
                 fps: tuple[int, int] = (30, 1), bd: int = 8, fast: bool = False, sub8: bool = False, scene_cut: bool = True,
                 cabac: bool = False, transform8: bool = True):
        import torch

        self.torch = torch
        self.lib = cuda_library()
        self.st = InterStage(width, height, max_refs=refs, nslices=nslices, lib=self.lib, bd=bd)
        self.st.set_entropy(cabac, transform8)
        self.loop = _Loop(width, height, qp, keyint, refs, bd, fps)
        self.fast, self.sub8, self.scene_cut = fast, sub8, scene_cut
        self.stream = torch.cuda.Stream()
        self.st.set_stream(self.stream.cuda_stream)
        dt = torch.uint8 if bd == 8 else torch.int16
        mb_w, mb_h, nmb = self.st.mb_w, self.st.mb_h, self.st.nmb
        dev = torch.device("cuda", torch.cuda.current_device())
        # the source as given (width x height, two pictures: the scene-cut measure reads the previous one)
        self.d_src = [torch.zeros((height, width), dtype=dt, device=dev) for _ in range(2)]
        self.d_src_c = torch.zeros((2, height // 2, width // 2), dtype=dt, device=dev)
        self.d_rec = torch.zeros((mb_h * 16, mb_w * 16), dtype=dt, device=dev)
        self.d_rec_c = torch.zeros((2, mb_h * 8, mb_w * 8), dtype=dt, device=dev)
        self.d_states = torch.zeros(nmb * MBSTATE_DTYPE.itemsize, dtype=torch.uint8, device=dev)
        self.d_codes = torch.zeros(nmb * MBCODE_DTYPE.itemsize, dtype=torch.uint8, device=dev)
        self.d_mbs = torch.zeros(nmb * DBK_MB_DTYPE.itemsize, dtype=torch.uint8, device=dev)
        self.slices = np.zeros(nslices, dtype=DBK_SLICE_DTYPE)  # every slice filtered, no offsets (enc/mod.rs:648)
        self.k = 0
        self.params = write_parameter_sets(width, height, bd, fps, refs, lib=self.lib, cabac=cabac, transform8=transform8)
        # called as before_p(encoder, d_y, stride) once a P picture's parameters are set and before it is
        # decided, on the encoder's stream (the learned form computes its proposals there)
        self.before_p = None

    def close(self) -> None:
        self.st.close()

    @staticmethod
    def _check(status: int, what: str) -> None:
        InterStage._check(status, what)

    def _up(self, dst, a: np.ndarray) -> None:
        dst.copy_(self.torch.from_numpy(np.ascontiguousarray(a).view(np.int16) if a.dtype == np.uint16 else np.ascontiguousarray(a)),
                  non_blocking=False)

    def encode(self, y: np.ndarray, cb: np.ndarray, cr: np.ndarray) -> bytes:
        """Codes a picture given as host arrays: its planes go up to the encoder's own device buffers first."""
        cur = self.d_src[self.k]
        with self.torch.cuda.stream(self.stream):
            self._up(cur, y)
            self._up(self.d_src_c[0], cb)
            self._up(self.d_src_c[1], cr)
        prev = self.d_src[self.k ^ 1].data_ptr() if self.loop.count > 0 else None
        self.k ^= 1
        return self.encode_device(cur.data_ptr(), self.d_src_c[0].data_ptr(), self.d_src_c[1].data_ptr(), self.st.width, prev)

    def encode_device(self, d_y: int, d_cb: int, d_cr: int, stride: int, d_prev_y: int | None) -> bytes:
        """Codes a picture already in device memory (luma width x height and chroma half that, rows `stride`
        and `stride // 2` samples apart, on or ordered before the encoder's stream); d_prev_y is the previous
        picture's luma for the scene-cut measure (None for the first). Returns the picture's Annex B bytes."""
        st, L, lib = self.st, self.loop, self.lib
        w = st.width
        cut = False
        if self.scene_cut and d_prev_y is not None:
            out = np.zeros(2, dtype=np.int64)
            self._check(lib.ironav_scene_change_device(st.ctx, d_prev_y, d_y, stride, out.ctypes.data), "ironav_scene_change_device")
            cut = float(out[0]) > SCENE_CUT * float(out[1])  # enc/mod.rs:707-711
        idr = L.choose(cut)
        st.set_source_device(d_y, stride)
        self._check(lib.ironav_set_source_chroma_device(st.ctx, d_cb, d_cr, stride // 2), "ironav_set_source_chroma_device")
        qpp = L.qp_prime(idr)
        pw, cw = st.mb_w * 16, st.mb_w * 8
        ry, rc, sts, codes = self.d_rec, self.d_rec_c, self.d_states, self.d_codes
        if idr:
            st.clear_references()
            st.begin_i_picture(qpp, fast=self.fast)
            self._check(lib.ironav_decide_i_picture_device(st.ctx, sts.data_ptr(), codes.data_ptr(), ry.data_ptr(), pw,
                                                           rc[0].data_ptr(), rc[1].data_ptr(), cw), "ironav_decide_i_picture_device")
            data = self.params + st.write_slices_device(True, L.frame_num, L.idr_id, codes.data_ptr())
        else:
            st.begin_p_picture(qpp, nrefs_active=min(L.held, L.nrefs), fast=self.fast, sub8=self.sub8)
            if self.before_p is not None:
                self.before_p(self, d_y, stride)
            self._check(lib.ironav_decide_p_picture_device(st.ctx, sts.data_ptr(), codes.data_ptr(), ry.data_ptr(), pw,
                                                           rc[0].data_ptr(), rc[1].data_ptr(), cw), "ironav_decide_p_picture_device")
            data = st.write_slices_device(False, L.frame_num, 0, codes.data_ptr())
        self._check(lib.ironav_decide_dbk_records_device(st.ctx, codes.data_ptr(), sts.data_ptr(), self.d_mbs.data_ptr()),
                    "ironav_decide_dbk_records_device")
        st.deblock_device(ry.data_ptr(), pw, rc[0].data_ptr(), rc[1].data_ptr(), cw, self.d_mbs.data_ptr(), self.slices)
        # the filtered picture becomes the newest reference: its planes and chroma are copied into the context
        st.push_reference_device(ry.data_ptr(), pw, pw, st.mb_h * 16, None if idr else sts.data_ptr())
        self._check(lib.ironav_push_reference_chroma_device(st.ctx, rc[0].data_ptr(), rc[1].data_ptr(), cw, cw, st.mb_h * 8),
                    "ironav_push_reference_chroma_device")
        st.sync()
        L.after(idr)
        return data

    def recon(self):
        """The last picture's filtered reconstruction (y, cb, cr) as host arrays."""
        self.st.sync()
        y = self.d_rec.cpu().numpy()
        c = self.d_rec_c.cpu().numpy()
        if self.loop.bd > 8:
            return y.view(np.uint16), c[0].view(np.uint16), c[1].view(np.uint16)
        return y, c[0], c[1]

    def codes(self) -> np.ndarray:
        self.st.sync()
        return self.d_codes.cpu().numpy().view(MBCODE_DTYPE)

    def states(self) -> np.ndarray:
        self.st.sync()
        return self.d_states.cpu().numpy().view(MBSTATE_DTYPE)
