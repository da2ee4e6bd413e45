"""Decoding Annex B streams with a decoder that is not this project's: OpenCV's bundled FFmpeg (cv2 4.13,
libavcodec 62.11) through cv2.VideoCapture (test infrastructure).

With CAP_PROP_CONVERT_RGB off, OpenCV hands back plane 0 of a decoded yuv420p frame unconverted: the luma,
byte for byte. Chroma comes back only through swscale's conversion to BGR, so it is checked by converting
the encoder's reconstruction (written as a Y4M file, which FFmpeg reads as yuv420p) the same way and
comparing the BGR pictures: with the luma already equal, equal BGR pins both chroma planes but for samples
the conversion clips."""
from __future__ import annotations

import os

import numpy as np


def _capture(path: str, raw: bool):
    import cv2

    cap = cv2.VideoCapture(path, cv2.CAP_FFMPEG)
    assert cap.isOpened(), f"FFmpeg cannot open {path}"
    if raw:
        cap.set(cv2.CAP_PROP_CONVERT_RGB, 0)
    frames = []
    while True:
        ok, fr = cap.read()
        if not ok:
            break
        frames.append(fr.copy())
    cap.release()
    return frames


def decode_luma(path: str) -> list[np.ndarray]:
    """Every decoded picture's luma (height x width, uint8) in output order."""
    return _capture(path, raw=True)


def decode_bgr(path: str) -> list[np.ndarray]:
    return _capture(path, raw=False)


def write_y4m(path: str, pictures, width: int, height: int, fps: tuple[int, int] = (30, 1)) -> None:
    """Pictures (y, cb, cr) cropped to width x height as a 4:2:0 Y4M file."""
    with open(path, "wb") as f:
        f.write(f"YUV4MPEG2 W{width} H{height} F{fps[0]}:{fps[1]} Ip A1:1 C420mpeg2\n".encode())
        for y, cb, cr in pictures:
            f.write(b"FRAME\n")
            f.write(np.ascontiguousarray(y[:height, :width], dtype=np.uint8).tobytes())
            f.write(np.ascontiguousarray(cb[: height // 2, : width // 2], dtype=np.uint8).tobytes())
            f.write(np.ascontiguousarray(cr[: height // 2, : width // 2], dtype=np.uint8).tobytes())


def check_stream_decodes_to(tmpdir: str, name: str, stream: bytes, recons, width: int, height: int) -> None:
    """Asserts that FFmpeg decodes `stream` to the pictures `recons` ((y, cb, cr), macroblock-aligned, in
    coding order = output order): the luma byte for byte, the chroma through equal BGR conversions."""
    path = os.path.join(tmpdir, name + ".h264")
    with open(path, "wb") as f:
        f.write(stream)
    got = decode_luma(path)
    assert len(got) == len(recons), f"{name}: FFmpeg decoded {len(got)} pictures of {len(recons)}"
    for t, (g, r) in enumerate(zip(got, recons)):
        want = r[0][:height, :width]
        assert g.shape == want.shape, f"{name} picture {t}: decoded {g.shape}, expected {want.shape}"
        bad = np.argwhere(g != want)
        assert len(bad) == 0, f"{name} picture {t}: luma differs at {len(bad)} samples, first {bad[:3].tolist()}"
    ypath = os.path.join(tmpdir, name + "_recon.y4m")
    write_y4m(ypath, recons, width, height)
    a, b = decode_bgr(path), decode_bgr(ypath)
    assert len(a) == len(b) == len(recons)
    for t, (x, y) in enumerate(zip(a, b)):
        assert np.array_equal(x, y), f"{name} picture {t}: chroma differs (BGR conversions differ at {int((x != y).sum())} samples)"
