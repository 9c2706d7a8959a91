"""A small PNG encoder (zlib from the standard library), used to write glTF
images and to make PNG test inputs of every colour type, bit depth, filter and
interlace mode the library's decoder (cg_png_decode) reads."""
from __future__ import annotations

import struct
import zlib

import numpy as np

# colour types
GREY, RGB, PALETTE, GREY_ALPHA, RGBA = 0, 2, 3, 4, 6
_CHANNELS = {GREY: 1, RGB: 3, PALETTE: 1, GREY_ALPHA: 2, RGBA: 4}
_ADAM7 = [(0, 0, 8, 8), (4, 0, 8, 8), (0, 4, 4, 8), (2, 0, 4, 4), (0, 2, 2, 4), (1, 0, 2, 2),
          (0, 1, 1, 2)]


def _chunk(kind: bytes, body: bytes) -> bytes:
    return struct.pack(">I", len(body)) + kind + body + struct.pack(">I", zlib.crc32(kind + body))


def _pack_rows(samples: np.ndarray, depth: int) -> np.ndarray:
    """(h, w*channels) samples -> (h, stride) bytes at `depth` bits."""
    h = samples.shape[0]
    if depth == 8:
        return samples.astype(np.uint8)
    if depth == 16:
        s = samples.astype(">u2")
        return s.view(np.uint8).reshape(h, -1)
    per = 8 // depth
    n = samples.shape[1]
    stride = (n * depth + 7) // 8
    out = np.zeros((h, stride), np.uint8)
    for i in range(n):
        out[:, i // per] |= (samples[:, i].astype(np.uint8) << (8 - depth * (i % per + 1))).astype(np.uint8)
    return out


def _filter(rows: np.ndarray, bpp: int, ftype: int) -> bytes:
    out = bytearray()
    prev = np.zeros(rows.shape[1], np.int32)
    for r in rows.astype(np.int32):
        ft = ftype if ftype >= 0 else (len(out) // max(rows.shape[1] + 1, 1)) % 5
        a = np.concatenate([np.zeros(bpp, np.int32), r[:-bpp]]) if bpp < len(r) else np.zeros_like(r)
        c = np.concatenate([np.zeros(bpp, np.int32), prev[:-bpp]]) if bpp < len(r) else np.zeros_like(r)
        b = prev
        if ft == 0:
            f = r
        elif ft == 1:
            f = r - a
        elif ft == 2:
            f = r - b
        elif ft == 3:
            f = r - (a + b) // 2
        else:
            p = a + b - c
            pa, pb, pc = np.abs(p - a), np.abs(p - b), np.abs(p - c)
            pred = np.where((pa <= pb) & (pa <= pc), a, np.where(pb <= pc, b, c))
            f = r - pred
        out.append(ft)
        out += (f & 255).astype(np.uint8).tobytes()
        prev = r
    return bytes(out)


def encode(samples: np.ndarray, color_type: int = RGBA, depth: int = 8, palette=None, trns=None,
           filter_type: int = 0, interlace: bool = False, level: int = 6) -> bytes:
    """samples: (h, w, channels) integer samples at `depth` bits (palette:
    indices).  filter_type -1 cycles through the five filters row by row."""
    samples = np.asarray(samples)
    if samples.ndim == 2:
        samples = samples[..., None]
    h, w, ch = samples.shape
    assert ch == _CHANNELS[color_type]
    bpp = max(1, ch * depth // 8)
    raw = bytearray()
    passes = _ADAM7 if interlace else [(0, 0, 1, 1)]
    for x0, y0, dx, dy in passes:
        sub = samples[y0::dy, x0::dx]
        if sub.size == 0:
            continue
        rows = _pack_rows(sub.reshape(sub.shape[0], -1), depth)
        raw += _filter(rows, bpp, filter_type)
    out = b"\x89PNG\r\n\x1a\n"
    out += _chunk(b"IHDR", struct.pack(">IIBBBBB", w, h, depth, color_type, 0, 0, 1 if interlace else 0))
    if palette is not None:
        out += _chunk(b"PLTE", np.asarray(palette, np.uint8).tobytes())
    if trns is not None:
        out += _chunk(b"tRNS", bytes(trns))
    data = zlib.compress(bytes(raw), level)
    # split the stream over two IDAT chunks (decoders must concatenate them)
    half = len(data) // 2
    out += _chunk(b"IDAT", data[:half]) + _chunk(b"IDAT", data[half:])
    out += _chunk(b"IEND", b"")
    return out


def encode_rgba8(img: np.ndarray) -> bytes:
    """An (h, w, 4) uint8 image as an RGBA8 PNG."""
    return encode(np.asarray(img, np.uint8), RGBA, 8)
