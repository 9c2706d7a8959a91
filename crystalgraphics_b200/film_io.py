"""Film images on disk: binary PPM for the RGBA8 sRGB film and PFM for the
float films, the file forms of the headless viewer (cxx/view_main.cpp).

The reference writes its CPU debug view as an ASCII PPM (src/cpu_view.cpp:
146-154); a rendered film is presented in a window there, which has no
counterpart here, so the films are written to files instead.  PFM is the
Portable Float Map: a "PF" (3 channels) or "Pf" (1 channel) header, the size,
a scale whose sign gives the byte order (negative: little endian), then the
rows bottom first.
"""
from __future__ import annotations

import os
import re

import numpy as np


def save_ppm(path: str | os.PathLike, rgba8: np.ndarray) -> None:
    """Writes an (h, w, 3 or 4) uint8 film as a binary (P6) PPM; alpha is dropped."""
    img = np.asarray(rgba8)
    if img.dtype != np.uint8 or img.ndim != 3 or img.shape[2] not in (3, 4):
        raise ValueError("save_ppm wants an (h, w, 3|4) uint8 image")
    h, w = img.shape[:2]
    with open(path, "wb") as f:
        f.write(f"P6\n{w} {h}\n255\n".encode())
        f.write(np.ascontiguousarray(img[..., :3]).tobytes())


def load_ppm(path: str | os.PathLike) -> np.ndarray:
    """Reads a binary (P6, 8-bit) PPM as (h, w, 3) uint8."""
    data = open(path, "rb").read()
    fields, pos = [], 0
    while len(fields) < 4:  # magic, width, height, maxval; '#' comments allowed
        while data[pos:pos + 1].isspace():
            pos += 1
        if data[pos:pos + 1] == b"#":
            pos = data.index(b"\n", pos)
            continue
        end = pos
        while end < len(data) and not data[end:end + 1].isspace():
            end += 1
        fields.append(data[pos:end])
        pos = end
    if fields[0] != b"P6" or int(fields[3]) != 255:
        raise ValueError("not an 8-bit binary PPM")
    w, h = int(fields[1]), int(fields[2])
    pixels = np.frombuffer(data, np.uint8, w * h * 3, pos + 1)
    return pixels.reshape(h, w, 3).copy()


def save_pfm(path: str | os.PathLike, film: np.ndarray) -> None:
    """Writes an (h, w, 3) or (h, w) float32 film as a little-endian PFM, top row
    of the film last in the file (PFM stores rows bottom first)."""
    img = np.asarray(film)
    if img.dtype != np.float32 or not (img.ndim == 2 or (img.ndim == 3 and img.shape[2] == 3)):
        raise ValueError("save_pfm wants an (h, w, 3) or (h, w) float32 film")
    h, w = img.shape[:2]
    with open(path, "wb") as f:
        f.write(f"{'PF' if img.ndim == 3 else 'Pf'}\n{w} {h}\n-1.0\n".encode())
        f.write(np.ascontiguousarray(img[::-1]).astype("<f4").tobytes())


def load_pfm(path: str | os.PathLike) -> np.ndarray:
    """Reads a PFM of either byte order as float32, top row first."""
    data = open(path, "rb").read()
    head = re.match(rb"(P[Ff])\s+(\d+)\s+(\d+)\s+(\S+)\s", data)
    if not head:
        raise ValueError("not a PFM")
    w, h, scale = int(head[2]), int(head[3]), float(head[4])
    ch = 3 if head[1] == b"PF" else 1
    # the raster follows the single whitespace byte after the scale
    px = np.frombuffer(data, "<f4" if scale < 0 else ">f4", w * h * ch, head.end())
    img = px.astype(np.float32).reshape((h, w, 3) if ch == 3 else (h, w))
    return img[::-1].copy()
