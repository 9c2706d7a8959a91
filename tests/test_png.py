"""PNG decoding (cg_png_decode, used for glTF images): every colour type and bit
depth, the five scanline filters, Adam7 interlacing, stored / fixed / dynamic
DEFLATE blocks, and tRNS transparency, against the expected RGBA8 (8-bit
expansion as stb_image does it: 16-bit keeps the high byte, low-depth grey is
scaled to 0..255)."""
import struct
import zlib

import numpy as np
import pytest

from crystalgraphics_b200 import backend as B
from crystalgraphics_b200 import png


def _expand_grey(g, depth):
    if depth == 16:
        return (g >> 8).astype(np.uint8)
    return (g.astype(np.uint32) * 255 // ((1 << depth) - 1)).astype(np.uint8)


@pytest.mark.parametrize("interlace", [False, True])
@pytest.mark.parametrize("filter_type", [0, 1, 2, 3, 4, -1])
def test_rgba8_filters_and_interlace(interlace, filter_type):
    rng = np.random.default_rng(filter_type + 2 + 10 * interlace)
    img = rng.integers(0, 256, (13, 17, 4), dtype=np.uint8)
    img[3:7, 2:9] = (200, 10, 30, 255)  # runs the compressor turns into matches
    out = B.png_decode(png.encode(img, png.RGBA, 8, filter_type=filter_type, interlace=interlace))
    assert np.array_equal(out, img)


@pytest.mark.parametrize("level", [0, 1, 9])
def test_deflate_block_kinds(level):
    """level 0: stored blocks; 1 and 9: Huffman blocks (fixed and dynamic)."""
    rng = np.random.default_rng(level)
    img = np.repeat(rng.integers(0, 256, (40, 1, 4), dtype=np.uint8), 70, axis=1)
    img[::3, ::5] = rng.integers(0, 256, img[::3, ::5].shape, dtype=np.uint8)
    out = B.png_decode(png.encode(img, png.RGBA, 8, filter_type=-1, level=level))
    assert np.array_equal(out, img)


@pytest.mark.parametrize("depth", [1, 2, 4, 8, 16])
def test_grey_depths(depth):
    rng = np.random.default_rng(depth)
    g = rng.integers(0, 1 << depth, (9, 23), dtype=np.uint32)
    out = B.png_decode(png.encode(g[..., None], png.GREY, depth, filter_type=-1))
    e = _expand_grey(g, depth)
    assert np.array_equal(out[..., 0], e) and np.array_equal(out[..., 2], e)
    assert (out[..., 3] == 255).all()


@pytest.mark.parametrize("depth", [8, 16])
def test_rgb_and_grey_alpha(depth):
    rng = np.random.default_rng(depth + 1)
    rgb = rng.integers(0, 1 << depth, (7, 11, 3), dtype=np.uint32)
    out = B.png_decode(png.encode(rgb, png.RGB, depth, filter_type=4, interlace=True))
    assert np.array_equal(out[..., :3], _expand_grey(rgb, depth))
    assert (out[..., 3] == 255).all()
    ga = rng.integers(0, 1 << depth, (5, 6, 2), dtype=np.uint32)
    out = B.png_decode(png.encode(ga, png.GREY_ALPHA, depth, filter_type=3))
    assert np.array_equal(out[..., 0], _expand_grey(ga[..., 0], depth))
    assert np.array_equal(out[..., 3], _expand_grey(ga[..., 1], depth))


@pytest.mark.parametrize("depth", [1, 2, 4, 8])
def test_palette_with_transparency(depth):
    rng = np.random.default_rng(depth + 2)
    n = 1 << depth
    pal = rng.integers(0, 256, (n, 3), dtype=np.uint8)
    alpha = rng.integers(0, 256, max(1, n // 2), dtype=np.uint8)  # tRNS may be short
    idx = rng.integers(0, n, (10, 13), dtype=np.uint32)
    out = B.png_decode(png.encode(idx[..., None], png.PALETTE, depth, palette=pal,
                                  trns=alpha.tobytes(), filter_type=-1, interlace=depth == 4))
    assert np.array_equal(out[..., :3], pal[idx])
    full_alpha = np.concatenate([alpha, np.full(n - len(alpha), 255, np.uint8)])
    assert np.array_equal(out[..., 3], full_alpha[idx])


def test_rgb_colour_key():
    rgb = np.zeros((4, 4, 3), np.uint32)
    rgb[1, 2] = (10, 20, 30)
    out = B.png_decode(png.encode(rgb, png.RGB, 8, trns=bytes([0, 10, 0, 20, 0, 30])))
    assert out[1, 2, 3] == 0 and out[0, 0, 3] == 255


def test_jpeg_and_garbage_are_rejected():
    with pytest.raises(B.Error) as e:
        B.png_decode(b"\xff\xd8\xff\xe0" + b"\0" * 32)
    assert "JPEG" in str(e.value)
    with pytest.raises(B.Error):
        B.png_decode(b"not an image at all")
    good = png.encode_rgba8(np.zeros((3, 3, 4), np.uint8))
    with pytest.raises(B.Error):
        B.png_decode(good[: len(good) - 30])  # truncated stream


def _chunks(data):
    p, out = 8, []
    while p + 8 <= len(data):
        n = struct.unpack(">I", data[p:p + 4])[0]
        out.append([data[p + 4:p + 8], bytearray(data[p + 8:p + 8 + n])])
        p += 12 + n
    return out


def _assemble(chunks):
    out = b"\x89PNG\r\n\x1a\n"
    for kind, body in chunks:
        out += struct.pack(">I", len(body)) + kind + bytes(body) + struct.pack(">I", zlib.crc32(kind + bytes(body)))
    return out


@pytest.mark.parametrize("color_type,depth", [(png.RGBA, 8), (png.RGB, 16), (png.PALETTE, 4), (png.GREY, 1)])
def test_corrupt_pngs_with_valid_checksums_fail_cleanly(color_type, depth):
    """Header fields, palette / transparency lengths and scanline bytes changed
    with the chunk CRCs and the zlib stream kept valid, so that the checks
    after decompression are what reject them (or the image decodes)."""
    rng = np.random.default_rng(depth)
    ch = {png.RGBA: 4, png.RGB: 3, png.PALETTE: 1, png.GREY: 1}[color_type]
    samples = rng.integers(0, 1 << depth, (9, 13, ch))
    pal = rng.integers(0, 256, (16, 3)) if color_type == png.PALETTE else None
    trns = rng.integers(0, 256, 5) if color_type == png.PALETTE else None
    chunks = _chunks(png.encode(samples, color_type, depth, palette=pal, trns=trns, interlace=depth == 4))
    raw0 = zlib.decompress(b"".join(bytes(b) for k, b in chunks if k == b"IDAT"))
    head = [c for c in chunks if c[0] not in (b"IDAT", b"IEND")]
    for _ in range(150):  # errors are fine; a crash would end the test run
        cs = [[k, bytearray(b)] for k, b in head]
        for k, b in cs:
            if k == b"IHDR" and rng.random() < 0.6:
                f = int(rng.integers(0, 13))
                b[f] = int(rng.integers(0, 256)) if f >= 8 else b[f] ^ (1 << int(rng.integers(0, 8)))
            if k in (b"PLTE", b"tRNS") and rng.random() < 0.3:
                del b[int(rng.integers(0, len(b) + 1)):]
        raw = bytearray(raw0)
        for _ in range(int(rng.integers(0, 4))):
            p = int(rng.integers(0, len(raw)))
            if rng.random() < 0.5:
                raw[p] = int(rng.integers(0, 256))
            else:
                del raw[p:p + int(rng.integers(1, 20))]
        data = _assemble(cs + [[b"IDAT", zlib.compress(bytes(raw))], [b"IEND", b""]])
        try:
            out = B.png_decode(data)
            assert out.ndim == 3 and out.shape[2] == 4
        except B.Error:
            pass
