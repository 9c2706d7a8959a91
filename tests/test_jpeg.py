"""JPEG decoding of glTF images (cg_jpeg.cpp), against libjpeg through Pillow.

The reference decodes glTF images with stb_image; this library's decoder
follows ITU-T T.81.  Its samples may differ from other decoders' by a level
or two (IDCT and colour-conversion rounding), so the comparison allows that
much, and more for the sampling ratios whose chroma this decoder replicates
(4:1:1, 4:4:0) where libjpeg interpolates.
"""
import base64
import io
import json

import numpy as np
import pytest

from crystalgraphics_b200 import backend as B

PIL = pytest.importorskip("PIL.Image")


def _image(h, w, seed):
    rng = np.random.default_rng(seed)
    y, x = np.mgrid[0:h, 0:w]
    img = np.stack([(x * 3 + y) % 256, (y * 4) % 256, ((x + y) * 2) % 256], -1)
    img = img + rng.integers(-24, 24, img.shape)
    return np.clip(img, 0, 255).astype(np.uint8)


def _pil_jpeg(img, **kw):
    buf = io.BytesIO()
    PIL.fromarray(img).save(buf, "JPEG", **kw)
    return buf.getvalue()


def _libjpeg(data, mode="RGB"):
    return np.asarray(PIL.open(io.BytesIO(data)).convert(mode))


@pytest.mark.parametrize("h,w", [(1, 1), (7, 9), (17, 33), (64, 48), (101, 3)])
@pytest.mark.parametrize("subsampling", [0, 1, 2])
@pytest.mark.parametrize("progressive", [False, True])
def test_colour_jpegs_match_libjpeg(h, w, subsampling, progressive):
    img = _image(h, w, h * 31 + w)
    data = _pil_jpeg(img, quality=88, subsampling=subsampling, progressive=progressive)
    got = B.jpeg_decode(data)
    assert got.shape == (h, w, 4) and (got[..., 3] == 255).all()
    d = np.abs(got[..., :3].astype(int) - _libjpeg(data).astype(int))
    # libjpeg replicates subsampled chroma (both ways) when the chroma is at
    # most 2 samples wide; this decoder, like stb_image, filters every plane
    # wider than 1 sample, so on such narrow noisy images only the means agree
    if subsampling > 0 and (w + 1) // 2 <= 2:
        assert d.mean() <= 4.0, d.mean()
    else:
        assert d.max() <= 4 and d.mean() <= 0.5, (d.max(), d.mean())


@pytest.mark.parametrize("quality", [10, 50, 100])
def test_quality_extremes(quality):
    img = _image(40, 56, quality)
    data = _pil_jpeg(img, quality=quality, subsampling=2)
    d = np.abs(B.jpeg_decode(data)[..., :3].astype(int) - _libjpeg(data).astype(int))
    assert d.max() <= 4 and d.mean() <= 0.5, (d.max(), d.mean())


def test_grey_jpeg():
    g = _image(30, 45, 5)[..., 0]
    buf = io.BytesIO()
    PIL.fromarray(g, "L").save(buf, "JPEG", quality=90)
    data = buf.getvalue()
    got = B.jpeg_decode(data)
    ref = _libjpeg(data, "L")
    assert (got[..., 0] == got[..., 1]).all() and (got[..., 1] == got[..., 2]).all()
    assert np.abs(got[..., 0].astype(int) - ref.astype(int)).max() <= 2


def test_rgb_jpeg_with_adobe_marker():
    img = _image(24, 32, 6)
    try:
        data = _pil_jpeg(img, quality=92, keep_rgb=True, subsampling=0)
    except TypeError:
        pytest.skip("this Pillow cannot write RGB JPEGs")
    d = np.abs(B.jpeg_decode(data)[..., :3].astype(int) - _libjpeg(data).astype(int))
    assert d.max() <= 2


cv2 = pytest.importorskip("cv2")


def _cv2_jpeg(img, params):
    ok, enc = cv2.imencode(".jpg", img[..., ::-1], params)
    assert ok
    return enc.tobytes()


@pytest.mark.parametrize("interval", [1, 3, 17])
@pytest.mark.parametrize("progressive", [0, 1])
def test_restart_intervals(interval, progressive):
    img = _image(50, 70, interval)
    data = _cv2_jpeg(img, [cv2.IMWRITE_JPEG_QUALITY, 90, cv2.IMWRITE_JPEG_RST_INTERVAL, interval,
                           cv2.IMWRITE_JPEG_PROGRESSIVE, progressive])
    assert b"\xff\xdd" in data  # a restart interval was written
    d = np.abs(B.jpeg_decode(data)[..., :3].astype(int) - _libjpeg(data).astype(int))
    assert d.max() <= 4 and d.mean() <= 0.5, (d.max(), d.mean())


@pytest.mark.parametrize("factor", ["411", "440"])
def test_other_sampling_ratios(factor):
    y, x = np.mgrid[0:48, 0:64]
    smooth = np.stack([x * 4, y * 5, (x + y) * 2], -1).clip(0, 255).astype(np.uint8)
    code = getattr(cv2, f"IMWRITE_JPEG_SAMPLING_FACTOR_{factor}")
    data = _cv2_jpeg(smooth, [cv2.IMWRITE_JPEG_QUALITY, 95, cv2.IMWRITE_JPEG_SAMPLING_FACTOR, code])
    d = np.abs(B.jpeg_decode(data)[..., :3].astype(int) - _libjpeg(data).astype(int))
    assert d.mean() <= 2.0, d.mean()


def test_corrupt_jpegs_fail_cleanly():
    data = bytearray(_pil_jpeg(_image(32, 40, 9), quality=80, progressive=True))
    rng = np.random.default_rng(1)
    for trial in range(300):  # errors are fine; a crash would end the test run
        d = bytearray(data)
        for _ in range(int(rng.integers(1, 6))):
            d[int(rng.integers(2, len(d)))] = int(rng.integers(0, 256))
        if trial % 3 == 0:
            d = d[: int(rng.integers(2, len(d)))]
        try:
            out = B.jpeg_decode(bytes(d))
            assert out.ndim == 3 and out.shape[2] == 4
        except B.Error:
            pass
    for bad in (b"", b"\xff\xd8", b"\xff\xd8\xff\xd9", b"\x89PNG\r\n\x1a\n"):
        with pytest.raises(B.Error):
            B.jpeg_decode(bad)


def test_gltf_jpeg_texture_and_ibl_faces(tmp_path):
    tex = _image(16, 16, 11)
    tex_jpg = _pil_jpeg(tex, quality=90)
    face_jpgs = [_pil_jpeg(_image(8, 8, 20 + k), quality=95) for k in range(6)]
    uri = lambda b: "data:image/jpeg;base64," + base64.b64encode(b).decode()  # noqa: E731
    doc = {"asset": {"version": "2.0"},
           "images": [{"uri": uri(tex_jpg)}] + [{"uri": uri(b)} for b in face_jpgs],
           "textures": [{"source": 0}],
           "materials": [{"pbrMetallicRoughness": {"baseColorTexture": {"index": 0}}}],
           "extensionsUsed": ["EXT_lights_image_based"],
           "extensions": {"EXT_lights_image_based": {"lights": [{"specularImages": [[1, 2, 3, 4, 5, 6]]}]}}}
    p = tmp_path / "jpeg.gltf"
    p.write_text(json.dumps(doc))
    s = B.parse_gltf(p)
    assert len(s.textures) == 1
    np.testing.assert_array_equal(s.textures[0][0], B.jpeg_decode(tex_jpg))
    faces = np.stack([B.jpeg_decode(b).astype(np.float32) / np.float32(255.0) for b in face_jpgs])
    faces[..., :3] = faces[..., :3] ** np.float32(2.2)
    np.testing.assert_allclose(s.env, B.env_from_cube(faces), rtol=3e-7, atol=0)
