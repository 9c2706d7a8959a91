"""Environment maps of glTF image-based lights (EXT_lights_image_based).

The reference resamples the first specular cube of the light into its
lat-long RGBA32F environment (src/scene.cpp:541-625) and decodes the faces
with stb_image's float loader (src/image_decode.cpp:51-88: Radiance HDR as is,
8-bit images with gamma 2.2).  Checked here: the Radiance decoder against
files written by a small encoder below (flat and run-length scanlines), the
cube conversion against an independent numpy restatement of the reference's
steps, and the glTF loader end to end.
"""
import base64
import json
import math

import numpy as np
import pytest

from crystalgraphics_b200 import backend as B
from crystalgraphics_b200 import png


def _rgbe(rgb):
    """Float RGB (h, w, 3) -> RGBE bytes (h, w, 4), the usual frexp rule."""
    rgb = np.asarray(rgb, np.float64)
    m = rgb.max(axis=-1)
    out = np.zeros(rgb.shape[:-1] + (4,), np.uint8)
    nz = m > 1e-32
    mant, exp = np.frexp(m[nz])
    scale = mant * 256.0 / m[nz]
    out[nz, :3] = np.clip(np.floor(rgb[nz] * scale[:, None]), 0, 255).astype(np.uint8)
    out[nz, 3] = (exp + 128).astype(np.uint8)
    return out


def _hdr_bytes(rgbe, rle):
    h, w, _ = rgbe.shape
    head = b"#?RADIANCE\n# written by the test\nFORMAT=32-bit_rle_rgbe\n\n" + \
        f"-Y {h} +X {w}\n".encode()
    body = bytearray()
    for y in range(h):
        if not rle:
            body += rgbe[y].tobytes()
            continue
        body += bytes([2, 2, w >> 8, w & 0xFF])
        for c in range(4):
            vals = rgbe[y, :, c]
            x = 0
            while x < w:  # runs of equal values, else literals (at most 128)
                run = 1
                while x + run < w and run < 127 and vals[x + run] == vals[x]:
                    run += 1
                if run >= 3:
                    body += bytes([128 + run, int(vals[x])])
                    x += run
                    continue
                lit = 1
                while x + lit < w and lit < 128 and not (
                        x + lit + 2 < w and vals[x + lit] == vals[x + lit + 1] == vals[x + lit + 2]):
                    lit += 1
                body += bytes([lit]) + vals[x:x + lit].tobytes()
                x += lit
    return head + bytes(body)


def _rgbe_to_float(rgbe):
    e = rgbe[..., 3].astype(np.int32)
    f = np.where(e == 0, 0.0, np.ldexp(1.0, e - 136)).astype(np.float32)
    out = np.ones(rgbe.shape[:-1] + (4,), np.float32)
    out[..., :3] = rgbe[..., :3].astype(np.float32) * f[..., None]
    return out


@pytest.mark.parametrize("w,h,rle", [(5, 3, False), (16, 4, False), (16, 4, True), (130, 2, True)])
def test_hdr_decode_flat_and_rle(w, h, rle):
    rng = np.random.default_rng(w * 7 + h)
    rgb = rng.lognormal(0.0, 2.0, (h, w, 3))
    rgb[:, : w // 3] = rgb[0, 0]          # a run for the run-length coder
    rgb[0, -1] = 0.0                      # exponent 0: black
    rgbe = _rgbe(rgb)
    img = B.hdr_decode(_hdr_bytes(rgbe, rle))
    assert img.shape == (h, w, 4)
    np.testing.assert_array_equal(img, _rgbe_to_float(rgbe))


@pytest.mark.parametrize("data", [b"", b"P6\n1 1\n255\n\0\0\0", b"#?RADIANCE\n\n-Y 1 +X 1\n\0\0\0\0",
                                  b"#?RADIANCE\nFORMAT=32-bit_rle_rgbe\n\n+Y 1 +X 1\n\0\0\0\0",
                                  b"#?RADIANCE\nFORMAT=32-bit_rle_rgbe\n\n-Y 2 +X 2\n\0\0\0\0"])
def test_hdr_decode_rejects_bad_files(data):
    with pytest.raises(B.Error):
        B.hdr_decode(data)


def _ref_env(faces, rot):
    """The reference's steps (CubeToEnvironmentTexture, SampleCube, ImageTexel,
    RotateVector, EngineToGltfDirection) in numpy float32, vectorised."""
    f32 = np.float32
    _, h, w, _ = faces.shape
    W, H = 4 * w, 2 * h
    pi = f32(math.pi)
    v = (np.arange(H, dtype=f32) + f32(0.5)) / f32(H)
    u = (np.arange(W, dtype=f32) + f32(0.5)) / f32(W)
    theta = (v * pi)[:, None]
    phi = ((u - f32(0.5)) * f32(2.0) * pi)[None, :]
    st, z = np.sin(theta), np.cos(theta)
    ex, ey, ez = np.cos(phi) * st, np.sin(phi) * st, np.broadcast_to(z, (H, W))
    d = np.stack([ex, -ez, ey], axis=-1).astype(f32)  # glTF direction
    q = np.array([-rot[0], -rot[1], -rot[2], rot[3]], f32)
    n = f32(q[0] * q[0] + q[1] * q[1] + q[2] * q[2]) + q[3] * q[3]
    if n > 0:  # a zero quaternion leaves the direction as it is
        im, re = q[:3] / np.sqrt(n), q[3] / np.sqrt(n)
        t = f32(2.0) * np.cross(im, d)
        d = (d + re * t + np.cross(im, t)).astype(f32)
    ax, ay, az = np.abs(d[..., 0]), np.abs(d[..., 1]), np.abs(d[..., 2])
    xm = (ax >= ay) & (ax >= az)
    ym = ~xm & (ay >= az)
    zm = ~xm & ~ym
    face = np.where(xm, np.where(d[..., 0] >= 0, 1, 0),
                    np.where(ym, np.where(d[..., 1] >= 0, 2, 3), np.where(d[..., 2] >= 0, 4, 5)))
    with np.errstate(divide="ignore", invalid="ignore"):
        s = np.where(xm, (np.where(d[..., 0] >= 0, -d[..., 2], d[..., 2]) / ax + 1) * f32(0.5),
                     np.where(ym, (d[..., 0] / ay + 1) * f32(0.5),
                              (np.where(d[..., 2] >= 0, d[..., 0], -d[..., 0]) / az + 1) * f32(0.5)))
        tt = np.where(xm, (-d[..., 1] / ax + 1) * f32(0.5),
                      np.where(ym, (np.where(d[..., 1] >= 0, d[..., 2], -d[..., 2]) / ay + 1) * f32(0.5),
                               (1 - d[..., 1] / az) * f32(0.5)))
    s = np.clip(f32(1) - s.astype(f32), 0, 1)
    tt = np.clip(f32(1) - tt.astype(f32), 0, 1)
    x = np.minimum(w - 1, (s * f32(w)).astype(np.int64))
    y = np.minimum(h - 1, (tt * f32(h)).astype(np.int64))
    out = faces[face, y, x].copy()
    out[..., 3] = 1.0
    return out


def _id_faces(w, h):
    """Faces whose texels hold their own (face, x, y) as exact floats."""
    f = np.zeros((6, h, w, 4), np.float32)
    for k in range(6):
        yy, xx = np.mgrid[0:h, 0:w]
        f[k, ..., 0] = k
        f[k, ..., 1] = xx
        f[k, ..., 2] = yy
    return f


@pytest.mark.parametrize("rot", [(0, 0, 0, 1), (0, math.sin(0.6), 0, math.cos(0.6)),
                                 (0.3, -0.2, 0.5, 0.7), (0, 0, 0, 0)])
def test_cube_to_lat_long_matches_the_reference_steps(rot):
    faces = _id_faces(16, 12)
    env = B.env_from_cube(faces, rot)
    ref = _ref_env(faces, np.array(rot, np.float32))
    assert env.shape == ref.shape == (24, 64, 4)
    same = np.all(env == ref, axis=-1)
    # numpy's and glibc's float sin/cos may differ by an ulp, which can move a
    # direction across a texel or face boundary; everywhere else the choice of
    # face and texel is the same
    assert same.mean() >= 0.99, same.mean()
    assert (env[..., 3] == 1).all()


def test_cube_directions_land_on_the_expected_faces():
    faces = _id_faces(8, 8)
    env = B.env_from_cube(faces)
    H, W = env.shape[:2]
    # engine z is up; glTF direction = (x, -z, y): engine +x -> +X face (1),
    # engine +y -> glTF +Z (4), engine up -> glTF -Y (3), down -> +Y (2)
    assert env[H // 2, W // 2, 0] == 1
    assert env[H // 2, 3 * W // 4, 0] == 4
    assert env[0, W // 2, 0] == 3
    assert env[H - 1, W // 2, 0] == 2
    assert env[H // 2, 0, 0] == 0 and env[H // 2, W // 4, 0] == 5


def _gltf_with_ibl(tmp_path, images, mime, rotation=None, sets=None):
    imgs = [{"uri": f"data:{mime};base64," + base64.b64encode(b).decode()} for b in images]
    light = {"specularImages": sets if sets is not None else [list(range(6))]}
    if rotation is not None:
        light["rotation"] = list(rotation)
    doc = {"asset": {"version": "2.0"}, "images": imgs,
           "extensionsUsed": ["EXT_lights_image_based"],
           "extensions": {"EXT_lights_image_based": {"lights": [light]}}}
    p = tmp_path / "ibl.gltf"
    p.write_text(json.dumps(doc))
    return p


def test_gltf_ibl_with_hdr_faces(tmp_path):
    rng = np.random.default_rng(3)
    rgbe = [_rgbe(rng.lognormal(0.0, 1.5, (8, 8, 3))) for _ in range(6)]
    rot = (0.1, 0.7, -0.2, 0.65)
    p = _gltf_with_ibl(tmp_path, [_hdr_bytes(e, True) for e in rgbe], "image/vnd.radiance", rot)
    s = B.parse_gltf(p)
    faces = np.stack([_rgbe_to_float(e) for e in rgbe])
    np.testing.assert_array_equal(s.env, B.env_from_cube(faces, rot))
    assert s.env.shape == (16, 32, 4)


def test_gltf_ibl_with_png_faces_uses_gamma_2_2(tmp_path):
    rng = np.random.default_rng(4)
    rgba = [rng.integers(0, 256, (6, 6, 4), dtype=np.uint8) for _ in range(6)]
    p = _gltf_with_ibl(tmp_path, [png.encode(a) for a in rgba], "image/png")
    s = B.parse_gltf(p)
    lin = np.stack([a.astype(np.float32) / np.float32(255.0) for a in rgba])
    lin[..., :3] = lin[..., :3] ** np.float32(2.2)
    np.testing.assert_allclose(s.env, B.env_from_cube(lin), rtol=3e-7, atol=0)


def test_gltf_ibl_errors_and_absence(tmp_path):
    one = png.encode(np.zeros((4, 4, 4), np.uint8))
    other = png.encode(np.zeros((4, 8, 4), np.uint8))
    with pytest.raises(B.Error, match="do not share one size"):
        B.parse_gltf(_gltf_with_ibl(tmp_path, [one] * 5 + [other], "image/png"))
    with pytest.raises(B.Error, match="invalid image"):
        B.parse_gltf(_gltf_with_ibl(tmp_path, [one] * 6, "image/png", sets=[[0, 1, 2, 3, 4, 9]]))
    # fewer than six images: no environment, as in the reference
    s = B.parse_gltf(_gltf_with_ibl(tmp_path, [one] * 6, "image/png", sets=[[0, 1, 2]]))
    assert s.env is None


def test_corrupt_hdr_files_fail_cleanly():
    rng = np.random.default_rng(8)
    seeds = [_hdr_bytes(_rgbe(rng.lognormal(0, 2, (4, 16, 3))), True),
             _hdr_bytes(_rgbe(rng.lognormal(0, 2, (3, 9, 3))), False)]
    for trial in range(400):  # errors are fine; a crash would end the test run
        d = bytearray(seeds[trial % 2])
        for _ in range(int(rng.integers(1, 6))):
            p = int(rng.integers(0, len(d)))
            d[p] = int(rng.integers(0, 256)) if rng.random() < 0.7 else d[p] ^ 1
        if trial % 3 == 0:
            d = d[: int(rng.integers(1, len(d)))]
        try:
            img = B.hdr_decode(bytes(d))
            assert img.ndim == 3 and img.shape[2] == 4
        except B.Error:
            pass
