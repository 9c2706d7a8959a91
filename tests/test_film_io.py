"""Film files (crystalgraphics_b200/film_io.py): binary PPM of the RGBA8 film
and PFM of the float films.  The viewer's own files are checked against the
device films in tests/test_gpu_forms.py."""
import numpy as np
import pytest

from crystalgraphics_b200 import film_io


def test_ppm_round_trip(tmp_path):
    rng = np.random.default_rng(0)
    rgba = rng.integers(0, 256, (7, 11, 4), dtype=np.uint8)
    film_io.save_ppm(tmp_path / "a.ppm", rgba)
    data = (tmp_path / "a.ppm").read_bytes()
    assert data.startswith(b"P6\n11 7\n255\n") and len(data) == 12 + 7 * 11 * 3
    np.testing.assert_array_equal(film_io.load_ppm(tmp_path / "a.ppm"), rgba[..., :3])


def test_ppm_reader_skips_comments(tmp_path):
    px = np.arange(2 * 3 * 3, dtype=np.uint8).reshape(2, 3, 3)
    (tmp_path / "c.ppm").write_bytes(b"P6\n# a comment\n3 2\n255\n" + px.tobytes())
    np.testing.assert_array_equal(film_io.load_ppm(tmp_path / "c.ppm"), px)


@pytest.mark.parametrize("shape", [(5, 9, 3), (4, 6)])
def test_pfm_round_trip_is_exact_and_bottom_up(tmp_path, shape):
    rng = np.random.default_rng(1)
    film = rng.lognormal(0, 3, shape).astype(np.float32)
    film.reshape(-1)[:3] = [0.0, np.inf, 1e-40]  # zero, infinity, a subnormal
    film_io.save_pfm(tmp_path / "a.pfm", film)
    data = (tmp_path / "a.pfm").read_bytes()
    h, w = shape[:2]
    head = f"{'PF' if len(shape) == 3 else 'Pf'}\n{w} {h}\n-1.0\n".encode()
    assert data.startswith(head)
    # the first row in the file is the film's bottom row
    row = w * (3 if len(shape) == 3 else 1)
    np.testing.assert_array_equal(np.frombuffer(data, "<f4", row, len(head)), film[-1].reshape(-1))
    assert film_io.load_pfm(tmp_path / "a.pfm").tobytes() == film.tobytes()


def test_pfm_big_endian_files_read(tmp_path):
    film = np.arange(12, dtype=np.float32).reshape(2, 2, 3)
    (tmp_path / "b.pfm").write_bytes(b"PF\n2 2\n1.0\n" + film[::-1].astype(">f4").tobytes())
    np.testing.assert_array_equal(film_io.load_pfm(tmp_path / "b.pfm"), film)


def test_writers_reject_wrong_films(tmp_path):
    with pytest.raises(ValueError):
        film_io.save_ppm(tmp_path / "x.ppm", np.zeros((2, 2, 3), np.float32))
    with pytest.raises(ValueError):
        film_io.save_pfm(tmp_path / "x.pfm", np.zeros((2, 2, 4), np.float32))
    (tmp_path / "y.pfm").write_bytes(b"P6\n1 1\n255\n\0\0\0")
    with pytest.raises(ValueError):
        film_io.load_pfm(tmp_path / "y.pfm")
