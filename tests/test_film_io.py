"""Film output (lightmetrica_b200.film_io) on CPU: the reference
HDRBitmapFilm's naming rules (hdrfilm.cpp:204-240), its row order (film
row 0 = the image's bottom row, FreeImage scanline 0), Radiance RGBE
encoding known answers, and write/read round trips."""
import os

import numpy as np
import pytest

from lightmetrica_b200.film_io import (read_exr, read_hdr, read_pfm, resolve_output_path, rgbe_decode, rgbe_encode,
                                       save_film, write_pfm)
from lightmetrica_b200.scene import HDRBitmapFilm


def test_output_path_rules():
    assert resolve_output_path("", "radiancehdr") == "result.hdr"
    assert resolve_output_path("out", "radiancehdr") == "out.hdr"
    assert resolve_output_path("out", "openexr") == "out.exr"
    assert resolve_output_path("a/out.hdr", "radiancehdr") == "a/out.hdr"
    assert resolve_output_path("out.exr", "radiancehdr") == "result.hdr"
    assert resolve_output_path("out.png", "openexr") == "result.hdr"
    with pytest.raises(ValueError):
        resolve_output_path("x", "png")


def test_rgbe_known_answers():
    q = rgbe_encode(np.array([[1.0, 1.0, 1.0], [0.0, 0.0, 0.0], [0.5, 0.25, 0.0], [1e-40, 0, 0]]))
    np.testing.assert_array_equal(q, [[128, 128, 128, 129], [0, 0, 0, 0], [128, 64, 0, 128], [0, 0, 0, 0]])
    np.testing.assert_allclose(rgbe_decode(q)[0], [1.0 + 1 / 256] * 3, rtol=1e-7)


def test_hdr_round_trip_and_row_order(tmp_path):
    rng = np.random.default_rng(0)
    film = rng.uniform(0, 50, (5, 7, 3)).astype(np.float32)
    film[0, 0] = (100.0, 0.0, 0.0)              # row 0: the image's bottom row
    path = save_film(film, str(tmp_path / "img"), "radiancehdr")
    assert path.endswith("img.hdr")
    back = read_hdr(path)
    assert back.shape == film.shape
    # RGBE keeps 8 mantissa bits of the largest channel.
    assert np.all(np.abs(back - film) <= film.max(axis=-1, keepdims=True) / 128)
    raw = open(path, "rb").read()
    body = raw[raw.index(b"+X 7\n") + 5:]
    first_file_row = np.frombuffer(body, np.uint8, 4 * 7).reshape(7, 4)
    np.testing.assert_array_equal(first_file_row, rgbe_encode(film[4]))      # top row first in the file
    assert tuple(np.frombuffer(body, np.uint8)[-28:-24]) == tuple(rgbe_encode(film[0, :1])[0])


def test_hdr_reads_run_length_scanlines(tmp_path):
    W, H = 10, 2
    pix = np.zeros((H, W, 4), np.uint8)
    pix[..., 3] = 129
    pix[0, :, 0] = 128
    pix[1, :, 1] = np.arange(W) * 10
    data = b"#?RADIANCE\nFORMAT=32-bit_rle_rgbe\n\n-Y 2 +X 10\n"
    for y in range(H):
        data += bytes([2, 2, 0, W])
        for ch in range(4):
            vals = pix[y, :, ch]
            if np.all(vals == vals[0]):
                data += bytes([128 + W, int(vals[0])])
            else:
                data += bytes([W]) + vals.tobytes()
    p = tmp_path / "rle.hdr"
    p.write_bytes(data)
    img = read_hdr(str(p))
    np.testing.assert_allclose(img[1], rgbe_decode(pix[0]))    # file row 0 is the film's top row
    np.testing.assert_allclose(img[0], rgbe_decode(pix[1]))


def test_exr_and_pfm_round_trips(tmp_path):
    rng = np.random.default_rng(1)
    film = rng.uniform(-1, 1e4, (3, 9, 3)).astype(np.float32)
    p = save_film(film, str(tmp_path / "sub" / "img.exr"), "openexr", weight=0.5)
    assert os.path.exists(p)
    np.testing.assert_array_equal(read_exr(p), film * np.float32(0.5))
    write_pfm(str(tmp_path / "img.pfm"), film)
    np.testing.assert_array_equal(read_pfm(str(tmp_path / "img.pfm")), film)


def test_film_save_methods(tmp_path):
    f = HDRBitmapFilm(4, 2, image_type="openexr")
    f.internal_data()[:] = 2.0
    p = f.rescale_and_save(str(tmp_path / "r"), 0.25)
    assert p.endswith("r.exr")
    np.testing.assert_array_equal(read_exr(p), 0.5)
