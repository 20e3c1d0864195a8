"""Host check of stratified_raster's pixel index (csrc/pathtrace.cuh).

The kernels find pixel = sample mod (W*H) from a double-precision quotient
estimate, trunc(double(sample) * (1 / double(pixels))), corrected by one
step. For sample < 2^53 and pixels < 2^31 (the render entry points check
both) this must equal the 64-bit integer remainder. numpy's float64
multiply and truncation round like the device's, so the same steps are
restated here and compared with Python's exact remainder, including the
edges of both ranges.
"""
import numpy as np


def pixel_index(sample: np.ndarray, pixels: int) -> np.ndarray:
    inv = 1.0 / float(pixels)
    q = (sample.astype(np.float64) * inv).astype(np.int64)
    pix = sample - q * pixels
    pix = np.where(pix < 0, pix + pixels, pix)
    return np.where(pix >= pixels, pix - pixels, pix)


def test_pixel_index_equals_integer_remainder():
    rng = np.random.default_rng(3)
    limit = 1 << 53
    pixel_counts = [1, 2, 3, 7, 1920 * 1080, 4096 * 2160, 512 * 512, (1 << 31) - 1, (1 << 31) - 3, 65537, 999_983]
    pixel_counts += [int(x) for x in rng.integers(1, 1 << 31, size=40)]
    for p in pixel_counts:
        s = np.concatenate([
            rng.integers(0, limit, size=20000, dtype=np.int64),
            rng.integers(0, 1 << 32, size=2000, dtype=np.int64),
            np.arange(0, 3000, dtype=np.int64),
            limit - 1 - np.arange(0, 3000, dtype=np.int64),
            # around multiples of the pixel count, where a quotient estimate
            # off by one shows
            (rng.integers(1, limit // p, size=3000, dtype=np.int64) * p)[:, None] + np.array([-1, 0, 1])[None, :],
        ], axis=None)
        s = s[(s >= 0) & (s < limit)]
        want = np.array([int(x) % p for x in s], dtype=np.int64)
        np.testing.assert_array_equal(pixel_index(s, p), want, err_msg=f"pixels={p}")
