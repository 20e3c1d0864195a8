"""The oracle's path-tracer restatement (lmoracle_pt.c, double) against the
reference's own double-precision renders, and its FP64 gradient against
central differences of itself."""
import os

import numpy as np
import pytest

import oracle
from lightmetrica_b200 import scenes
from lightmetrica_b200.diff import light_emission, triangle_albedo


def relmse(x, r):
    return float(np.mean((x - r) ** 2 / (r ** 2 + 1e-2)))


@pytest.mark.parametrize("technique", ["pt.mis", "pt.direct"])
def test_oracle_image_matches_reference_image(golden_dir, technique):
    ref = np.load(os.path.join(golden_dir, "cornell_classic_ref_mis.npz"))["film"]
    img = oracle.oracle_render(scenes.cornell_box(128, 128), technique, spp=256, rr_depth=3, max_path_vertices=9,
                               seed=5)
    # 256 spp: Monte Carlo noise of about 2.6e-3 relMSE (measured 1.8e-3).
    assert relmse(img, ref) < 4e-3
    np.testing.assert_allclose(img.mean(axis=(0, 1)), ref.mean(axis=(0, 1)), rtol=5e-3)


def test_oracle_gradient_matches_fp64_central_differences():
    """With Russian roulette off (rr_depth -1) the estimator is a smooth
    function of the parameters for fixed random numbers, and its gradient
    must match central differences to rounding. (With Russian roulette on,
    the gradient holds the roulette probabilities at their sampled values:
    an unbiased estimate of the gradient of the expected image, which
    per-seed finite differences do not measure.)"""
    rr_depth, tol = -1, 1e-4
    prims = scenes.cornell_box(16, 16)
    alb0 = triangle_albedo(prims).astype(np.float64)
    le0 = light_emission(prims).astype(np.float64)
    kw = dict(technique="pt.mis", spp=16, rr_depth=rr_depth, max_path_vertices=9, seed=3, threads=4)
    target = oracle.oracle_render(prims, tri_albedo=alb0 * 0.7, **kw)

    def loss(a, le):
        return float(((oracle.oracle_render(prims, tri_albedo=a, light_Le=le, **kw) - target) ** 2).sum())

    img = oracle.oracle_render(prims, tri_albedo=alb0, **kw)
    ga, gl = oracle.oracle_grad(prims, 2 * (img - target), tri_albedo=alb0, **kw)
    h = 1e-4
    for tri, c in [(6, 0), (8, 1), (2, 2)]:      # red wall, green wall, back wall
        d = np.zeros_like(alb0)
        d[tri, c] = 1.0
        # parameters reach the oracle as float32: use the rounded step
        step = float(np.float32(alb0[tri, c] + h)) - float(np.float32(alb0[tri, c] - h))
        fd = (loss(alb0 + h * d, le0) - loss(alb0 - h * d, le0)) / step
        assert abs(ga[tri, c] - fd) <= tol * abs(fd), (tri, c, ga[tri, c], fd)
    for c in range(3):
        d = np.zeros_like(le0)
        d[0, c] = 1.0
        step = float(np.float32(le0[0, c] + h)) - float(np.float32(le0[0, c] - h))
        fd = (loss(alb0, le0 + h * d) - loss(alb0, le0 - h * d)) / step
        assert abs(gl[0, c] - fd) <= tol * abs(fd), (c, gl[0, c], fd)
