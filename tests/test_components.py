"""The oracle's sampling, camera and BSDF restatements (lmoracle_pt.c) against
the reference's own component tests. The expected values restate the cited
assertions; the camera tests load "PerspectiveCameraNode_Success" (fovy 90,
test.perspectivecamera.cpp:38-43) over the tests' stub film of 200 x 100
(stub.film.h:38-39), and a primitive's transform is the camera's view matrix.
"""
import math

import numpy as np
import pytest

import oracle

S2, S3 = math.sqrt(2.0), math.sqrt(3.0)

# test.math.stats.cpp:34-61 (UniformConcentricDiskSample)
DISK = [((0.5, 0.5), (0, 0)), ((1, 0.5), (1, 0)), ((0.5, 1), (0, 1)), ((0, 0.5), (-1, 0)), ((0.5, 0), (0, -1))]
# test.math.stats.cpp:63-84 (CosineSampleHemisphere; its loop checks the first
# row of three; all three rows hold)
COSINE = [((0.5, 0.5), (0, 0, 1)), ((1, 0.5), (1, 0, 0)), ((0.75, 0.75), (S2 / 4, S2 / 4, S3 / 2))]

FILM = (200, 100)
FOVY = 90.0
# Primitive transforms of the camera tests as (eye, center, up): Identity,
# and LookAt(Vec3(1), Vec3(0), Vec3(0, 0, 1)).
CAMERAS = {"identity": ((0, 0, 0), (0, 0, -1), (0, 1, 0)), "lookat": ((1, 1, 1), (0, 0, 0), (0, 0, 1))}


def unit(*v):
    v = np.asarray(v, dtype=np.float64)
    return v / np.linalg.norm(v)


# test.perspectivecamera.cpp:100-141 (SampleRay): raster -> origin, direction
SAMPLE_RAY = [("identity", (0.5, 0.5), (0, 0, 0), unit(0, 0, -1)),
              ("identity", (1.0, 1.0), (0, 0, 0), unit(2, 1, -1)),
              ("lookat", (0.5, 0.5), (1, 1, 1), unit(-1, -1, -1))]
# test.perspectivecamera.cpp:143-176 (RayToRasterPosition): origin, direction -> raster
RAY_TO_RASTER = [("identity", (0, 0, 0), unit(0, 0, -1), (0.5, 0.5)),
                 ("identity", (0, 0, 0), unit(2, 1, -1), (1.0, 1.0)),
                 ("lookat", (1, 1, 1), unit(-1, -1, -1), (0.5, 0.5))]

# test.generalizedbsdf.cpp:129-215: sn = gn = (0, 1, 0), wi = normalize(1, 1, 1)
BSDF_FRAME = (0, 1, 0, 0, 1, 0)
BSDF_WI = unit(1, 1, 1)


def test_concentric_disk_known_answers():
    u = np.array([a for a, _ in DISK])
    np.testing.assert_allclose(oracle.eval_disk(u), np.array([b for _, b in DISK]), atol=1e-12)


def test_cosine_hemisphere_known_answers():
    u = np.array([a for a, _ in COSINE])
    np.testing.assert_allclose(oracle.eval_cosine(u), np.array([b for _, b in COSINE]), atol=1e-12)


@pytest.mark.parametrize("cam, raster, origin, direction", SAMPLE_RAY)
def test_camera_sample_ray_known_answers(cam, raster, origin, direction):
    rays, pdf = oracle.camera_rays([raster], *CAMERAS[cam], FOVY, *FILM)
    np.testing.assert_allclose(rays[0, :3], origin, atol=1e-12)
    np.testing.assert_allclose(rays[0, 3:], direction, atol=1e-12)
    assert pdf[0] > 0


@pytest.mark.parametrize("cam, origin, direction, raster", RAY_TO_RASTER)
def test_camera_ray_to_raster_known_answers(cam, origin, direction, raster):
    got, valid = oracle.camera_raster([np.r_[origin, direction]], *CAMERAS[cam], FOVY, *FILM)
    np.testing.assert_allclose(got[0], raster, atol=1e-12)
    if raster == (0.5, 0.5):
        assert valid[0]


def test_camera_round_trip():
    """RayToRasterPosition inverts SampleDirection over the film."""
    rng = np.random.default_rng(3)
    raster = rng.uniform(0.01, 0.99, size=(1000, 2))
    for cam in CAMERAS.values():
        rays, _ = oracle.camera_rays(raster, *cam, FOVY, *FILM)
        back, valid = oracle.camera_raster(rays, *cam, FOVY, *FILM)
        assert valid.all()
        np.testing.assert_allclose(back, raster, atol=1e-12)


@pytest.mark.parametrize("bsdf", ["diffuse", "diffuse_mirror"])
def test_bsdf_sample_is_consistent_with_evaluate(bsdf):
    """Consistency_PDF and Consistency_SampleAndEstimateDirection
    (test.generalizedbsdf.cpp:129-215): for a non-delta sample, the sampled
    pdf equals EvaluateDirectionPDF and the weight equals f / pdf."""
    rng = np.random.default_rng(5)
    n = 1 << 10
    frames = np.tile(BSDF_FRAME, (n, 1))
    wi = np.tile(BSDF_WI, (n, 1))
    u = rng.uniform(size=(n, 3))
    R = (1.0, 1.0, 1.0)
    s = oracle.bsdf_sample(bsdf, R, frames, wi, u)
    diffuse = ~s["specular"]
    assert diffuse.sum() > (n // 3 if bsdf == "diffuse_mirror" else n - 1)
    assert (s["pdf"] > 0).all()
    f, pdf = oracle.bsdf_eval(bsdf, R, frames[diffuse], wi[diffuse], s["wo"][diffuse])
    np.testing.assert_allclose(pdf, s["pdf"][diffuse], rtol=1e-12)
    np.testing.assert_allclose(f / pdf[:, None], s["weight"][diffuse], rtol=1e-12)


def test_mirror_sample_reflects():
    """PerfectMirrorBSDF (mirror.cpp:84-107): wo = reflection of wi about sn,
    weight R, pdf 1 / cos."""
    frames = np.array([BSDF_FRAME])
    s = oracle.bsdf_sample("mirror", (0.5, 0.25, 1.0), frames, [BSDF_WI], [(0.3, 0.6, 0.9)])
    np.testing.assert_allclose(s["wo"][0], unit(-1, 1, -1), atol=1e-12)
    np.testing.assert_allclose(s["weight"][0], (0.5, 0.25, 1.0), atol=1e-12)
    np.testing.assert_allclose(s["pdf"][0], S3, rtol=1e-12)
    assert s["specular"][0]


# test.hdrfilm.cpp, FilmNode_1: a 40 x 30 film (:32-38)
def film_40x30():
    from lightmetrica_b200.scene import HDRBitmapFilm
    f = HDRBitmapFilm(40, 30)
    f.allocate(40, 30)
    return f


def pixel_centres(f):
    return [((x + 0.5) / f.width, (y + 0.5) / f.height) for y in range(f.height) for x in range(f.width)]


def test_film_allocate():
    """Allocate (test.hdrfilm.cpp:264-275)."""
    f = film_40x30()
    assert (f.width, f.height) == (40, 30) and f.internal_data().size == 40 * 30 * 3


def test_film_accumulate_contribution_known_answers():
    """AccumulateContribution (test.hdrfilm.cpp:127-150): ten times (1,1,1) at
    raster (0,0) and (2,2,2) at (1,1) -> first pixel 10, last pixel 20."""
    f = film_40x30()
    for _ in range(10):
        assert f.accumulate_contribution((0, 0), (1, 1, 1))
        assert f.accumulate_contribution((1, 1), (2, 2, 2))
    d = f.internal_data().reshape(-1)
    np.testing.assert_array_equal(d[:3], 10)
    np.testing.assert_array_equal(d[-3:], 20)
    assert d[3:-3].sum() == 0


def test_film_accumulate_film_known_answers():
    """AccumulateContribution_2 (test.hdrfilm.cpp:152-178): a film of ones,
    recorded at the pixel centres, added ten times -> 10 everywhere."""
    ones = film_40x30()
    for r in pixel_centres(ones):
        assert ones.record_contribution(r, (1, 1, 1))
    f = film_40x30()
    for _ in range(10):
        assert f.accumulate_film(ones)
    np.testing.assert_array_equal(f.internal_data(), 10)
    g = film_40x30()
    g.allocate(20, 30)
    assert not f.accumulate_film(g)             # size mismatch is ignored


def test_film_rescale_and_clone_known_answers():
    """Rescale (test.hdrfilm.cpp:297-317) and Clone (:240-262)."""
    f = film_40x30()
    for r in pixel_centres(f):
        f.record_contribution(r, (1, 1, 1))
    c = f.clone()
    f.rescale(2)
    np.testing.assert_array_equal(f.internal_data(), 2)
    np.testing.assert_array_equal(c.internal_data(), 1)


def test_film_ignores_positions_outside_the_raster():
    f = film_40x30()
    for r in ((-0.01, 0.5), (0.5, 1.01), (1.0001, 1.0)):
        assert not f.accumulate_contribution(r, (1, 1, 1))
    assert f.internal_data().sum() == 0
