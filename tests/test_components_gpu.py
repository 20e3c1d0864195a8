"""The device's sampling, camera and BSDF functions (the ones the renderers
inline), through lmgpu_eval_sampling / lmgpu_camera_* / lmgpu_bsdf_*:
against the reference's component tests' known answers (restated in
test_components.py) and against the oracle's FP64 restatement on random
inputs. Tolerances are float32 rounding of a few operations."""
import numpy as np
import pytest

import oracle
from lightmetrica_b200 import components as C
from lightmetrica_b200 import native
from lightmetrica_b200.scene import HDRBitmapFilm, PerspectiveCamera, Scene, soup_primitives
from test_components import (BSDF_FRAME, BSDF_WI, CAMERAS, COSINE, DISK, FILM, FOVY, RAY_TO_RASTER, SAMPLE_RAY,
                             unit)

pytestmark = pytest.mark.gpu


def camera_scene(eye, center, up, fovy=FOVY, film=FILM):
    """A scene with one far-away triangle and the given camera."""
    pos = np.array([[100, 100, 100], [101, 100, 100], [100, 101, 100]], dtype=np.float32)
    prims = soup_primitives(pos, np.array([[0, 1, 2]], dtype=np.uint32))
    prims.camera = PerspectiveCamera(fovy=fovy, eye=eye, center=center, up=up, film=HDRBitmapFilm(*film))
    s = Scene("bvh")
    s.load(prims)
    s.configure({})
    s.build()
    return s


def test_sampling_known_answers(cuda):
    np.testing.assert_allclose(C.uniform_concentric_disk_sample([a for a, _ in DISK]), [b for _, b in DISK], atol=1e-6)
    np.testing.assert_allclose(C.cosine_sample_hemisphere([a for a, _ in COSINE]), [b for _, b in COSINE], atol=1e-6)


def test_sampling_matches_oracle(cuda):
    u = np.random.default_rng(11).uniform(size=(100000, 2)).astype(np.float32)
    np.testing.assert_allclose(C.uniform_concentric_disk_sample(u), oracle.eval_disk(u), atol=2e-6)
    got, want = C.cosine_sample_hemisphere(u), oracle.eval_cosine(u)
    np.testing.assert_allclose(got[:, :2], want[:, :2], atol=2e-6)
    # z = sqrt(1 - x^2 - y^2) magnifies float rounding near the rim: compare z^2.
    np.testing.assert_allclose(got[:, 2] ** 2, want[:, 2] ** 2, atol=5e-6)


@pytest.mark.parametrize("cam, raster, origin, direction", SAMPLE_RAY)
def test_camera_sample_ray_known_answers(cuda, cam, raster, origin, direction):
    s = camera_scene(*CAMERAS[cam])
    rays, pdf = C.camera_sample_rays(s, [raster])
    np.testing.assert_allclose(rays[0, :3], origin, atol=1e-6)
    np.testing.assert_allclose(rays[0, 3:], direction, atol=1e-6)
    assert pdf[0] > 0
    s.close()


@pytest.mark.parametrize("cam, origin, direction, raster", RAY_TO_RASTER)
def test_camera_ray_to_raster_known_answers(cuda, cam, origin, direction, raster):
    s = camera_scene(*CAMERAS[cam])
    got, valid = C.camera_ray_to_raster(s, [np.r_[origin, direction]])
    np.testing.assert_allclose(got[0], raster, atol=1e-6)
    if raster == (0.5, 0.5):
        assert valid[0]
    s.close()


def test_camera_matches_oracle(cuda):
    rng = np.random.default_rng(12)
    raster = rng.uniform(size=(20000, 2)).astype(np.float32)
    cams = [((0.3, -1.2, 2.0), (0.1, 0.2, -0.3), (0.2, 1.0, 0.1), 40.0, (256, 192)), (*CAMERAS["lookat"], FOVY, FILM)]
    for eye, center, up, fovy, film in cams:
        s = camera_scene(eye, center, up, fovy, film)
        rays, pdf = C.camera_sample_rays(s, raster)
        want, want_pdf = oracle.camera_rays(raster, eye, center, up, fovy, *film)
        np.testing.assert_allclose(rays, want, atol=2e-5)
        # EvaluateImportance snaps cos within EpsLarge of 1 to 1; EpsLarge is
        # 1e-3 in the float build (the device) and 1e-5 in the double build
        # (the oracle), so the two differ, as the reference's builds do, for
        # 1e-5 < 1 - cos < 1e-3.
        f = np.asarray(center, float) - np.asarray(eye, float)
        cos = want[:, 3:] @ (f / np.linalg.norm(f))
        outside = 1 - cos > 1.01e-3
        assert outside.mean() > 0.9
        np.testing.assert_allclose(pdf[outside], want_pdf[outside], rtol=2e-4)
        back, valid = C.camera_ray_to_raster(s, rays)
        interior = ((raster > 1e-3) & (raster < 1 - 1e-3)).all(axis=1)
        assert valid[interior].all()
        np.testing.assert_allclose(back[interior], raster[interior], atol=2e-4)
        s.close()


@pytest.mark.parametrize("bsdf", ["diffuse", "diffuse_mirror"])
def test_bsdf_consistency_and_oracle(cuda, bsdf):
    """test.generalizedbsdf.cpp:129-215 on the device (sampled pdf = evaluated
    pdf, weight = f / pdf for non-delta samples), and the device's samples
    against the oracle's for the same numbers."""
    rng = np.random.default_rng(13)
    n = 1 << 12
    frames = np.tile(BSDF_FRAME, (n, 1)).astype(np.float32)
    wi = np.tile(BSDF_WI, (n, 1)).astype(np.float32)
    u = rng.uniform(size=(n, 3)).astype(np.float32)
    R = (0.8, 0.5, 0.25)
    s = C.bsdf_sample(bsdf, R, frames, wi, u)
    d = ~s["specular"]
    f, pdf = C.bsdf_evaluate(bsdf, R, frames[d], wi[d], s["wo"][d])
    np.testing.assert_allclose(pdf, s["pdf"][d], rtol=1e-6)
    np.testing.assert_allclose(f / pdf[:, None], s["weight"][d], rtol=1e-5)
    o = oracle.bsdf_sample(bsdf, R, frames, wi, u)
    np.testing.assert_array_equal(s["specular"], o["specular"])
    np.testing.assert_allclose(s["wo"], o["wo"], atol=2e-5)
    np.testing.assert_allclose(s["weight"], o["weight"], atol=1e-6)
    np.testing.assert_allclose(s["pdf"], o["pdf"], rtol=1e-5)


def test_bsdf_random_frames_match_oracle(cuda):
    """Tilted shading normals (the shading-normal correction factor of
    bsdf.h:57-83 zeroes some samples) and all three BSDFs."""
    rng = np.random.default_rng(14)
    n = 1 << 12
    gn = rng.normal(size=(n, 3))
    gn /= np.linalg.norm(gn, axis=1, keepdims=True)
    sn = gn + 0.3 * rng.normal(size=(n, 3))
    sn /= np.linalg.norm(sn, axis=1, keepdims=True)
    wi = rng.normal(size=(n, 3))
    wi /= np.linalg.norm(wi, axis=1, keepdims=True)
    frames = np.hstack([gn, sn]).astype(np.float32)
    u = rng.uniform(size=(n, 3)).astype(np.float32)
    wo = rng.normal(size=(n, 3))
    wo = (wo / np.linalg.norm(wo, axis=1, keepdims=True)).astype(np.float32)
    wi = wi.astype(np.float32)
    for bsdf in ("diffuse", "mirror", "diffuse_mirror"):
        s = C.bsdf_sample(bsdf, (1, 1, 1), frames, wi, u)
        o = oracle.bsdf_sample(bsdf, (1, 1, 1), frames, wi, u)
        # Away from the decision boundaries (cos ~ 0 on either side), the
        # device and the oracle take the same branches.
        lwi = np.einsum("ij,ij->i", wi, sn)
        ok = (np.abs(lwi) > 1e-3) & (np.abs(np.einsum("ij,ij->i", o["wo"], gn)) > 1e-3)
        assert ok.mean() > 0.99
        np.testing.assert_allclose(s["weight"][ok], o["weight"][ok], atol=1e-6)
        np.testing.assert_allclose(s["pdf"][ok], o["pdf"][ok], rtol=1e-4)
        f, pdf = C.bsdf_evaluate(bsdf, (1, 1, 1), frames, wi, wo)
        of, opdf = oracle.bsdf_eval(bsdf, (1, 1, 1), frames, wi, wo)
        ok2 = (np.abs(lwi) > 1e-3) & (np.abs(np.einsum("ij,ij->i", wo, sn)) > 1e-3) & \
              (np.abs(np.einsum("ij,ij->i", wo, gn)) > 1e-3) & (np.abs(np.einsum("ij,ij->i", wi, gn)) > 1e-3)
        np.testing.assert_allclose(f[ok2], of[ok2], atol=1e-6)
        np.testing.assert_allclose(pdf[ok2], opdf[ok2], rtol=1e-6)


def test_component_errors(cuda):
    L = native.lib()
    u = np.zeros((4, 2), np.float32)
    assert L.lmgpu_eval_sampling(7, u.ctypes.data, 4, u.ctypes.data) == native.ERR_INVALID
    assert L.lmgpu_eval_sampling(0, u.ctypes.data, -1, u.ctypes.data) == native.ERR_INVALID
    assert L.lmgpu_eval_sampling(0, None, 0, None) == native.OK
    assert L.lmgpu_camera_sample_rays(None, u.ctypes.data, 4, None, None) == native.ERR_INVALID
    with pytest.raises(KeyError):
        C.bsdf_sample("dielectric", (1, 1, 1), np.zeros((1, 6)), np.zeros((1, 3)), np.zeros((1, 3)))
    with pytest.raises(native.LmgpuError):
        native.check(L.lmgpu_bsdf_sample(9, np.ones(3, np.float32).ctypes.data, None, None, None, 1, None, None, None,
                                         None))


def test_film_pixels_match_host_film(cuda):
    """The renderers' raster -> pixel mapping against the host film's
    restatement of HDRBitmapFilm::AccumulateContribution: edges, pixel
    boundaries, outside positions and random positions."""
    from lightmetrica_b200.scene import HDRBitmapFilm
    W, H = 37, 23
    s = camera_scene(*CAMERAS["identity"], film=(W, H))
    film = HDRBitmapFilm(W, H)
    rng = np.random.default_rng(15)
    raster = np.concatenate([
        [(0, 0), (1, 1), (1, 0), (0, 1), (0.5, 0.5), (-0.001, 0.5), (0.5, 1.001), (1.0000001, 0.5)],
        [(x / W, y / H) for x in range(W + 1) for y in (0, H // 2, H)],
        rng.uniform(-0.05, 1.05, size=(20000, 2))]).astype(np.float32)
    got = C.film_pixels(s, raster)
    want = np.array([film.pixel_of(r) for r in raster], dtype=np.int32)
    np.testing.assert_array_equal(got, want)
    assert got[0] == 0 and got[1] == W * H - 1
    s.close()


def light_scene(level):
    """Two area lights and the constant environment: an icosphere light of
    `level` (level 1: 80 triangles, at most a few CDF entries per guide bin,
    which the device scans; level 5: 20,480, about 80 per bin, which it
    halves) and a two-triangle quad light of another area and luminance."""
    from lightmetrica_b200 import scenes
    from lightmetrica_b200.scene import (AreaLight, ConstantEnvironmentLight, DiffuseBSDF, Primitive, Primitives,
                                         TriangleMesh)
    prims = Primitives()
    V, F = scenes.icosphere(level)
    prims.add(Primitive(mesh=TriangleMesh((V * 0.5 + [0.0, 3.0, 0.0]).astype(np.float32), F, V.copy()),
                        bsdf=DiffuseBSDF((0.0, 0.0, 0.0)), light=AreaLight((40.0, 36.0, 30.0))))
    qv = np.array([[-2, 1, -2], [1, 1, -2], [1, 1.5, 1], [-2, 1.5, 1]], dtype=np.float32)
    qn = np.tile(np.array([[0.0, -0.986, 0.164]], dtype=np.float32), (4, 1))
    prims.add(Primitive(mesh=TriangleMesh(qv, np.array([[0, 1, 2], [0, 2, 3]], dtype=np.uint32), qn),
                        bsdf=DiffuseBSDF((0.0, 0.0, 0.0)), light=AreaLight((5.0, 6.0, 7.0))))
    prims.environment_light = ConstantEnvironmentLight((0.5, 0.5, 0.5))
    prims.camera = PerspectiveCamera(fovy=45.0, eye=(0.0, 2.0, 6.0), center=(0.0, 1.0, 0.0), up=(0, 1, 0),
                                     film=HDRBitmapFilm(32, 32))
    s = Scene("bvh")
    s.load(prims)
    s.configure({})
    s.build()
    return prims, s


@pytest.mark.parametrize("level", [1, 5], ids=["scanned_guide_ranges", "halved_guide_ranges"])
def test_light_sample_matches_oracle(cuda, level):
    """Scene::SampleLightSelection + SamplePosition: light choice, position,
    normal and pdf against the FP64 restatement. The device's triangle CDF
    is float: where u1 lies within its rounding of a boundary (a fraction
    ~1e-3 or less of the samples here) it may pick the neighbouring
    triangle; all other samples agree to float rounding."""
    prims, scene = light_scene(level)
    u = np.random.default_rng(5 + level).uniform(size=(200000, 2)).astype(np.float32)
    got = C.light_sample(scene, u)
    want, wl = oracle.light_sample(prims, u)
    np.testing.assert_array_equal(got["light"], wl)
    assert set(np.unique(wl)) == {0, 1, 2}                       # both area lights and the environment
    np.testing.assert_allclose(got["pdf"], want[:, 6], rtol=2e-6)
    d = np.linalg.norm(got["position"] - want[:, :3], axis=1)
    scale = np.linalg.norm(want[:, :3], axis=1) + 1.0
    close = d < 2e-5 * scale
    assert close.mean() > 0.998, close.mean()
    # The normal is the cross product of two float edge vectors: on the
    # level-5 sphere the edges (~0.016) are differences of coordinates near 3,
    # so each carries ~3e-8 * 3 / 0.016 ~ 1e-5 relative rounding.
    nz = np.linalg.norm(want[:, 3:6], axis=1) > 0
    np.testing.assert_allclose(got["normal"][close & nz], want[close & nz, 3:6], atol=1e-4)
    scene.close()
