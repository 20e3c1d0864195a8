"""The path tracer's building blocks evaluated on the device for given inputs
(lmgpu_eval_sampling, lmgpu_camera_*, lmgpu_bsdf_*): the same device
functions the renderers inline, one query per row, float32.

    uniform_concentric_disk_sample(u)          Math::UniformConcentricDiskSample (math.stats.inl:25-56)
    cosine_sample_hemisphere(u)                Math::CosineSampleHemisphere (math.stats.inl:64-69)
    camera_sample_rays(scene, raster)          PerspectiveCamera::SamplePosition + SampleDirection
                                               (perspectivecamera.cpp:170-240)
    camera_ray_to_raster(scene, rays)          PerspectiveCamera::RayToRasterPosition (:304-323)
    film_pixels(scene, raster)                 HDRBitmapFilm::AccumulateContribution's pixel (hdrfilm.cpp:151-171)
    bsdf_sample(bsdf, R, frames, wi, u)        BSDF::SampleAndEstimateDirection, EL
    bsdf_evaluate(bsdf, R, frames, wi, wo)     BSDF::EvaluateDirection / EvaluateDirectionPDF (NonDelta)

`frames` rows are (gn, sn); the tangents come from sn as
SurfaceGeometry::ComputeTangentSpace makes them. Each call copies its inputs
to the device and synchronises (checks and tools, not a hot path).
"""
from __future__ import annotations

import ctypes

import numpy as np

from . import native as N

BSDFS = {"diffuse": N.BSDF_DIFFUSE, "mirror": N.BSDF_MIRROR, "diffuse_mirror": N.BSDF_DIFFUSE_MIRROR}


def _f32(a, cols):
    return np.ascontiguousarray(np.asarray(a, dtype=np.float32).reshape(-1, cols))


def _p(a):
    return ctypes.c_void_p(a.ctypes.data)


def _sampling(fn, u, cols):
    u = _f32(u, 2)
    out = np.empty((u.shape[0], cols), dtype=np.float32)
    N.check(N.lib().lmgpu_eval_sampling(fn, _p(u), u.shape[0], _p(out)))
    return out


def uniform_concentric_disk_sample(u):
    """u (n x 2) in [0,1]^2 -> points on the unit disk (n x 2)."""
    return _sampling(N.EVAL_CONCENTRIC_DISK, u, 2)


def cosine_sample_hemisphere(u):
    """u (n x 2) -> cosine-distributed directions about +z (n x 3)."""
    return _sampling(N.EVAL_COSINE_HEMISPHERE, u, 3)


def camera_sample_rays(scene, raster):
    """The scene's camera: raster positions (n x 2, y = 0 at the bottom) ->
    (rays (n x 6: origin, direction), pdf (n))."""
    r = _f32(raster, 2)
    rays = np.empty((r.shape[0], 6), dtype=np.float32)
    pdf = np.empty(r.shape[0], dtype=np.float32)
    N.check(N.lib().lmgpu_camera_sample_rays(scene.handle, _p(r), r.shape[0], _p(rays), _p(pdf)))
    return rays, pdf


def camera_ray_to_raster(scene, rays):
    """Rays (n x 6) -> (raster positions (n x 2), valid (n): False where the
    direction leaves the film)."""
    r = _f32(rays, 6)
    raster = np.empty((r.shape[0], 2), dtype=np.float32)
    valid = np.empty(r.shape[0], dtype=np.int32)
    N.check(N.lib().lmgpu_camera_raster_positions(scene.handle, _p(r), r.shape[0], _p(raster), _p(valid)))
    return raster, valid.astype(bool)


def film_pixels(scene, raster):
    """Raster positions (n x 2) -> pixel indices y * W + x of the scene
    camera's film (-1 outside [0,1]^2), as the renderers splat them."""
    r = _f32(raster, 2)
    out = np.empty(r.shape[0], dtype=np.int32)
    N.check(N.lib().lmgpu_film_pixels(scene.handle, _p(r), r.shape[0], _p(out)))
    return out


def light_sample(scene, u):
    """(u0, u1) (n x 2) -> dict of position, normal (n x 3), pdf (n: area pdf
    times the light selection probability) and light (n: area light index,
    the number of area lights for the environment), as the renderers' next
    event estimation samples the scene's lights."""
    uu = _f32(u, 2)
    pts = np.empty((uu.shape[0], 7), dtype=np.float32)
    light = np.empty(uu.shape[0], dtype=np.int32)
    N.check(N.lib().lmgpu_light_sample(scene.handle, _p(uu), uu.shape[0], _p(pts), _p(light)))
    return {"position": pts[:, 0:3], "normal": pts[:, 3:6], "pdf": pts[:, 6], "light": light}


def bsdf_sample(bsdf, reflectance, frames, wi, u):
    """SampleAndEstimateDirection (EL) -> dict of wo, weight (n x 3), pdf (n,
    projected solid angle), specular (n)."""
    R = _f32(reflectance, 3)
    f, w, uu = _f32(frames, 6), _f32(wi, 3), _f32(u, 3)
    n = f.shape[0]
    if w.shape[0] != n or uu.shape[0] != n:
        raise ValueError("frames, wi and u need one row per query")
    out = {"wo": np.empty((n, 3), np.float32), "weight": np.empty((n, 3), np.float32),
           "pdf": np.empty(n, np.float32), "specular": np.empty(n, np.int32)}
    N.check(N.lib().lmgpu_bsdf_sample(BSDFS[bsdf], _p(R), _p(f), _p(w), _p(uu), n, _p(out["wo"]), _p(out["weight"]),
                                      _p(out["pdf"]), _p(out["specular"])))
    out["specular"] = out["specular"].astype(bool)
    return out


def bsdf_evaluate(bsdf, reflectance, frames, wi, wo):
    """EvaluateDirection and EvaluateDirectionPDF of the non-delta part ->
    (f (n x 3), pdf (n))."""
    R = _f32(reflectance, 3)
    f, a, b = _f32(frames, 6), _f32(wi, 3), _f32(wo, 3)
    n = f.shape[0]
    if a.shape[0] != n or b.shape[0] != n:
        raise ValueError("frames, wi and wo need one row per query")
    fs = np.empty((n, 3), np.float32)
    pdf = np.empty(n, np.float32)
    N.check(N.lib().lmgpu_bsdf_evaluate(BSDFS[bsdf], _p(R), _p(f), _p(a), _p(b), n, _p(fs), _p(pdf)))
    return fs, pdf
