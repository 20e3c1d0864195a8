"""Adjoint path replay (lmgpu_adjoint_forward / _backward) against central
finite differences (h = 1e-3, common random numbers) and against the FP64
CPU reference gradient of the oracle (same random numbers, same paths).
The torch.autograd.Function below exists only in this test harness.
"""
import os

import numpy as np
import pytest

import oracle
from lightmetrica_b200 import create_renderer, create_scene, scenes
from lightmetrica_b200.diff import DifferentiableRender, light_emission, triangle_albedo

pytestmark = pytest.mark.gpu

RR_DEPTH, MAX_PV = 3, 9


def setup(prims, technique="pt.mis", spp=64, seed=11, rr_depth=RR_DEPTH):
    scene = create_scene("bvh")
    scene.load(prims)
    scene.configure({})
    scene.build()
    r = create_renderer(technique)
    r.configure({"rr_depth": rr_depth, "max_path_vertices": MAX_PV, "sampler": {"rng_seed": seed}})
    W, H = prims.camera.film.width, prims.camera.film.height
    return scene, DifferentiableRender(scene, r, W * H * spp)


def make_autograd(dr):
    import torch

    class LmgpuRenderFunction(torch.autograd.Function):
        @staticmethod
        def forward(ctx, albedo, emission):
            ctx.save_for_backward(albedo, emission)
            return dr.forward(albedo, emission)

        @staticmethod
        def backward(ctx, grad_image):
            albedo, emission = ctx.saved_tensors
            return dr.backward(albedo, emission, grad_image)
    return LmgpuRenderFunction.apply


def test_forward_matches_renderer(cuda):
    import torch
    from lightmetrica_b200 import create_scheduler
    prims = scenes.cornell_box(64, 64, variant="mixed")
    scene, dr = setup(prims, spp=64)
    alb = torch.from_numpy(triangle_albedo(prims)).to(cuda)
    em = torch.from_numpy(light_emission(prims)).to(cuda)
    img = dr.forward(alb, em).cpu().numpy()
    s = create_scheduler("mt")
    s.configure({"num_samples": 64 * 64 * 64})
    film = s.render(dr.renderer, scene)
    # Same estimator, same random numbers: identical paths, only the
    # atomic summation order differs.
    np.testing.assert_allclose(img, film, rtol=1e-3, atol=1e-5)


@pytest.mark.parametrize("technique", ["pt.mis", "pt.direct", "pt"])
def test_gradient_matches_fp64_oracle(cuda, technique):
    import torch
    prims = scenes.cornell_box(32, 32)
    spp = 32
    scene, dr = setup(prims, technique, spp=spp)
    alb0 = triangle_albedo(prims)
    em0 = light_emission(prims)
    rng = np.random.default_rng(4)
    target_alb = np.clip(alb0 * rng.uniform(0.6, 1.4, alb0.shape), 0.05, 0.95).astype(np.float32)
    alb = torch.from_numpy(alb0).to(cuda)
    em = torch.from_numpy(em0).to(cuda)
    target = dr.forward(torch.from_numpy(target_alb).to(cuda), em)
    img = dr.forward(alb, em)
    dL = 2.0 * (img - target)
    da, de = dr.backward(alb, em, dL)
    ga, gl = oracle.oracle_grad(prims, dL.cpu().numpy(), technique, spp=spp, rr_depth=RR_DEPTH,
                                max_path_vertices=MAX_PV, seed=11, tri_albedo=alb0, threads=8)
    da = da.cpu().numpy()
    de = de.cpu().numpy()
    rel = np.linalg.norm(da - ga) / np.linalg.norm(ga)
    print(f"{technique}: |d_albedo - fp64| / |fp64| = {rel:.2e}")
    assert rel <= 1e-2
    np.testing.assert_allclose(de, gl, rtol=1e-2)


def test_gradient_matches_central_differences(cuda):
    """Central differences (h = 1e-3) of L = sum (I - T)^2 with common random
    numbers, for the red wall's albedo (per channel, all its triangles moved
    together; each wall's dominant channel) and for the light's emission.
    Russian roulette is off here so
    that the fixed-seed estimator is smooth in the parameters (with it on,
    the adjoint is the unbiased gradient of the expected image, which
    per-seed differences do not measure)."""
    import torch
    prims = scenes.cornell_box(48, 48)
    scene, dr = setup(prims, "pt.mis", spp=128, rr_depth=-1)
    alb0 = triangle_albedo(prims)
    em0 = light_emission(prims)
    alb = torch.from_numpy(alb0).to(cuda)
    em = torch.from_numpy(em0).to(cuda)
    # Target with the scene's own emission: pixels that see the light directly
    # then have I - T ~ 0, so the film's float-atomic summation noise at
    # those bright pixels (radiance ~17) is not amplified into the loss.
    target = dr.forward(torch.from_numpy((alb0 * 0.8).astype(np.float32)).to(cuda), em).double()

    def loss(a, e):
        return float(((dr.forward(a, e).double() - target) ** 2).sum())

    img = dr.forward(alb, em)
    da, de = dr.backward(alb, em, 2.0 * (img.double() - target).float())
    h = 1e-3
    # Each wall's dominant channel: a perturbation whose effect on the image
    # stands well above the float-atomic summation noise of the film.
    groups = {"red wall": (np.arange(6, 8), 0), "green wall": (np.arange(8, 10), 1),
              "floor/ceiling/back": (np.arange(0, 6), 2)}
    for name, (tris, c) in groups.items():
        d = torch.zeros_like(alb)
        d[tris, c] = 1.0
        fd = (loss(alb + h * d, em) - loss(alb - h * d, em)) / (2 * h)
        ad = float(da[tris, c].sum())
        print(f"{name} ch{c}: fd {fd:.6e} adjoint {ad:.6e}")
        assert abs(ad - fd) <= 1e-2 * abs(fd)
    for c in range(3):
        e = torch.zeros_like(em)
        e[0, c] = 1.0
        fd = (loss(alb, em + h * e) - loss(alb, em - h * e)) / (2 * h)
        ad = float(de[0, c])
        print(f"emission ch{c}: fd {fd:.6e} adjoint {ad:.6e}")
        assert abs(ad - fd) <= 1e-2 * abs(fd)


def test_autograd_function(cuda):
    import torch
    prims = scenes.cornell_box(32, 32)
    scene, dr = setup(prims, "pt.mis", spp=16)
    fn = make_autograd(dr)
    alb = torch.from_numpy(triangle_albedo(prims)).to(cuda).requires_grad_(True)
    em = torch.from_numpy(light_emission(prims)).to(cuda).requires_grad_(True)
    target = dr.forward(alb.detach() * 0.5, em.detach())
    loss = ((fn(alb, em) - target) ** 2).sum()
    loss.backward()
    img = dr.forward(alb.detach(), em.detach())
    da, de = dr.backward(alb.detach(), em.detach(), 2 * (img - target))
    torch.testing.assert_close(alb.grad, da, rtol=1e-4, atol=1e-6)
    torch.testing.assert_close(em.grad, de, rtol=1e-4, atol=1e-6)


def test_c4_scene_gradient_matches_fp64_oracle_and_fd(cuda):
    """The adjoint on the differentiable-rendering scene itself: the Cornell
    box refined to 36,864 triangles (each of its 36 triangles split into 4^5),
    per-triangle albedo U[0.1, 0.9] (seed 3) against a target of seed-4
    albedos, pt.mis, max depth 8; reduced to 64 x 64 pixels at 16 spp.
    (1) With Russian roulette from vertex 3: the whole albedo gradient and the
    emission gradient against the oracle's FP64 gradient on the same random
    numbers (relative 1e-2). (2) With Russian roulette off (the fixed-seed
    estimator is then a polynomial in the albedos): the adjoint against
    central differences (h = 1e-3) of the FP64 loss, for 20 individual
    triangles drawn at random among the 200 with the largest gradients, and
    for the light's emission."""
    import torch
    W = H = 64
    spp = 16
    prims = scenes.cornell_refined(5, W, H)
    T = scenes.num_triangles(prims)
    assert T == 36 * 4 ** 5
    alb0 = np.random.default_rng(3).uniform(0.1, 0.9, (T, 3)).astype(np.float32)
    alb_t = np.random.default_rng(4).uniform(0.1, 0.9, (T, 3)).astype(np.float32)
    em0 = light_emission(prims)
    alb, em = torch.from_numpy(alb0).to(cuda), torch.from_numpy(em0).to(cuda)
    threads = os.cpu_count() or 1

    scene, dr = setup(prims, "pt.mis", spp=spp)
    target = dr.forward(torch.from_numpy(alb_t).to(cuda), em)
    dL = 2.0 * (dr.forward(alb, em) - target)
    da, de = dr.backward(alb, em, dL)
    ga, gl = oracle.oracle_grad(prims, dL.cpu().numpy(), "pt.mis", spp=spp, rr_depth=RR_DEPTH,
                                max_path_vertices=MAX_PV, seed=11, tri_albedo=alb0, threads=threads)
    da = da.cpu().numpy()
    rel = np.linalg.norm(da - ga) / np.linalg.norm(ga)
    print(f"C4 scene: |d_albedo - fp64| / |fp64| = {rel:.2e}")
    assert rel <= 1e-2
    np.testing.assert_allclose(de.cpu().numpy(), gl, rtol=1e-2)

    scene, dr = setup(prims, "pt.mis", spp=spp, rr_depth=-1)
    kw = dict(technique="pt.mis", spp=spp, rr_depth=-1, max_path_vertices=MAX_PV, seed=11, threads=threads)
    target = oracle.oracle_render(prims, tri_albedo=alb_t, **kw)

    def loss(a, le=None):
        return float(((oracle.oracle_render(prims, tri_albedo=a, light_Le=le, **kw) - target) ** 2).sum())

    img = oracle.oracle_render(prims, tri_albedo=alb0, **kw)
    da, de = dr.backward(alb, em, torch.from_numpy((2.0 * (img - target)).astype(np.float32)).to(cuda))
    da, de = da.cpu().numpy(), de.cpu().numpy()
    flat = np.abs(da).reshape(-1)
    top = np.argsort(flat)[-200:]
    pick = np.random.default_rng(5).choice(top, 20, replace=False)
    h = 1e-3
    # The oracle takes float32 parameters: the step is the float32 one.
    for idx in pick:
        t, c = divmod(int(idx), 3)
        ap, am = alb0.copy(), alb0.copy()
        ap[t, c] = np.float32(alb0[t, c] + h)
        am[t, c] = np.float32(alb0[t, c] - h)
        fd = (loss(ap) - loss(am)) / (float(ap[t, c]) - float(am[t, c]))
        print(f"triangle {t} ch{c}: fd {fd:.6e} adjoint {da[t, c]:.6e}")
        assert abs(da[t, c] - fd) <= 1e-2 * abs(fd)
    for c in range(3):
        lp, lm = em0.copy(), em0.copy()
        lp[0, c] = np.float32(em0[0, c] + h)
        lm[0, c] = np.float32(em0[0, c] - h)
        fd = (loss(alb0, lp) - loss(alb0, lm)) / (float(lp[0, c]) - float(lm[0, c]))
        print(f"emission ch{c}: fd {fd:.6e} adjoint {de[0, c]:.6e}")
        assert abs(de[0, c] - fd) <= 1e-2 * abs(fd)


def closed_box(width, height, light_absorbs=True):
    """The Cornell box closed by a front wall and seen from inside it: a
    perfect-mirror back wall and tall box, a diffuse-mirror short box, highly
    reflective diffuse walls (0.95; red and green side walls). With the
    light's black BSDF its only exit is the light, which takes ~1% of the
    bounces: without Russian roulette paths run for about a hundred vertices.
    With `light_absorbs` False the light reflects too and no path ends."""
    from lightmetrica_b200.scene import (AreaLight, DiffuseBSDF, DiffuseMirrorBSDF, HDRBitmapFilm,
                                         PerfectMirrorBSDF, PerspectiveCamera, Primitive, Primitives)
    from lightmetrica_b200.scenes import _box, _mesh, _quad
    white, red, green = DiffuseBSDF((0.95, 0.95, 0.95)), DiffuseBSDF((0.95, 0.6, 0.5)), DiffuseBSDF((0.5, 0.95, 0.6))
    prims = Primitives()
    prims.add(Primitive(mesh=_mesh([_quad((0, 0, 0), (1, 0, 0), (1, 0, 1), (0, 0, 1), (0, 1, 0)),
                                    _quad((0, 1, 0), (1, 1, 0), (1, 1, 1), (0, 1, 1), (0, -1, 0)),
                                    _quad((0, 0, 1), (1, 0, 1), (1, 1, 1), (0, 1, 1), (0, 0, -1))]), bsdf=white))
    prims.add(Primitive(mesh=_mesh([_quad((0, 0, 0), (1, 0, 0), (1, 1, 0), (0, 1, 0), (0, 0, 1))]),
                        bsdf=PerfectMirrorBSDF((0.98, 0.98, 0.98))))
    prims.add(Primitive(mesh=_mesh([_quad((0, 0, 0), (0, 1, 0), (0, 1, 1), (0, 0, 1), (1, 0, 0))]), bsdf=red))
    prims.add(Primitive(mesh=_mesh([_quad((1, 0, 0), (1, 1, 0), (1, 1, 1), (1, 0, 1), (-1, 0, 0))]), bsdf=green))
    prims.add(Primitive(mesh=_box((0.33, 0.0, 0.62), (0.30, 0.30, 0.30), -17.0),
                        bsdf=DiffuseMirrorBSDF((0.9, 0.85, 0.8))))
    prims.add(Primitive(mesh=_box((0.68, 0.0, 0.35), (0.30, 0.60, 0.30), 17.0),
                        bsdf=PerfectMirrorBSDF((0.98, 0.98, 0.98))))
    y = 1.0 - 1e-3
    prims.add(Primitive(mesh=_mesh([_quad((0.37, y, 0.40), (0.63, y, 0.40), (0.63, y, 0.60), (0.37, y, 0.60),
                                          (0, -1, 0))]),
                        bsdf=DiffuseBSDF((0.0, 0.0, 0.0) if light_absorbs else (0.9, 0.9, 0.9)),
                        light=AreaLight((17.0, 12.0, 4.0))))
    prims.camera = PerspectiveCamera(fovy=70.0, eye=(0.5, 0.5, 0.97), center=(0.5, 0.45, 0.0), up=(0, 1, 0),
                                     film=HDRBitmapFilm(width, height))
    return prims


def test_long_paths_gradient_matches_fp64_oracle(cuda):
    """Unbounded depth (max_path_vertices = -1) and no Russian roulette in
    the closed mirror-and-diffuse box: paths run for hundreds of vertices.
    The adjoint keeps records for the first 32 vertices and replays deeper
    tails from a checkpoint; its albedo and emission gradients must equal
    the oracle's FP64 gradient on the same random numbers, and its forward
    image the wavefront renderer's image of the same samples."""
    import torch
    from lightmetrica_b200 import create_scheduler
    W = H = 24
    spp = 8
    prims = closed_box(W, H)
    scene = create_scene("bvh")
    scene.load(prims)
    scene.configure({})
    scene.build()
    r = create_renderer("pt.mis")
    r.configure({"rr_depth": -1, "max_path_vertices": -1, "sampler": {"rng_seed": 21}})
    sched = create_scheduler("mt")
    sched.configure({"num_samples": W * H * spp, "film_fp64": True})
    film = sched.render(r, scene)
    deepest = sched.last_stats["max_bounces_run"]
    print(f"deepest bounce: {deepest}")
    assert deepest > 100
    dr = DifferentiableRender(scene, r, W * H * spp)
    alb0 = triangle_albedo(prims)
    em0 = light_emission(prims)
    alb, em = torch.from_numpy(alb0).to(cuda), torch.from_numpy(em0).to(cuda)
    img = dr.forward(alb, em)
    np.testing.assert_allclose(img.cpu().numpy(), film, rtol=1e-3, atol=1e-5)
    target = dr.forward(torch.from_numpy((alb0 * 0.9).astype(np.float32)).to(cuda), em)
    dL = 2.0 * (img - target)
    da, de = dr.backward(alb, em, dL)
    ga, gl = oracle.oracle_grad(prims, dL.cpu().numpy(), "pt.mis", spp=spp, rr_depth=-1, max_path_vertices=-1,
                                seed=21, tri_albedo=alb0, threads=os.cpu_count() or 1)
    da = da.cpu().numpy()
    rel = np.linalg.norm(da - ga) / np.linalg.norm(ga)
    print(f"long paths: |d_albedo - fp64| / |fp64| = {rel:.2e}")
    assert rel <= 1e-2
    np.testing.assert_allclose(de.cpu().numpy(), gl, rtol=1e-2)
    # Vertices beyond the recorded 32 carry a real share of the gradient:
    # truncating the paths there changes it.
    r33 = create_renderer("pt.mis")
    r33.configure({"rr_depth": -1, "max_path_vertices": 34, "sampler": {"rng_seed": 21}})
    da33, _ = DifferentiableRender(scene, r33, W * H * spp).backward(alb, em, dL)
    assert np.linalg.norm(da33.cpu().numpy() - da) > 0.05 * np.linalg.norm(da)
    scene.close()


def test_replay_bound_overflow_is_reported(cuda):
    """A closed box whose light reflects too: without Russian roulette no
    path ends (nor would the reference's loop). The replay stops at its
    bound of 4096 surface vertices, raises the status word, and both passes
    report LMGPU_ERR_QUEUE_OVERFLOW; with a depth bound the same scene then
    renders."""
    import torch
    from lightmetrica_b200 import native
    prims = closed_box(8, 8, light_absorbs=False)
    scene = create_scene("bvh")
    scene.load(prims)
    scene.configure({})
    scene.build()
    r = create_renderer("pt.mis")
    r.configure({"rr_depth": -1, "max_path_vertices": -1, "sampler": {"rng_seed": 3}})
    dr = DifferentiableRender(scene, r, 8 * 8)
    alb = torch.from_numpy(triangle_albedo(prims)).to(cuda)
    em = torch.from_numpy(light_emission(prims)).to(cuda)
    with pytest.raises(native.LmgpuError) as e:
        dr.forward(alb, em)
    assert e.value.code == native.ERR_QUEUE_OVERFLOW
    with pytest.raises(native.LmgpuError) as e:
        dr.backward(alb, em, torch.ones((8, 8, 3), device=cuda))
    assert e.value.code == native.ERR_QUEUE_OVERFLOW
    r.configure({"rr_depth": -1, "max_path_vertices": 64, "sampler": {"rng_seed": 3}})
    img = DifferentiableRender(scene, r, 8 * 8 * 4).forward(alb, em)
    assert torch.isfinite(img).all() and float(img.max()) > 0
    scene.close()
