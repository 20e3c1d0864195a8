"""Scene documents and film output end to end on the GPU: a scene read back
from its XML document renders like the scene it was written from; a
primitive with a transform intersects exactly like its mesh transformed on
the host in the reference's float order; progress images are written while
the budget renders in chunks and the final film is unchanged."""
import ctypes

import numpy as np
import pytest

from lightmetrica_b200 import create_renderer, create_scene, create_scheduler, native, scenes
from lightmetrica_b200.film_io import read_hdr
from lightmetrica_b200.scene import DiffuseBSDF, Primitive, Primitives, TriangleMesh
from lightmetrica_b200.sceneio import load_scene, mat_mul, rotate, save_scene, scale, translate
from lightmetrica_b200.workloads import random_rays

pytestmark = pytest.mark.gpu


def build(prims):
    s = create_scene("bvh")
    s.load(prims)
    s.configure({})
    s.build()
    return s


def fp64_render(scene, renderer, n):
    import torch
    cam = scene.main_camera()
    f = torch.zeros(cam.film.width * cam.film.height * 3, dtype=torch.float64, device="cuda")
    p = renderer.params(n, film_fp64=True)
    st = native.RenderStats()
    native.check(native.lib().lmgpu_render_device(scene.handle, ctypes.byref(p), ctypes.c_void_p(f.data_ptr()),
                                                  ctypes.c_void_p(torch.cuda.current_stream().cuda_stream),
                                                  ctypes.byref(st)))
    torch.cuda.synchronize()
    return f.cpu().numpy()


def test_xml_scene_renders_like_its_source(cuda):
    P = scenes.cornell_box(48, 48, variant="mixed")
    doc = load_scene(save_scene(P, renderer={"type": "pt.mis", "rr_depth": 3, "max_path_vertices": 9,
                                             "sampler": {"rng_seed": 3}}))
    r = create_renderer(doc.renderer_type)
    r.configure(doc.renderer_config)
    a, b = build(P), build(doc.primitives)
    want = fp64_render(a, r, 48 * 48 * 32)
    assert want.max() > 0
    np.testing.assert_allclose(fp64_render(b, r, 48 * 48 * 32), want, rtol=1e-9, atol=1e-12)


def test_transformed_primitive_intersects_like_host_transformed_mesh(cuda):
    rng = np.random.default_rng(3)
    n = 2000
    c = rng.uniform(-1, 1, (n, 3))
    e1, e2 = rng.normal(0, 0.05, (n, 3)), rng.normal(0, 0.05, (n, 3))
    pos = np.stack([c, c + e1, c + e2], 1).astype(np.float32).reshape(-1, 3)
    faces = np.arange(3 * n, dtype=np.uint32).reshape(-1, 3)
    M = mat_mul(mat_mul(translate((0.3, -0.2, 0.5)), rotate(37.0, (1, 2, 3))), scale((1.5, 0.5, 2.0)))
    # The builder's order for Mat4f * Vec4f: (m0 x + m1 y) + (m2 z + m3), float.
    f32 = np.float32
    world = np.empty_like(pos)
    for r in range(3):
        world[:, r] = ((M[r, 0] * pos[:, 0]).astype(f32) + (M[r, 1] * pos[:, 1]).astype(f32)).astype(f32) + \
                      ((M[r, 2] * pos[:, 2]).astype(f32) + (M[r, 3] * f32(1.0)).astype(f32)).astype(f32)
    A = Primitives(primitives=[Primitive(mesh=TriangleMesh(pos, faces), transform=M, bsdf=DiffuseBSDF())])
    B = Primitives(primitives=[Primitive(mesh=TriangleMesh(world, faces), bsdf=DiffuseBSDF())])
    rays = random_rays(100000, seed=5, extent=2.5)
    ha = build(A).intersect_host(rays)
    hb = build(B).intersect_host(rays)
    assert (ha["tri_id"] >= 0).sum() > 1000
    np.testing.assert_array_equal(ha["tri_id"], hb["tri_id"])
    np.testing.assert_array_equal(ha["t"], hb["t"])


def test_progress_images(cuda, tmp_path, monkeypatch):
    monkeypatch.chdir(tmp_path)
    P = scenes.cornell_box(32, 32)
    scene = build(P)
    r = create_renderer("pt.mis")
    r.configure({"rr_depth": 3, "max_path_vertices": 9, "sampler": {"rng_seed": 2}})
    n = 32 * 32 * 128
    s = create_scheduler("mt")
    s.configure({"num_samples": n, "progress_image_interval": 1e-9})
    film = s.render(r, scene)
    assert len(s.progress_images) >= 10
    assert all(p.startswith("progress.pt.mis/") and p.endswith(".hdr") for p in s.progress_images)
    last = read_hdr(s.progress_images[-1])
    assert last.shape == (32, 32, 3) and np.isfinite(last).all() and last.max() > 0
    plain = create_scheduler("mt")
    plain.configure({"num_samples": n})
    np.testing.assert_allclose(film, plain.render(r, scene), rtol=1e-4, atol=1e-6)
