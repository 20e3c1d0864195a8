"""The allocation-free render entry point, lmgpu_render_device_noalloc.

It exists for callers that cannot allocate device memory while they render
(a host application's render callback under a memory manager that forbids
allocations, a process at its memory budget). It renders into the caller's
film with its wave workspace in a static 32 MiB device array instead of
memory from cudaMalloc. This file is collected last so that a failure here
cannot stop the other GPU tests; it also passes on its own in a fresh
process.
"""
import ctypes

import numpy as np
import pytest

from lightmetrica_b200 import create_renderer, create_scene, native, scenes

pytestmark = pytest.mark.gpu

SPP = 64   # 64 x 64 x 64 = 262,144 samples: two waves of the static workspace


def _scene_and_params(technique="pt.mis", film_fp64=True, max_path_vertices=9, seed=5):
    prims = scenes.cornell_box(64, 64, variant="mixed")
    scene = create_scene("bvh")
    scene.load(prims)
    scene.configure({})
    scene.build()
    r = create_renderer(technique)
    r.configure({"rr_depth": 3, "max_path_vertices": max_path_vertices, "sampler": {"rng_seed": seed}})
    p = r.params(64 * 64 * SPP, film_fp64=film_fp64)
    return scene, p


def _render_both(cuda, scene, p, film_fp64):
    """The allocating entry point once, then the allocation-free one twice in
    a row (the static workspace keeps the previous call's contents)."""
    import torch
    dtype = torch.float64 if film_fp64 else torch.float32
    stream = torch.cuda.current_stream().cuda_stream
    want = torch.zeros(64 * 64 * 3, dtype=dtype, device=cuda)
    st = native.RenderStats()
    native.check(native.lib().lmgpu_render_device(scene.handle, ctypes.byref(p), ctypes.c_void_p(want.data_ptr()),
                                                  ctypes.c_void_p(stream), ctypes.byref(st)))
    torch.cuda.synchronize()
    got = []
    for _ in range(2):
        g = torch.zeros(64 * 64 * 3, dtype=dtype, device=cuda)
        native.check(native.lib().lmgpu_render_device_noalloc(scene.handle, ctypes.byref(p),
                                                              ctypes.c_void_p(g.data_ptr()), ctypes.c_void_p(stream)))
        torch.cuda.synchronize()
        got.append(g.cpu().numpy().astype(np.float64))
    return want.cpu().numpy().astype(np.float64), got


@pytest.mark.parametrize("film_fp64", [True, False], ids=["fp64_film", "fp32_film"])
@pytest.mark.parametrize("technique", ["pt", "pt.direct", "pt.mis"])
def test_noalloc_render_matches_render_device_twice(cuda, technique, film_fp64):
    scene, p = _scene_and_params(technique, film_fp64)
    want, got = _render_both(cuda, scene, p, film_fp64)
    assert want.max() > 0
    # Same samples and paths; only the order of the film's atomic additions
    # differs (FP64 film: 1e-9 relative; FP32 film: 1e-4 relative).
    rtol, atol = (1e-9, 1e-12) if film_fp64 else (1e-4, 1e-6)
    for g in got:
        np.testing.assert_allclose(g, want, rtol=rtol, atol=atol)
    scene.close()


@pytest.mark.parametrize("max_path_vertices", [0, 1])
def test_noalloc_paths_without_vertices_beyond_the_camera(cuda, max_path_vertices):
    # max_path_vertices <= 1 leaves no vertex beyond the camera: both entry
    # points return an untouched film.
    scene, p = _scene_and_params("pt.mis", True, max_path_vertices=max_path_vertices)
    want, got = _render_both(cuda, scene, p, True)
    assert not want.any()
    for g in got:
        assert not g.any()
    scene.close()


def test_noalloc_rejects_waves_beyond_the_static_workspace(cuda):
    import torch
    scene, p = _scene_and_params()
    p.wave_paths = 1 << 20
    film = torch.zeros(64 * 64 * 3, dtype=torch.float64, device=cuda)
    rc = native.lib().lmgpu_render_device_noalloc(scene.handle, ctypes.byref(p), ctypes.c_void_p(film.data_ptr()),
                                                  ctypes.c_void_p(torch.cuda.current_stream().cuda_stream))
    assert rc == native.ERR_INVALID
    assert b"no-alloc workspace" in native.lib().lmgpu_last_error()
    scene.close()
