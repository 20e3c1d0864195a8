"""The allocation-free render entry point, lmgpu_render_device_noalloc.

It exists for callers that cannot allocate device memory while they render
(a host application's render callback under a memory manager that forbids
allocations, code running during CUDA stream capture, a process at its
memory budget). It renders into the caller's film with its wave workspace in
a static 32 MiB device array instead of memory from cudaMalloc. This file is
collected last so that a failure here cannot stop the other GPU tests; it
also passes on its own in a fresh process.
"""
import ctypes

import numpy as np
import pytest

from lightmetrica_b200 import create_renderer, create_scene, native, scenes

pytestmark = pytest.mark.gpu

SPP = 64   # 64 x 64 x 64 = 262,144 samples: two waves of the static workspace


def _scene_and_params(seed=5):
    prims = scenes.cornell_box(64, 64, variant="mixed")
    scene = create_scene("bvh")
    scene.load(prims)
    scene.configure({})
    scene.build()
    r = create_renderer("pt.mis")
    r.configure({"rr_depth": 3, "max_path_vertices": 9, "sampler": {"rng_seed": seed}})
    p = r.params(64 * 64 * SPP, film_fp64=True)
    return scene, p


def test_noalloc_render_matches_render_device_twice(cuda):
    import torch
    scene, p = _scene_and_params()
    stream = torch.cuda.current_stream().cuda_stream
    want = torch.zeros(64 * 64 * 3, dtype=torch.float64, device=cuda)
    st = native.RenderStats()
    native.check(native.lib().lmgpu_render_device(scene.handle, ctypes.byref(p), ctypes.c_void_p(want.data_ptr()),
                                                  ctypes.c_void_p(stream), ctypes.byref(st)))
    torch.cuda.synchronize()
    want = want.cpu().numpy()
    assert want.max() > 0
    for _ in range(2):     # the static workspace keeps the previous call's contents
        got = torch.zeros(64 * 64 * 3, dtype=torch.float64, device=cuda)
        native.check(native.lib().lmgpu_render_device_noalloc(scene.handle, ctypes.byref(p),
                                                              ctypes.c_void_p(got.data_ptr()), ctypes.c_void_p(stream)))
        torch.cuda.synchronize()
        # Same samples and paths; only the order of the FP64 film additions differs.
        np.testing.assert_allclose(got.cpu().numpy(), want, rtol=1e-9, atol=1e-12)
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
