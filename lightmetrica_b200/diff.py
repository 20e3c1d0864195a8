"""Differentiable rendering through the C ABI's forward / adjoint pair
(lmgpu_adjoint_forward / lmgpu_adjoint_backward).

Parameters are per-triangle RGB albedo of diffuse BSDFs (reference TriAccel
numbering: primitive-major, face order) and per-area-light RGB emission.
torch CUDA tensors carry device memory; the computation is the native path
replay in liblmgpu.so.
"""
from __future__ import annotations

import ctypes

import numpy as np

from . import native as N
from .render import Renderer


def triangle_albedo(prims) -> np.ndarray:
    """(T, 3) float32: each triangle's BSDF reflectance (0 where none)."""
    out = []
    for p in prims.primitives:
        n = p.mesh.faces.shape[0] if p.mesh is not None else 0
        R = np.zeros(3, np.float32) if p.bsdf is None else np.broadcast_to(np.asarray(p.bsdf.reflectance, np.float32), (3,))
        out.append(np.tile(R, (n, 1)))
    return np.concatenate(out).astype(np.float32) if out else np.zeros((0, 3), np.float32)


def light_emission(prims) -> np.ndarray:
    """(L, 3) float32 emission of the area lights in first-use order."""
    seen, out = set(), []
    for p in prims.primitives:
        if p.light is not None and id(p.light) not in seen:
            seen.add(id(p.light))
            out.append(np.broadcast_to(np.asarray(p.light.luminance, np.float32), (3,)))
    return np.array(out, np.float32).reshape(-1, 3)


class DifferentiableRender:
    """Forward image and adjoint gradients of one scene/camera/sample budget."""

    def __init__(self, scene, renderer: Renderer, num_samples: int):
        self.scene = scene
        self.renderer = renderer
        self.num_samples = int(num_samples)
        cam = scene.main_camera()
        self.W, self.H = cam.film.width, cam.film.height
        self.last_forward_ms = None
        self.last_backward_ms = None

    def _params(self):
        return self.renderer.params(self.num_samples)

    def forward(self, albedo, emission, stream=None):
        """albedo (T, 3), emission (L, 3): float32 CUDA tensors. Returns the
        rescaled image (H, W, 3) as a float32 CUDA tensor."""
        import torch
        albedo = albedo.contiguous()
        emission = emission.contiguous()
        img = torch.zeros((self.H, self.W, 3), dtype=torch.float32, device=albedo.device)
        dp = N.DiffParams(albedo.data_ptr(), emission.data_ptr() if emission.numel() else None)
        p = self._params()
        st = N.RenderStats()
        s = stream if stream is not None else torch.cuda.current_stream(albedo.device).cuda_stream
        N.check(N.lib().lmgpu_adjoint_forward(self.scene.handle, ctypes.byref(p), ctypes.byref(dp), img.data_ptr(),
                                              ctypes.c_void_p(s), ctypes.byref(st)))
        self.scene.status(s)
        self.last_forward_ms = st.device_ms
        return img

    def backward(self, albedo, emission, dL_dimage, stream=None):
        """Returns (d_albedo (T, 3), d_emission (L, 3)) CUDA tensors."""
        import torch
        albedo = albedo.contiguous()
        emission = emission.contiguous()
        g = dL_dimage.contiguous().to(torch.float32)
        da = torch.zeros_like(albedo)
        de = torch.zeros_like(emission) if emission.numel() else torch.zeros(3, device=albedo.device)
        dp = N.DiffParams(albedo.data_ptr(), emission.data_ptr() if emission.numel() else None)
        p = self._params()
        st = N.RenderStats()
        s = stream if stream is not None else torch.cuda.current_stream(albedo.device).cuda_stream
        N.check(N.lib().lmgpu_adjoint_backward(self.scene.handle, ctypes.byref(p), ctypes.byref(dp), g.data_ptr(),
                                               da.data_ptr(), de.data_ptr(), ctypes.c_void_p(s), ctypes.byref(st)))
        self.scene.status(s)
        self.last_backward_ms = st.device_ms
        return da, de[:emission.shape[0]] if emission.numel() else de[:0]
