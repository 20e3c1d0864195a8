"""Multi-scene batch rendering through lmgpu_batch_* (no counterpart in the
reference, whose RenderProcessScheduler renders one scene at a time,
sched.mt.cpp:93-266).

    batch = SceneBatch([scene_a, scene_b, ...])       # built Scene objects
    batch.autotune(renderers, num_samples)            # optional: layout, wave size, shading grid
    films = batch.render(renderers, num_samples)      # one (H, W, 3) film per scene

Each scene keeps its own camera, film, renderer parameters (technique shared
by the batch) and sample count, and renders exactly the samples it would
render alone through RenderProcessScheduler.render: same random numbers,
same paths. All scenes' paths run in fixed waves ("waves"), in fixed waves
over two pools of path state whose tails overlap the next wave's first
bounces ("overlap"), or in one pool of path slots that take new paths as
old ones finish ("stream"); the kernel sequence is replayed from a captured
CUDA graph.
"""
from __future__ import annotations

import ctypes
from typing import Sequence

import numpy as np

from . import native as N
from .render import Renderer

# "bvh": binary float nodes, "qbvh": 4-wide, "bvh_q16": binary nodes with
# 16-bit quantised child boxes, "bvh_qshadow": float nodes for bounce rays
# and quantised ones for shadow rays (the last two: batch renders only).
LAYOUTS = {"bvh": N.LAYOUT_BVH2, "qbvh": N.LAYOUT_BVH4, "bvh_q16": N.LAYOUT_BVH2Q,
           "bvh_qshadow": N.LAYOUT_BVH2_QSHADOW}
MODES = {"waves": N.BATCH_WAVES, "stream": N.BATCH_STREAM, "overlap": N.BATCH_OVERLAP}


class SceneBatch:
    def __init__(self, scenes: Sequence):
        if not scenes:
            raise ValueError("a batch needs at least one scene")
        self.scenes = list(scenes)
        arr = (ctypes.c_void_p * len(self.scenes))(*[s.handle.value for s in self.scenes])
        self._keep = arr
        self.handle = ctypes.c_void_p()
        N.check(N.lib().lmgpu_batch_create(arr, len(self.scenes), ctypes.byref(self.handle)))
        self.last_stats = None

    # ------------------------------------------------------------ config --
    @property
    def config(self) -> dict:
        c = N.BatchConfig()
        N.check(N.lib().lmgpu_batch_get_config(self.handle, ctypes.byref(c)))
        return {"layout": {v: k for k, v in LAYOUTS.items()}[c.layout], "wave_paths": c.wave_paths,
                "shade_blocks_per_sm": c.shade_blocks_per_sm, "use_graph": bool(c.use_graph),
                "mode": {v: k for k, v in MODES.items()}[c.mode], "overlap_bounce": c.overlap_bounce}

    def configure(self, layout: str | None = None, wave_paths: int | None = None,
                  shade_blocks_per_sm: int | None = None, use_graph: bool | None = None,
                  mode: str | None = None, overlap_bounce: int | None = None) -> None:
        c = N.BatchConfig()
        N.check(N.lib().lmgpu_batch_get_config(self.handle, ctypes.byref(c)))
        if layout is not None:
            if layout not in LAYOUTS:
                raise ValueError("layout must be one of " + ", ".join(LAYOUTS))
            c.layout = LAYOUTS[layout]
        if wave_paths is not None:
            c.wave_paths = int(wave_paths)
        if shade_blocks_per_sm is not None:
            c.shade_blocks_per_sm = int(shade_blocks_per_sm)
        if use_graph is not None:
            c.use_graph = 1 if use_graph else 0
        if mode is not None:
            if mode not in MODES:
                raise ValueError("mode must be 'waves', 'stream' or 'overlap'")
            c.mode = MODES[mode]
        if overlap_bounce is not None:
            c.overlap_bounce = int(overlap_bounce)
        N.check(N.lib().lmgpu_batch_set_config(self.handle, ctypes.byref(c)))

    # ------------------------------------------------------------ render --
    def _params(self, renderers, num_samples, film_fp64, sample_offsets=None):
        n = len(self.scenes)
        if isinstance(renderers, Renderer):
            renderers = [renderers] * n
        if np.isscalar(num_samples):
            num_samples = [int(num_samples)] * n
        if sample_offsets is None or np.isscalar(sample_offsets):
            sample_offsets = [int(sample_offsets or 0)] * n
        if len(renderers) != n or len(num_samples) != n or len(sample_offsets) != n:
            raise ValueError("one renderer, one sample count and one sample offset per scene")
        arr = (N.RenderParams * n)()
        for i, (r, k, o) in enumerate(zip(renderers, num_samples, sample_offsets)):
            arr[i] = r.params(int(k), sample_offset=int(o), film_fp64=film_fp64)
        return arr

    @staticmethod
    def _stats(st):
        return {"rays_traced": st.rays_traced, "shadow_rays": st.shadow_rays, "paths": st.paths,
                "waves": st.waves, "max_bounces_run": st.max_bounces_run, "device_ms": st.device_ms}

    def render_device(self, renderers, num_samples, films, stream=None, stats: bool = True, sample_offsets=None):
        """Accumulates each scene's un-rescaled samples into `films[i]`
        (CUDA tensors of W*H*3 float32, or float64 with film_fp64);
        `sample_offsets` gives each scene's first sample index (default 0)."""
        import torch
        fp64 = films[0].dtype == torch.float64
        params = self._params(renderers, num_samples, fp64, sample_offsets)
        ptrs = (ctypes.c_void_p * len(films))(*[f.data_ptr() for f in films])
        s = stream if stream is not None else torch.cuda.current_stream(films[0].device).cuda_stream
        st = N.RenderStats() if stats else None
        N.check(N.lib().lmgpu_batch_render_device(self.handle, params, ptrs, ctypes.c_void_p(s),
                                                  ctypes.byref(st) if stats else None))
        if stats:
            self.last_stats = self._stats(st)
        return films

    def render(self, renderers, num_samples, film_fp64: bool = False, sample_offsets=None, out=None):
        """Renders every scene through lmgpu_batch_render; returns the
        rescaled films (H, W, 3) float32 (the reference's Rescale(W * H /
        num_samples)). `out` may give the host arrays to fill."""
        n = len(self.scenes)
        params = self._params(renderers, num_samples, film_fp64, sample_offsets)
        if out is None:
            out = []
            for s in self.scenes:
                cam = s.main_camera()
                out.append(np.empty((cam.film.height, cam.film.width, 3), np.float32))
        for s, f in zip(self.scenes, out):
            cam = s.main_camera()
            if f.dtype != np.float32 or f.size != cam.film.width * cam.film.height * 3 or not f.flags.c_contiguous:
                raise ValueError("each output film must be a C-contiguous float32 array of W*H*3 values")
        ptrs = (ctypes.c_void_p * n)(*[f.ctypes.data for f in out])
        st = N.RenderStats()
        N.check(N.lib().lmgpu_batch_render(self.handle, params, ptrs, ctypes.byref(st)))
        self.last_stats = self._stats(st)
        return out

    def profile(self, renderers, num_samples, films, count_tests: bool = False, stream=None,
                sample_offsets=None) -> dict:
        """One measurement render (lmgpu_batch_profile): direct launches in
        fixed waves with CUDA events around every traversal launch; with
        `count_tests`, the slab and TriAccel tests of every ray (counting
        kernels: their times are not the render's)."""
        import torch
        fp64 = films[0].dtype == torch.float64
        params = self._params(renderers, num_samples, fp64, sample_offsets)
        ptrs = (ctypes.c_void_p * len(films))(*[f.data_ptr() for f in films])
        s = stream if stream is not None else torch.cuda.current_stream(films[0].device).cuda_stream
        p = N.TraceProfile()
        N.check(N.lib().lmgpu_batch_profile(self.handle, params, ptrs, ctypes.c_void_p(s), 1 if count_tests else 0,
                                            ctypes.byref(p)))
        out = {"render_ms": p.render_ms}
        for k, name in ((0, "closest"), (1, "shadow")):
            out[name] = {"rays": p.rays[k], "launches": p.launches[k], "trace_ms": p.trace_ms[k]}
            if count_tests:
                out[name]["node_tests"] = int(p.node_tests[k])
                out[name]["tri_tests"] = int(p.tri_tests[k])
        return out

    def autotune(self, renderers, num_samples, sample_fraction: float = 0.125, stream=None) -> dict:
        """Chooses mode, layout, wave size, shading grid and overlap bounce by timing scaled-down
        renders of this batch (each candidate on at least four of its waves, or
        the whole render; compared by time per sample); the choice becomes the
        batch's configuration. trial_ms is the winner's time at sample_fraction."""
        import torch
        params = self._params(renderers, num_samples, False)
        s = stream if stream is not None else torch.cuda.current_stream().cuda_stream
        c = N.BatchConfig()
        ms = ctypes.c_double()
        N.check(N.lib().lmgpu_batch_autotune(self.handle, params, float(sample_fraction), ctypes.c_void_p(s),
                                             ctypes.byref(c), ctypes.byref(ms)))
        out = self.config
        out["trial_ms"] = ms.value
        return out

    def close(self) -> None:
        if self.handle is not None and self.handle.value:
            N.lib().lmgpu_batch_destroy(self.handle)
        self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
