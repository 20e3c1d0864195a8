"""Renderer / RenderProcessScheduler side of the component mirror
(reference renderer.h:39-133, sched.h:52-127, pathtrace.cpp:122-154,
sched.mt.cpp:41-266).

The reference's schedulers call ProcessSingleSample once per sample; on the
GPU the scheduler hands the whole `num_samples` budget to one C-ABI call and
writes the film with the reference's rescale semantics
(Rescale(W * H / num_samples), sched.mt.cpp:250-256).
"""
from __future__ import annotations

import ctypes
from typing import Optional

import numpy as np

from . import native as N

_TECHNIQUES = {"pt": N.RENDER_PT, "pt.direct": N.RENDER_PT_DIRECT, "pt.mis": N.RENDER_PT_MIS,
               "plugin.gpupt": N.RENDER_PT}


class Renderer:
    """Reference Renderer component ("pt", "pt.direct", "pt.mis")."""

    def __init__(self, impl: str = "pt"):
        if impl not in _TECHNIQUES:
            raise ValueError(f"unknown renderer '{impl}'")
        self.impl = impl
        self.technique = _TECHNIQUES[impl]
        self.rr_depth = 1
        self.max_path_vertices = -1
        self.seed = 1
        self.sampling = N.SAMPLING_STRATIFIED

    def type(self) -> str:
        return self.impl

    def configure(self, node: Optional[dict] = None, assets=None, scene=None, sched=None) -> bool:
        """Reads `rr_depth` (default 1), `max_path_vertices` (default -1) and
        `sampler` {`rng_seed`, `sampling`} like pathtrace.cpp:122-154."""
        node = node or {}
        self.rr_depth = int(node.get("rr_depth", 1))
        self.max_path_vertices = int(node.get("max_path_vertices", -1))
        sampler = node.get("sampler", {}) or {}
        self.seed = int(sampler.get("rng_seed", 1))
        mode = sampler.get("sampling", "stratified")
        if mode not in ("stratified", "uniform"):
            raise ValueError("sampler.sampling must be 'stratified' or 'uniform'")
        self.sampling = N.SAMPLING_STRATIFIED if mode == "stratified" else N.SAMPLING_UNIFORM
        return True

    def params(self, num_samples: int, sample_offset: int = 0, film_fp64: bool = False, wave_paths: int = 0):
        p = N.RenderParams()
        p.technique = self.technique
        p.rr_depth = self.rr_depth
        p.max_path_vertices = self.max_path_vertices
        p.sampling = self.sampling
        p.seed = self.seed
        p.num_samples = int(num_samples)
        p.sample_offset = int(sample_offset)
        p.film_fp64 = 1 if film_fp64 else 0
        p.wave_paths = int(wave_paths)
        return p


class RenderProcessScheduler:
    """Reference scheduler ("mt"): renders the whole sample budget. On the GPU
    this is one batched call; `num_threads`/`samples_per_block` are accepted
    for configuration compatibility and ignored."""

    def __init__(self, impl: str = "mt"):
        self.impl = impl
        self.num_samples = 1
        self.film_fp64 = False
        self.wave_paths = 0
        self.progress_image_interval = -1.0
        self.progress_images = []
        self.termination_mode = "samples"
        self.termination_time = 0.0
        self.last_stats = None

    def set_termination_mode(self, mode: str, time: float = 0.0) -> None:
        """RenderProcessScheduler::SetTerminationMode (sched.h:85): "samples"
        renders num_samples; "time" renders passes of num_samples until
        `time` seconds have passed (at least one pass; the reference checks
        the clock after every block of samples, this after every pass) and
        rescales by the samples processed (sched.mt.cpp:174-256)."""
        if mode not in ("samples", "time"):
            raise ValueError("termination mode must be 'samples' or 'time'")
        if mode == "time" and not time > 0:
            raise ValueError("time mode needs a positive time")
        self.termination_mode = mode
        self.termination_time = float(time)

    def configure(self, node: Optional[dict] = None, assets=None) -> bool:
        node = node or {}
        self.num_samples = int(node.get("num_samples", 1))
        self.film_fp64 = bool(node.get("film_fp64", False))
        self.wave_paths = int(node.get("wave_paths", 0))
        self.progress_image_interval = float(node.get("progress_image_interval", -1.0))
        if self.num_samples <= 0:
            raise ValueError("num_samples must be positive")
        return True

    def render(self, renderer: Renderer, scene) -> np.ndarray:
        """RenderProcessScheduler::Render: returns the rescaled film (H, W, 3)
        and stores it in the main camera's film."""
        cam = scene.main_camera()
        if cam is None or cam.film is None:
            raise RuntimeError("scene has no main camera / film")
        if self.progress_image_interval > 0.0 or self.termination_mode == "time":
            return self._render_chunked(renderer, scene, cam)
        film = np.zeros((cam.film.height, cam.film.width, 3), np.float32)
        p = renderer.params(self.num_samples, film_fp64=self.film_fp64, wave_paths=self.wave_paths)
        st = N.RenderStats()
        N.check(N.lib().lmgpu_render(scene.handle, ctypes.byref(p), film.ctypes.data, ctypes.byref(st)))
        self.last_stats = {"rays_traced": st.rays_traced, "shadow_rays": st.shadow_rays, "paths": st.paths,
                           "waves": st.waves, "max_bounces_run": st.max_bounces_run, "device_ms": st.device_ms}
        cam.film.data = film
        return film


    def _render_chunked(self, renderer, scene, cam) -> np.ndarray:
        """Chunks of samples into one device film, for progress images and
        the time termination mode. progress_image_interval > 0
        (sched.mt.cpp:197-228): whenever more than the interval (seconds) has
        passed since the last image, the film so far is rescaled by W*H /
        processed samples and saved as progress.<renderer>/%010d(.hdr|.exr).
        Time mode: passes of num_samples until the time is up."""
        import os
        import time
        import torch
        W, H = cam.film.width, cam.film.height
        dev_film = torch.zeros(W * H * 3, dtype=torch.float64 if self.film_fp64 else torch.float32, device="cuda")
        stream = torch.cuda.current_stream().cuda_stream
        timed = self.termination_mode == "time"
        chunk = self.num_samples if timed else max(W * H, self.num_samples // 64)
        if timed and self.progress_image_interval > 0.0:
            chunk = max(1, min(chunk, max(W * H, self.num_samples // 64)))
        done, count = 0, 0
        start = last = time.perf_counter()
        out_dir = "progress." + renderer.type()
        self.progress_images = []
        totals = {"rays_traced": 0, "shadow_rays": 0, "paths": 0, "waves": 0, "max_bounces_run": 0, "device_ms": 0.0}
        while True:
            if timed:
                if done > 0 and done % self.num_samples == 0 and time.perf_counter() - start >= self.termination_time:
                    break
                n = min(chunk, self.num_samples - done % self.num_samples)
            else:
                if done >= self.num_samples:
                    break
                n = min(chunk, self.num_samples - done)
            p = renderer.params(n, sample_offset=done, film_fp64=self.film_fp64, wave_paths=self.wave_paths)
            st = N.RenderStats()
            N.check(N.lib().lmgpu_render_device(scene.handle, ctypes.byref(p), ctypes.c_void_p(dev_film.data_ptr()),
                                                ctypes.c_void_p(stream), ctypes.byref(st)))
            for k in ("rays_traced", "shadow_rays", "paths", "waves", "device_ms"):
                totals[k] += getattr(st, k)
            totals["max_bounces_run"] = max(totals["max_bounces_run"], st.max_bounces_run)
            done += n
            now = time.perf_counter()
            more = timed or done < self.num_samples
            if self.progress_image_interval > 0.0 and now - last > self.progress_image_interval and more:
                count += 1
                img = (dev_film.double().cpu().numpy() * (W * H / done)).astype(np.float32).reshape(H, W, 3)
                from .film_io import save_film
                self.progress_images.append(save_film(img, os.path.join(out_dir, "%010d" % count),
                                                      cam.film.image_type))
                last = now
        film = (dev_film.double().cpu().numpy() * (W * H / done)).astype(np.float32).reshape(H, W, 3)
        totals["processed_samples"] = done
        self.last_stats = totals
        cam.film.data = film
        return film


def release_render_memory() -> None:
    """Frees the device memory renders keep between calls on the current
    device (the wave workspace: 216 bytes per path of the largest wave so far,
    28.7 GB after a 1080p 64-spp frame; lmgpu_render's film buffers). The
    next render allocates it again."""
    N.check(N.lib().lmgpu_render_release())


def create_renderer(impl: str = "pt") -> Renderer:
    return Renderer(impl)


def create_scheduler(impl: str = "mt"):
    """"mt" (one GPU: the whole budget in one call) or "mpi" (one process per
    GPU, sample shards and one film reduce; lightmetrica_b200.distributed)."""
    if impl == "mpi":
        from .distributed import MPIRenderProcessScheduler
        return MPIRenderProcessScheduler(impl)
    return RenderProcessScheduler(impl)
