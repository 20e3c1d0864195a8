"""Multi-GPU rendering: sample sharding with one film reduce, the B200
counterpart of the reference's MPI scheduler (sched.mpi.cpp:107-311).

The reference's rank 0 hands out tasks of `samples_per_mpi_task` samples to
the other ranks, which render them, and MPI_Reduce sums the films onto rank 0
before it rescales by W*H / processed samples (sched.mpi.cpp:296-307). The
GPUs of one node are equal, so here every rank (rank 0 included) renders one
contiguous range of the sample sequence, of nearly equal size, on its own GPU
with its own copy of the scene, and one NCCL reduce (sum) of the device films
onto rank 0 replaces MPI_Reduce. A sample's random numbers depend only on its
index, so the sharded render is the one-GPU render of the same samples: only
the order of the film additions differs.

One process per GPU, launched by torchrun; the process group is the
caller's (torch.distributed, backend "nccl" on GPUs). `render_shard` can be
replaced, e.g. by a CPU renderer in tests over a "gloo" group.
"""
from __future__ import annotations

import ctypes
from typing import Callable, Optional, Tuple

import numpy as np

from . import native as N


def shard(num_samples: int, rank: int, world: int) -> Tuple[int, int]:
    """(offset, count) of rank's contiguous share of [0, num_samples):
    counts differ by at most one."""
    if world <= 0 or not 0 <= rank < world:
        raise ValueError("bad rank / world size")
    if num_samples < 0:
        raise ValueError("negative sample count")
    begin = num_samples * rank // world
    end = num_samples * (rank + 1) // world
    return begin, end - begin


def rank_and_world(group=None) -> Tuple[int, int]:
    import torch.distributed as dist
    if dist.is_available() and dist.is_initialized():
        return dist.get_rank(group), dist.get_world_size(group)
    return 0, 1


def max_over_ranks(value: float, group=None, device=None) -> float:
    """The largest `value` of all ranks (job time = the slowest rank's)."""
    import torch
    import torch.distributed as dist
    rank, world = rank_and_world(group)
    if world == 1:
        return float(value)
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX, group=group)
    return float(t[0])


def aggregate_rate(units_per_rank: int, steps: int, job_ms: float, world: int) -> float:
    """Whole-job throughput (units per second) of `world` ranks that each
    processed units_per_rank per step for `steps` steps in job_ms."""
    if job_ms <= 0:
        raise ValueError("job time must be positive")
    return world * units_per_rank * steps / (job_ms / 1e3)


class MPIRenderProcessScheduler:
    """The "mpi" scheduler: configuration keys of sched.mpi.cpp:84-105
    (`num_samples`, `samples_per_mpi_task`, `samples_per_block`; the latter
    two are accepted for compatibility: the shards are static)."""

    def __init__(self, impl: str = "mpi"):
        self.impl = impl
        self.num_samples = 1
        self.samples_per_task = 1000000
        self.film_fp64 = True
        self.termination_mode = "samples"
        self.termination_time = 0.0
        self.last_shard = None
        self.processed_samples = 0

    def set_termination_mode(self, mode: str, time: float = 0.0) -> None:
        """SetTerminationMode (sched.mpi.cpp:64): "samples" renders
        num_samples over the ranks; "time" renders rounds of num_samples (each
        rank its shard of each round) until rank 0 has seen `time` seconds
        pass (at least one round; the reference hands out tasks until then,
        sched.mpi.cpp:146-186), and rescales by the samples processed."""
        if mode not in ("samples", "time"):
            raise ValueError("termination mode must be 'samples' or 'time'")
        if mode == "time" and not time > 0:
            raise ValueError("time mode needs a positive time")
        self.termination_mode = mode
        self.termination_time = float(time)

    def configure(self, node: Optional[dict] = None, assets=None) -> bool:
        node = node or {}
        self.num_samples = int(node.get("num_samples", 1))
        self.samples_per_task = int(node.get("samples_per_mpi_task", 1000000))
        self.film_fp64 = bool(node.get("film_fp64", True))
        if self.num_samples <= 0:
            raise ValueError("num_samples must be positive")
        if int(node.get("samples_per_block", 100)) <= 0:
            raise ValueError("Invalid value for 'samples_per_block'")     # sched.mpi.cpp:95-98
        return True

    def _gpu_shard(self, renderer, scene, offset: int, count: int):
        """This rank's un-rescaled device film of samples [offset, offset + count)."""
        import torch
        cam = scene.main_camera()
        W, H = cam.film.width, cam.film.height
        film = torch.zeros(W * H * 3, dtype=torch.float64 if self.film_fp64 else torch.float32, device="cuda")
        if count > 0:
            p = renderer.params(count, sample_offset=offset, film_fp64=self.film_fp64)
            st = N.RenderStats()
            N.check(N.lib().lmgpu_render_device(scene.handle, ctypes.byref(p), ctypes.c_void_p(film.data_ptr()),
                                                ctypes.c_void_p(torch.cuda.current_stream().cuda_stream),
                                                ctypes.byref(st)))
        return film

    def render(self, renderer, scene, group=None,
               render_shard: Optional[Callable[[int, int], "object"]] = None):
        """Renders this rank's shard and reduces the films onto rank 0.
        Returns the rescaled film (H, W, 3) on rank 0 and None elsewhere.
        `render_shard(offset, count)` returns the shard's un-rescaled film as
        a torch tensor of W*H*3 values (default: this rank's GPU)."""
        import time
        import torch
        import torch.distributed as dist
        rank, world = rank_and_world(group)
        offset, count = shard(self.num_samples, rank, world)
        self.last_shard = (offset, count)
        render_shard = render_shard or (lambda o, c: self._gpu_shard(renderer, scene, o, c))
        film = render_shard(offset, count)
        rounds = 1
        if self.termination_mode == "time":
            # Rank 0 decides after each round and every rank follows, so all
            # ranks take the same collective steps.
            start = time.perf_counter()
            while True:
                go = torch.tensor([1 if time.perf_counter() - start < self.termination_time else 0],
                                  dtype=torch.int32, device=film.device)
                if world > 1:
                    dist.broadcast(go, src=0, group=group)
                if not int(go.item()):
                    break
                film = film + render_shard(rounds * self.num_samples + offset, count)
                rounds += 1
        self.processed_samples = rounds * self.num_samples
        if world > 1:
            dist.reduce(film, dst=0, op=dist.ReduceOp.SUM, group=group)
        if rank != 0:
            return None
        cam = scene.main_camera()
        W, H = cam.film.width, cam.film.height
        out = (film.double().cpu().numpy() * (W * H / self.processed_samples)).astype(np.float32).reshape(H, W, 3)
        cam.film.data = out
        return out
