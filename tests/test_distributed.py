"""Multi-process host logic on CPU (world size 2, "gloo"): sample shards,
the film reduce of the "mpi" scheduler, and the max-over-ranks job time the
benchmark uses. Each rank renders its shard with the oracle (the GPU render
of a shard is the same function of the same samples); rank 0's reduced film
must equal the one-process render of all samples.
"""
import os
import socket

import numpy as np
import pytest

from lightmetrica_b200 import create_scheduler, scenes
from lightmetrica_b200.distributed import aggregate_rate, max_over_ranks, shard

SPP, RR, MAX_PV, SEED = 8, 3, 9, 5


def test_shards_cover_the_samples_contiguously():
    for n in (0, 1, 7, 1000, 1 << 33):
        for world in (1, 2, 3, 8):
            parts = [shard(n, r, world) for r in range(world)]
            assert parts[0][0] == 0
            for (o, c), (o2, _) in zip(parts, parts[1:]):
                assert o + c == o2
            assert sum(c for _, c in parts) == n
            assert max(c for _, c in parts) - min(c for _, c in parts) <= 1
    with pytest.raises(ValueError):
        shard(10, 2, 2)
    with pytest.raises(ValueError):
        shard(-1, 0, 1)


def test_rate_and_single_process_max():
    assert aggregate_rate(1 << 24, 10, 1000.0, 4) == pytest.approx(4 * (1 << 24) * 10)
    with pytest.raises(ValueError):
        aggregate_rate(1, 1, 0.0, 1)
    assert max_over_ranks(3.5) == 3.5


def test_mpi_scheduler_configuration():
    s = create_scheduler("mpi")
    s.configure({"num_samples": 100, "samples_per_mpi_task": 10})
    assert s.num_samples == 100
    with pytest.raises(ValueError):
        s.configure({"num_samples": 0})
    with pytest.raises(ValueError):
        s.configure({"num_samples": 10, "samples_per_block": 0})


class _CameraOnly:
    """Stand-in scene for the CPU test: the scheduler only needs the camera."""

    def __init__(self, prims):
        self.prims = prims

    def main_camera(self):
        return self.prims.camera


def _worker(rank, world, port, out_dir, time_limit=0.0):
    import torch
    import torch.distributed as dist
    import oracle
    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=world)
    try:
        prims = scenes.cornell_box(16, 16)
        n = 16 * 16 * SPP
        sched = create_scheduler("mpi")
        sched.configure({"num_samples": n})
        if time_limit > 0:
            sched.set_termination_mode("time", time_limit)

        def render_shard(offset, count):
            return torch.from_numpy(oracle.oracle_render_range(prims, offset, offset + count, "pt.mis", RR, MAX_PV,
                                                               SEED))
        film = sched.render(None, _CameraOnly(prims), render_shard=render_shard)
        job = max_over_ranks(float(rank + 1))
        np.save(os.path.join(out_dir, f"rank{rank}.npy"),
                {"film": film, "shard": sched.last_shard, "job": job, "processed": sched.processed_samples},
                allow_pickle=True)
    finally:
        dist.destroy_process_group()


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def test_two_ranks_reduce_to_the_one_process_film(tmp_path):
    import torch.multiprocessing as mp
    import oracle
    world = 2
    mp.start_processes(_worker, args=(world, _free_port(), str(tmp_path)), nprocs=world, join=True,
                       start_method="spawn")
    r0 = np.load(tmp_path / "rank0.npy", allow_pickle=True).item()
    r1 = np.load(tmp_path / "rank1.npy", allow_pickle=True).item()
    n = 16 * 16 * SPP
    assert r0["shard"] == (0, n // 2) and r1["shard"] == (n // 2, n - n // 2)
    assert r1["film"] is None
    assert r0["job"] == 2.0 and r1["job"] == 2.0
    want = oracle.oracle_render(scenes.cornell_box(16, 16), "pt.mis", spp=SPP, rr_depth=RR, max_path_vertices=MAX_PV,
                                seed=SEED, threads=2)
    assert want.max() > 0
    np.testing.assert_allclose(r0["film"], want, rtol=1e-5, atol=1e-7)


def test_two_ranks_time_mode(tmp_path):
    """Time mode: rank 0 decides after each round of num_samples and both
    ranks follow; the reduced film is the one-process render of every
    processed sample."""
    import torch.multiprocessing as mp
    import oracle
    world = 2
    mp.start_processes(_worker, args=(world, _free_port(), str(tmp_path), 0.5), nprocs=world, join=True,
                       start_method="spawn")
    r0 = np.load(tmp_path / "rank0.npy", allow_pickle=True).item()
    r1 = np.load(tmp_path / "rank1.npy", allow_pickle=True).item()
    n = 16 * 16 * SPP
    done = r0["processed"]
    assert done == r1["processed"] and done >= n and done % n == 0
    assert r1["film"] is None
    want = oracle.oracle_render_range(scenes.cornell_box(16, 16), 0, done, "pt.mis", RR, MAX_PV, SEED)
    np.testing.assert_allclose(r0["film"], want.reshape(16, 16, 3) * (16 * 16 / done), rtol=1e-5, atol=1e-7)


def test_mpi_termination_mode_validation():
    s = create_scheduler("mpi")
    s.set_termination_mode("time", 2.0)
    assert (s.termination_mode, s.termination_time) == ("time", 2.0)
    with pytest.raises(ValueError):
        s.set_termination_mode("time", -1)

