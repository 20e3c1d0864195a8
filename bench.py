#!/usr/bin/env python
"""Benchmark of the B200 scene accelerator / path tracer.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--layout bvh|qbvh] [--sections render,adjoint]

Prints ONE JSON line on rank 0. Multi-GPU runs (torchrun, one process per
GPU) are independent replicas with weak scaling: every rank traces its own
seeded ray batch against its own copy of the scene; there is no data-path
collective. The job time is the max over ranks of the device time.

Workload `intersect` (the default): 2^24 rays (origins U[-2,2]^3, directions
uniform on the sphere) against 1,048,576 random triangles (centres U[-1,1]^3,
edges N(0, 0.01^2)), closest hit with the binary SAH BVH that reproduces the
reference BVHScene. One step = one launch over the whole ray batch, which is
larger than L2 (512 MB of rays), so no L2 flush is needed between steps.

At N=1 the same line carries `sections`: the full path tracer at 1920x1080
(3.4M-triangle terrain + icospheres, 64 spp, pt.mis, max depth 16, RR after
depth 4) in Mrays/s and spp/s with its relMSE against the reference's FP64
image, and the adjoint path replay's backward/forward time on the refined
Cornell box (512x512, 32 spp).
"""
from __future__ import annotations

import argparse
import ctypes
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

NUM_TRIS = 1 << 20
NUM_RAYS = 1 << 24
NODE_BYTES = 32      # compact binary node (6 f32 + 2 u32), per slab test
TRI_BYTES = 48       # TriAccel record, per triangle test
RAY_IO_BYTES = 32 + 16


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="intersect", choices=["intersect"])
    ap.add_argument("--layout", default="bvh", choices=["bvh", "qbvh"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true", help="skip the host-buffer pass (profiling runs)")
    ap.add_argument("--rays-log2", type=int, default=24, help="ray batch 2^k (profiling runs use less)")
    ap.add_argument("--render-spp", type=int, default=64, help="spp of the 1080p section (profiling runs use less)")
    ap.add_argument("--render-frames", type=int, default=3, help="timed frames of the 1080p section")
    ap.add_argument("--no-render-parity", action="store_true", help="skip the 1080p section's relMSE image")
    ap.add_argument("--batch-fraction", type=float, default=1.0,
                    help="scale every batch scene's sample count (profiling runs use less)")
    ap.add_argument("--batch-only", action="store_true",
                    help="batch section: only the batch, default configuration (profiling runs)")
    ap.add_argument("--sections", default="render,adjoint,batch",
                    help="extra single-GPU sections in the same line: render (1080p path tracer), "
                         "adjoint (forward/backward cost), batch (64-scene batch vs plain); '' for none")
    return ap.parse_args()


def dist_env():
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return rank, world, local


def measured_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.gpu = gpu_index
        self.proc = None
        self.lines = []
        self.thread = None

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.gpu}", f"--query-gpu={self.FIELDS}",
                                          "--format=csv,noheader,nounits", "-lms", "100"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except (FileNotFoundError, OSError):
            self.proc = None
            return
        self.thread = threading.Thread(target=self._read, daemon=True)
        self.thread.start()

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        if self.thread:
            self.thread.join(timeout=2)
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            parts = [x.strip() for x in ln.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                smax = float(parts[2])
            except ValueError:
                continue
            for nm, v in zip(names, parts[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": smax,
                "reasons": sorted(reasons), "samples": len(sm)}


def load_traffic(layout, num_rays):
    """DRAM bytes (read + write) of one full-size traversal launch, from the
    committed ncu summary of the kernel (profiles/): its line
    `dram_bytes_per_ray: X` (measured on a smaller capture, scaled by the
    rays of this launch), or None."""
    kernel_layout = {"bvh": "bvh2", "qbvh": "bvh4"}[layout]
    p = os.path.join(ROOT, "profiles", f"trace_closest_{kernel_layout}_intersect.md")
    if os.path.exists(p):
        with open(p) as f:
            for line in f:
                if line.startswith("dram_bytes_per_ray:"):
                    return int(float(line.split(":", 1)[1]) * num_rays)
    return None


# --------------------------------------------------------------- reference --

def cpu_reference_rate(pos, faces, rays, budget_s=12.0, threads=None):
    """The reference's own BVHScene (oracle/_ref, compiled from the reference
    sources) on the host cores: Mrays/s over a bounded sample of `rays`."""
    import oracle
    threads = threads or os.cpu_count() or 1
    if oracle.ref_available("f"):
        sc = oracle.RefScene(pos, faces, "bvh")
        kind = "reference"
        trace = lambda r: sc.intersect(r, threads=threads)  # noqa: E731
    else:
        sc = oracle.OracleScene(pos, faces, "bvh")
        kind = "port"
        threads = 1
        trace = lambda r: sc.intersect(r)  # noqa: E731
    n, done, t_total = 1 << 16, 0, 0.0
    while t_total < budget_s and done < rays.shape[0]:
        m = min(n, rays.shape[0] - done)
        t0 = time.perf_counter()
        trace(rays[done:done + m])
        t_total += time.perf_counter() - t0
        done += m
        n = min(n * 2, 1 << 22)
    return done / t_total / 1e6, kind, threads, done, t_total


def run_reference_arm(args):
    rank, world, _ = dist_env()
    if rank != 0:
        return
    from lightmetrica_b200.workloads import random_rays, random_soup
    pos, faces = random_soup(NUM_TRIS, seed=1)
    rays = random_rays(1 << 22, seed=2)
    import oracle
    threads = os.cpu_count() or 1
    if oracle.ref_available("f"):
        sc = oracle.RefScene(pos, faces, "bvh")
        kind = "reference"
        trace = lambda r: sc.intersect(r, threads=threads)  # noqa: E731
    else:
        sc = oracle.OracleScene(pos, faces, "bvh")
        kind, threads = "port", 1
        trace = lambda r: sc.intersect(r)  # noqa: E731
    # Each step: a bounded sample of the workload's rays (2^20 rays).
    sample = 1 << 20 if kind == "reference" else 1 << 15
    for w in range(args.warmup):
        trace(rays[:sample])
    times = []
    for k in range(args.steps):
        off = (k * sample) % (rays.shape[0] - sample + 1)
        t0 = time.perf_counter()
        trace(rays[off:off + sample])
        times.append(time.perf_counter() - t0)
    total = sum(times)
    value = sample * args.steps / total / 1e6
    line = {
        "impl": "reference", "metric": "closest-hit Mrays/s", "value": round(value, 4), "unit": "Mrays/s",
        "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": round(1e3 * total / args.steps, 3), "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": workload_config(args.layout),
        "cpu_baseline": {"value": round(value, 4), "unit": "Mrays/s", "cores": threads, "kind": kind,
                         "sample": f"{sample} rays per step of the 2^24-ray batch, BVHScene built once"},
        "e2e": {"value": round(value, 4), "unit": "Mrays/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def workload_config(layout, rays=NUM_RAYS):
    return {"workload": f"ray-intersection: 2^{rays.bit_length() - 1} rays x 1,048,576-triangle soup, closest hit",
            "rays": rays, "triangles": NUM_TRIS,
            "layout": {"bvh": "binary SAH BVH (reference bvh, bit-exact)",
                       "qbvh": "4-wide collapse of the reference tree (bit-exact)"}[layout],
            "l2": "inputs larger than L2 (512 MB of rays per step); no flush"}


# ---------------------------------------------------------------- ours ------

def run_ours(args):
    import torch
    rank, world, local = dist_env()
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    if world > 1:
        import torch.distributed as dist
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=120), device_id=dev)
    from lightmetrica_b200 import native
    from lightmetrica_b200.distributed import aggregate_rate, max_over_ranks
    from lightmetrica_b200.scene import Scene, soup_primitives
    from lightmetrica_b200.workloads import random_rays, random_soup, rays_soa

    pos, faces = random_soup(NUM_TRIS, seed=1)
    num_rays = 1 << args.rays_log2
    rays = random_rays(num_rays, seed=2 + rank)
    scene = Scene(args.layout)
    scene.load(soup_primitives(pos, faces))
    scene.configure({})
    scene.build()
    info = scene.info()

    n = num_rays
    soa = {k: torch.from_numpy(v).to(dev) for k, v in rays_soa(rays).items()}
    hits = {"tri_id": torch.empty(n, dtype=torch.int32, device=dev)}
    for k in ("t", "u", "v"):
        hits[k] = torch.empty(n, dtype=torch.float32, device=dev)
    R = native.RaysSoA(*[soa[k].data_ptr() for k in ("ox", "oy", "oz", "dx", "dy", "dz", "tmin", "tmax")])
    H = native.HitsSoA(*[hits[k].data_ptr() for k in ("tri_id", "t", "u", "v")])
    stream = torch.cuda.current_stream(dev)
    sptr = ctypes.c_void_p(stream.cuda_stream)
    L = native.lib()

    # Reference work per ray (binary slab tests, TriAccel tests), counted on
    # the device exactly as scene.bvh.cpp performs them; untimed.
    counters = torch.zeros(2, dtype=torch.int64, device=dev)
    native.check(L.lmgpu_intersect_counted(scene.handle, ctypes.byref(R), n, ctypes.byref(H),
                                           ctypes.c_void_p(counters.data_ptr()), sptr))
    scene.status(stream.cuda_stream)
    node_tests, tri_tests = int(counters[0]), int(counters[1])
    bytes_per_ray = RAY_IO_BYTES + NODE_BYTES * node_tests / n + TRI_BYTES * tri_tests / n
    hit_frac = float((hits["tri_id"] >= 0).float().mean())

    clocks = ClockSampler(local)
    clocks.start()
    for _ in range(args.warmup):
        native.check(L.lmgpu_intersect(scene.handle, ctypes.byref(R), n, ctypes.byref(H), sptr))
    torch.cuda.synchronize(dev)
    if world > 1:
        torch.distributed.barrier()
    torch.cuda.synchronize(dev)
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    t_start = torch.cuda.Event(enable_timing=True)
    t_end = torch.cuda.Event(enable_timing=True)
    t_start.record(stream)
    for k in range(args.steps):
        ev[k][0].record(stream)
        native.check(L.lmgpu_intersect(scene.handle, ctypes.byref(R), n, ctypes.byref(H), sptr))
        ev[k][1].record(stream)
    t_end.record(stream)
    torch.cuda.synchronize(dev)
    if world > 1:
        torch.distributed.barrier()
    torch.cuda.synchronize(dev)
    clk = clocks.stop()
    scene.status(stream.cuda_stream)
    total_ms = t_start.elapsed_time(t_end)
    launch_ms = [a.elapsed_time(b) for a, b in ev]
    total_ms = max_over_ranks(total_ms, device=dev)
    ms_per_step = total_ms / args.steps
    value = aggregate_rate(n, args.steps, total_ms, world) / 1e6

    # End to end through the host-buffer entry point: pinned AoS rays in, hit
    # arrays out, copies inside the timed region.
    e2e = None
    if not args.no_e2e:
        e2e = run_e2e(args, scene, rays, hits, world, dev)

    peak, peak_kind = measured_peaks()
    avg_launch_ms = sum(launch_ms) / len(launch_ms)
    achieved = bytes_per_ray * n / (avg_launch_ms / 1e3) / 1e9
    traffic = load_traffic(args.layout, n)

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        rate, kind, cores, done, secs = cpu_reference_rate(pos, faces, rays)
        cpu = {"value": round(rate, 4), "unit": "Mrays/s", "cores": cores, "kind": kind,
               "sample": f"first {done} rays of the 2^24-ray batch ({secs:.1f} s), reference BVHScene built once"}

    sections = run_sections(args, dev, rank, world)

    if rank == 0:
        line = {
            "metric": "closest-hit Mrays/s", "value": round(value, 3), "unit": "Mrays/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(ms_per_step, 4),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic (seeded; no public scene exists for this workload)",
            "config": dict(workload_config(args.layout, n), parallelism=f"replicas x{world}",
                           hit_fraction=round(hit_frac, 4), bvh_nodes=info["num_nodes"], bvh_depth=info["max_depth"],
                           build_seconds=round(info["build_seconds"], 3)),
            "e2e": e2e,
            "gpu_launches": args.steps,
            "roofline": {"bound": "hbm", "achieved": round(achieved, 1), "peak": peak, "unit": "GB/s",
                         "frac": round(achieved / peak, 4), "traffic": traffic,
                         "peak_source": peak_kind,
                         "bytes_per_ray": round(bytes_per_ray, 2),
                         "node_tests_per_ray": round(node_tests / n, 3), "tri_tests_per_ray": round(tri_tests / n, 4)},
            "cpu_baseline": cpu,
            "clocks": clk,
            "kernel_ms": {"avg": round(avg_launch_ms, 4), "min": round(min(launch_ms), 4),
                          "max": round(max(launch_ms), 4)},
        }
        if sections:
            line["sections"] = sections
        print(json.dumps(line), flush=True)
    if world > 1:
        torch.distributed.barrier()
        torch.distributed.destroy_process_group()


# ------------------------------------------------------------- sections ----

TERRAIN_W, TERRAIN_H = 1920, 1080
TERRAIN_RR, TERRAIN_MAX_PV = 5, 17       # Russian roulette after depth 4, max depth 16


def _timed_device_renders(L, scene, renderer, num_samples, film, stream, reps, native):
    """`reps` device renders of `num_samples` samples each (fresh sample
    ranges), each bracketed by CUDA events on the launching stream."""
    import torch
    out = []
    for k in range(reps):
        p = renderer.params(num_samples, sample_offset=k * num_samples)
        st = native.RenderStats()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(stream)
        native.check(L.lmgpu_render_device(scene.handle, ctypes.byref(p), ctypes.c_void_p(film.data_ptr()),
                                           ctypes.c_void_p(stream.cuda_stream), ctypes.byref(st)))
        b.record(stream)
        torch.cuda.synchronize()
        out.append((a.elapsed_time(b), st.rays_traced, st.shadow_rays, st.waves))
    return out


def render_section(args, dev, cpu_baseline):
    """The full path tracer at 1920 x 1080, 64 spp, pt.mis, max depth 16,
    Russian roulette after depth 4, on the 3.4M-triangle terrain + 64
    icosphere scene. relMSE is stated against the reference's FP64 pt.mis
    image of the same scene and camera at 96 x 54 (tests/golden, 16384 spp),
    rendered here at 65,536 spp."""
    import torch
    from lightmetrica_b200 import create_renderer, create_scene, create_scheduler, native, scenes
    L = native.lib()
    W, H, S = TERRAIN_W, TERRAIN_H, args.render_spp
    t0 = time.perf_counter()
    prims = scenes.terrain_spheres(W, H)
    gen_s = time.perf_counter() - t0
    scene = create_scene(args.layout)
    scene.load(prims)
    scene.configure({})
    scene.build()
    info = scene.info()
    r = create_renderer("pt.mis")
    r.configure({"rr_depth": TERRAIN_RR, "max_path_vertices": TERRAIN_MAX_PV, "sampler": {"rng_seed": 1}})
    stream = torch.cuda.current_stream(dev)
    film = torch.zeros(W * H * 3, dtype=torch.float32, device=dev)
    n = W * H * S
    _timed_device_renders(L, scene, r, n, film, stream, 1, native)          # warm-up
    runs = _timed_device_renders(L, scene, r, n, film, stream, max(1, args.render_frames), native)
    scene.status(stream.cuda_stream)
    ms = sum(x[0] for x in runs) / len(runs)
    rays = sum(x[1] for x in runs) / len(runs)
    shadow = sum(x[2] for x in runs) / len(runs)
    # The batch path with this one scene: autotuned configuration (untimed),
    # waves replayed from a captured CUDA graph, no host synchronisation.
    from lightmetrica_b200.batch import SceneBatch
    batch = SceneBatch([scene])
    t0 = time.perf_counter()
    tuned = batch.autotune([r], [n], sample_fraction=1.0 / 8)
    tune_s = time.perf_counter() - t0
    batch.render_device([r], [n], [film])                       # warm-up (graph capture)
    bruns = []
    for _ in range(max(1, args.render_frames)):
        batch.render_device([r], [n], [film])
        bruns.append((batch.last_stats["device_ms"], batch.last_stats["rays_traced"]))
    batch.close()
    b_ms = sum(x[0] for x in bruns) / len(bruns)
    b_rays = sum(x[1] for x in bruns) / len(bruns)
    # End to end through the scheduler (host film out, rescaled).
    sched = create_scheduler("mt")
    sched.configure({"num_samples": n})
    t0 = time.perf_counter()
    sched.render(r, scene)
    e2e_s = time.perf_counter() - t0
    scene.close()

    # Parity at the scaled-down size against the FP64 reference image.
    gold = np.load(os.path.join(ROOT, "tests", "golden", "terrain_ref_mis_96x54.npz"))
    rel = None
    if not args.no_render_parity:
        rel = _terrain_parity(args, r, gold)

    out = {
        "workload": f"full path tracer: {scenes.num_triangles(prims):,}-triangle fBm heightfield + 64 level-5 "
                    f"icospheres (diffuse / diffuse-mirror), spherical area light + constant environment 0.5, "
                    f"{W}x{H}, {S} spp, pt.mis, max depth 16, Russian roulette after depth 4",
        "Mrays_per_s": round(rays / (ms / 1e3) / 1e6, 1),
        "spp_per_s": round(S / (ms / 1e3), 2),
        "batched": {"Mrays_per_s": round(b_rays / (b_ms / 1e3) / 1e6, 1), "spp_per_s": round(S / (b_ms / 1e3), 2),
                    "ms_per_frame": round(b_ms, 2), "autotuned": tuned, "autotune_seconds": round(tune_s, 2),
                    "note": "the multi-scene batch path with this one scene: same samples, same paths"},
        "Msamples_per_s": round(n / (ms / 1e3) / 1e6, 2),
        "ms_per_frame": round(ms, 2), "rays_per_frame": int(rays), "shadow_rays_per_frame": int(shadow),
        "frames_timed": len(runs), "waves_per_frame": runs[0][3],
        "e2e": {"Mrays_per_s": round(rays / e2e_s / 1e6, 1), "seconds": round(e2e_s, 3),
                "d2h_bytes_per_step": W * H * 3 * 4, "h2d_bytes_per_step": 0},
        "relMSE_vs_fp64_reference": rel,
        "relMSE_case": "96x54 crop-free scale-down, same scene and camera; GPU 65,536 spp vs reference FP64 pt.mis "
                       f"{int(gold['spp'])} spp",
        "triangles": scenes.num_triangles(prims), "bvh_nodes": info["num_nodes"],
        "build_seconds": round(info["build_seconds"], 3), "scene_generation_seconds": round(gen_s, 2),
    }
    if cpu_baseline:
        out["cpu_baseline"] = _render_cpu_baseline(prims, n)
    return out


def _terrain_parity(args, r, gold):
    """relMSE of the terrain scene at 96 x 54 (65,536 spp) against the
    reference's FP64 image of the same scene and camera."""
    from lightmetrica_b200 import create_scene, create_scheduler, scenes
    small = scenes.terrain_spheres(96, 54)
    sc = create_scene(args.layout)
    sc.load(small)
    sc.configure({})
    sc.build()
    sched = create_scheduler("mt")
    sched.configure({"num_samples": 96 * 54 * 65536})
    img = sched.render(r, sc)
    sc.close()
    ref = gold["film"].astype(np.float64)
    return float(np.mean((img - ref) ** 2 / (ref ** 2 + 1e-2)))


def _render_cpu_baseline(prims, gpu_samples):
    """The reference's OpenMP pt.mis (oracle/_ref, float build, `mt`
    scheduler) on the host cores: a bounded 1-spp sample of the same frame."""
    try:
        import oracle
        if not oracle.ref_available("f"):
            return {"unavailable": "reference harness not built"}
        W, H = prims.camera.film.width, prims.camera.film.height
        threads = os.cpu_count() or 1
        samples = W * H
        _, secs = oracle.ref_render(prims, "pt.mis", num_samples=samples, rr_depth=TERRAIN_RR,
                                    max_path_vertices=TERRAIN_MAX_PV, seed=1, threads=threads, precision="f")
        return {"Msamples_per_s": round(samples / secs / 1e6, 4), "spp_per_s": round(samples / secs / (W * H), 4),
                "cores": threads, "kind": "reference",
                "sample": f"1 spp of the {W}x{H} frame ({samples:,} samples, {secs:.1f} s), BVHScene built untimed"}
    except Exception as e:      # a reported baseline only; never fails the bench
        return {"unavailable": str(e)[:200]}


def adjoint_section(args, dev):
    """Adjoint path replay on the Cornell box refined to 34,816 triangles,
    512 x 512, 32 spp, pt.mis (max depth 8, Russian roulette from depth 3):
    per-triangle albedo U[0.1, 0.9] (seed 1) against a target rendered with
    albedos of seed 2. Reports the backward / forward device-time ratio."""
    import torch
    from lightmetrica_b200 import create_renderer, create_scene, scenes
    from lightmetrica_b200.diff import DifferentiableRender, light_emission
    prims = scenes.cornell_refined(5, 512, 512)
    scene = create_scene(args.layout)
    scene.load(prims)
    scene.configure({})
    scene.build()
    r = create_renderer("pt.mis")
    r.configure({"rr_depth": 3, "max_path_vertices": 9, "sampler": {"rng_seed": 1}})
    dr = DifferentiableRender(scene, r, 512 * 512 * 32)
    T = scenes.num_triangles(prims)
    alb = torch.from_numpy(np.random.default_rng(1).uniform(0.1, 0.9, (T, 3)).astype(np.float32)).to(dev)
    alb_t = torch.from_numpy(np.random.default_rng(2).uniform(0.1, 0.9, (T, 3)).astype(np.float32)).to(dev)
    em = torch.from_numpy(light_emission(prims)).to(dev)
    target = dr.forward(alb_t, em)
    fwd, bwd = [], []
    for k in range(4):
        img = dr.forward(alb, em)
        f_ms = dr.last_forward_ms
        dL = 2.0 * (img - target)
        da, de = dr.backward(alb, em, dL)
        if k > 0:                       # first pair is warm-up
            fwd.append(f_ms)
            bwd.append(dr.last_backward_ms)
    torch.cuda.synchronize()
    loss = float(((img - target) ** 2).sum())
    scene.close()
    f, b = sum(fwd) / len(fwd), sum(bwd) / len(bwd)
    return {"workload": f"adjoint path replay: Cornell box refined to {T:,} triangles, 512x512, 32 spp, pt.mis, "
                        "max depth 8, RR from depth 3; d loss / d (per-triangle albedo, light emission)",
            "forward_ms": round(f, 3), "backward_ms": round(b, 3), "backward_over_forward": round(b / f, 3),
            "loss": loss, "grad_norm_albedo": float(da.norm()), "grad_emission": de.cpu().numpy().round(6).tolist()}


def batch_section(args, dev):
    """64 seeded scenes (random-triangle soups and fBm heightfields, 1k-200k
    triangles, 128^2-1024^2 films, 4-64 spp, max depth 8-16, Lambertian /
    mirror), pt.mis with Russian roulette after depth 4. Three ways to render
    the same samples: the batch (one stream of waves over all scenes, each
    wave a replayed CUDA graph, configuration from the autotuner), the plain
    one-scene-at-a-time wavefront renderer, and the plain one-scene megakernel
    (one thread per path, one launch per scene). The batch and the plain
    renderers trace the same paths, so their relMSE against any reference is
    equal; the films are compared to show it."""
    import torch
    from lightmetrica_b200 import create_renderer, create_scene, native, scenes
    from lightmetrica_b200.batch import SceneBatch
    from lightmetrica_b200.diff import DifferentiableRender, light_emission, triangle_albedo
    L = native.lib()
    t0 = time.perf_counter()
    items = [scenes.batch_scene(i) for i in range(64)]
    built, rs, ns, films = [], [], [], []
    for i, d in enumerate(items):
        sc = create_scene("bvh")
        sc.load(d["prims"])
        sc.configure({})
        sc.build()
        built.append(sc)
        r = create_renderer("pt.mis")
        r.configure({"rr_depth": 5, "max_path_vertices": d["max_path_vertices"], "sampler": {"rng_seed": i + 1}})
        rs.append(r)
        W = d["prims"].camera.film.width
        ns.append(max(1, int(W * W * d["spp"] * args.batch_fraction)))
        films.append(torch.zeros(W * W * 3, dtype=torch.float32, device=dev))
    setup_s = time.perf_counter() - t0
    stream = torch.cuda.current_stream(dev)
    total = sum(ns)

    def zero():
        for f in films:
            f.zero_()

    def plain_pass():
        st = native.RenderStats()
        rays = 0
        for sc, r, n, f in zip(built, rs, ns, films):
            p = r.params(n)
            native.check(L.lmgpu_render_device(sc.handle, ctypes.byref(p), ctypes.c_void_p(f.data_ptr()),
                                               ctypes.c_void_p(stream.cuda_stream), ctypes.byref(st)))
            rays += st.rays_traced
        return rays

    def timed(fn):
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        a.record(stream)
        out = fn()
        b.record(stream)
        torch.cuda.synchronize()
        return a.elapsed_time(b), out

    if args.batch_only:
        batch = SceneBatch(built)
        batch.render_device(rs, ns, films)
        batch_ms, _ = timed(lambda: batch.render_device(rs, ns, films, stats=False))
        batch.close()
        for sc in built:
            sc.close()
        return {"workload": "64-scene batch only (profiling run)", "samples": total, "batched_ms": round(batch_ms, 2),
                "config": "default"}

    # Batch configuration from the autotuner (untimed, like a build step).
    batch = SceneBatch(built)
    t0 = time.perf_counter()
    tuned = batch.autotune(rs, ns, sample_fraction=1.0 / 16)
    tune_s = time.perf_counter() - t0

    # One untimed pass of each renderer: warm-up, films for the comparison,
    # the batch's ray statistics.
    zero()
    plain_pass()
    plain = [f.clone() for f in films]
    zero()
    batch.render_device(rs, ns, films)
    st = batch.last_stats
    batched = [f.clone() for f in films]

    # Plain megakernel, one launch per scene (scene's own albedo and emission).
    drs = [DifferentiableRender(sc, r, n) for sc, r, n in zip(built, rs, ns)]
    params = [(torch.from_numpy(triangle_albedo(d["prims"])).to(dev), torch.from_numpy(light_emission(d["prims"])).to(dev))
              for d in items]

    def mega_pass():
        return [dr.forward(a, e) for dr, (a, e) in zip(drs, params)]
    mega_pass()

    # Timed: the three renderers in turn, `rounds` times, best time of each
    # (clocks and temperature drift by several percent over a run this long;
    # taking turns gives every renderer the same conditions).
    rounds = 3
    plain_ms = mega_ms = batch_ms = float("inf")
    plain_rays = 0
    for _ in range(rounds):
        ms, plain_rays = timed(plain_pass)
        plain_ms = min(plain_ms, ms)
        ms, _ = timed(mega_pass)
        mega_ms = min(mega_ms, ms)
        ms, _ = timed(lambda: batch.render_device(rs, ns, films, stats=False))
        batch_ms = min(batch_ms, ms)
    rel = []
    for a, b in zip(batched, plain):
        a64, b64 = a.double(), b.double()
        rel.append(float(((a64 - b64) ** 2 / (b64 ** 2 + 1e-2)).mean()))
    batch.close()
    for sc in built:
        sc.close()
    return {"workload": "64 scenes (soups / heightfields, log-uniform 1k-200k triangles, 128^2-1024^2, 4-64 spp, "
                        "max depth 8-16, Lambertian / mirror), pt.mis, RR after depth 4",
            "samples": total, "triangles": sum(d["triangles"] for d in items),
            "batched_ms": round(batch_ms, 2), "plain_wavefront_ms": round(plain_ms, 2),
            "plain_megakernel_ms": round(mega_ms, 2),
            "batched_over_plain_wavefront": round(plain_ms / batch_ms, 3),
            "batched_over_plain_megakernel": round(mega_ms / batch_ms, 3),
            "batched_Mrays_per_s": round(st["rays_traced"] / (batch_ms / 1e3) / 1e6, 1),
            "batched_Msamples_per_s": round(total / (batch_ms / 1e3) / 1e6, 1),
            "plain_wavefront_Mrays_per_s": round(plain_rays / (plain_ms / 1e3) / 1e6, 1),
            "waves": st["waves"], "autotuned": tuned, "autotune_seconds": round(tune_s, 2),
            "setup_seconds": round(setup_s, 2), "timing": f"best of {rounds} rounds, the three renderers in turn",
            "relMSE_batched_vs_plain_max": max(rel),
            "equal_relMSE": "same samples and paths in both; films differ only by float-atomic summation order"}


def run_sections(args, dev, rank, world):
    names = [x for x in args.sections.split(",") if x]
    if world > 1 or not names:
        return None
    out = {}
    if "render" in names:
        out["render_1080p"] = render_section(args, dev, cpu_baseline=(rank == 0 and not args.no_cpu_baseline))
    if "adjoint" in names:
        out["adjoint"] = adjoint_section(args, dev)
    if "batch" in names:
        out["batch64"] = batch_section(args, dev)
    return out


def run_e2e(args, scene, rays, hits, world, dev):
    """Same metric through the host-buffer entry point lmgpu_intersect_host:
    pinned AoS rays in, hit arrays out, copies inside the timed region."""
    import torch
    from lightmetrica_b200 import native
    from lightmetrica_b200.distributed import aggregate_rate, max_over_ranks
    L = native.lib()
    n = rays.shape[0]
    rays_pinned = torch.from_numpy(rays).pin_memory()
    out_id = torch.empty(n, dtype=torch.int32).pin_memory()
    out_t = torch.empty(n, dtype=torch.float32).pin_memory()
    out_u = torch.empty(n, dtype=torch.float32).pin_memory()
    out_v = torch.empty(n, dtype=torch.float32).pin_memory()
    e2e_steps = max(3, args.steps // 4)

    def e2e_once():
        native.check(L.lmgpu_intersect_host(scene.handle, rays_pinned.data_ptr(), n, out_id.data_ptr(),
                                            out_t.data_ptr(), out_u.data_ptr(), out_v.data_ptr()))
    e2e_once()
    if world > 1:
        torch.distributed.barrier()
    t0 = time.perf_counter()
    for _ in range(e2e_steps):
        e2e_once()
    e2e_s = max_over_ranks(time.perf_counter() - t0, device=dev)
    e2e_value = aggregate_rate(n, e2e_steps, e2e_s * 1e3, world) / 1e6
    assert np.array_equal(out_id.numpy(), hits["tri_id"].cpu().numpy()), "host and device paths disagree"
    return {"value": round(e2e_value, 3), "unit": "Mrays/s", "h2d_bytes_per_step": n * 32,
            "d2h_bytes_per_step": n * 16, "steps": e2e_steps}


def main():
    args = parse()
    if args.impl == "reference":
        run_reference_arm(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
