#!/usr/bin/env python
"""Benchmark of the B200 path tracer and scene accelerator.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--sections intersect,render,adjoint,batch]

Prints ONE JSON line on rank 0. Multi-GPU runs (torchrun, one process per
GPU) are independent replicas with weak scaling: every rank renders its own
frames (its own sample ranges) of its own copy of the scene; there is no
data-path collective. The job time is the max over ranks of the device time.

Headline workload: the full path tracer at 1920 x 1080, 64 spp, pt.mis, max
depth 16, Russian roulette after depth 4, on the 3,404,098-triangle scene
(a 1024 x 1024-vertex fBm heightfield and 64 level-5 icospheres, diffuse and
diffuse-mirror, a spherical area light and a constant environment of 0.5),
rendered through the multi-scene batch path (waves replayed from a captured
CUDA graph, configuration from the autotuner). One step = one whole frame
(132,710,400 samples) of fresh samples; the path state (28-39 GB) is far
larger than L2, so no flush is needed between steps. `value` is Mrays/s
(every closest-hit and shadow ray traced); `e2e` is the same through
SceneBatch.render (host film out, rescaled).

`--impl reference` times the reference's own OpenMP renderer (oracle/_ref:
its `mt` scheduler, `pt.mis`, `bvh` scene, float build) on the host cores
on the same scene and configuration, a bounded sample of the frame per step,
counting the rays its scene traces.

At N=1 the same line carries `sections`: the ray-intersection kernel (2^24
rays x 1,048,576-triangle soup, binary and 4-wide layouts, bit-exact against
the reference), the plain one-scene renderer on the headline frame, the
adjoint path replay's backward/forward time, and the 64-scene batch against
the plain renderers.
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
NODE4_BYTES = 128    # 4-wide node, per node fetch (four slab tests)
TRI_BYTES = 48       # TriAccel record, per triangle test
RAY_IO_BYTES = 32 + 16
# The headline metric, one string for both arms (the reference's renderer and
# this core's batched wavefront path trace the same frame).
FRAME_METRIC = "Mrays/s @1080p path tracing (pt.mis)"
QNODE_BYTES = 24     # quantised binary node (48 B: grid, 16-bit planes, children), per slab test


def node_bytes(layout: str, any_hit: bool) -> int:
    """Node bytes per slab test of a render walk under the batch layout."""
    quantised = layout == "bvh_q16" or (layout == "bvh_qshadow" and any_hit)
    return QNODE_BYTES if quantised else NODE_BYTES

# Headline frame: the full path tracer on the terrain + icospheres scene.
FRAME_W, FRAME_H = 1920, 1080
FRAME_RR, FRAME_MAX_PV = 5, 17       # Russian roulette after depth 4, max depth 16
REF_SAMPLES_PER_STEP = FRAME_W * FRAME_H // 4     # reference arm: a quarter of a spp per step


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true", help="skip the host-buffer passes (profiling runs)")
    ap.add_argument("--no-autotune", action="store_true", help="headline: the batch's default configuration")
    ap.add_argument("--frame-layout", default=None, choices=["bvh", "qbvh", "bvh_q16", "bvh_qshadow"],
                    help="headline: this node layout after any tuning (profiling runs)")
    ap.add_argument("--rays-log2", type=int, default=24, help="intersection section: ray batch 2^k")
    ap.add_argument("--render-spp", type=int, default=64, help="spp of the 1080p frame (profiling runs use less)")
    ap.add_argument("--render-frames", type=int, default=3, help="timed frames of the plain-renderer section")
    ap.add_argument("--no-render-parity", action="store_true", help="skip the relMSE image")
    ap.add_argument("--batch-fraction", type=float, default=1.0,
                    help="scale every batch scene's sample count (profiling runs use less)")
    ap.add_argument("--batch-only", action="store_true",
                    help="batch section: only the batch, default configuration (profiling runs)")
    ap.add_argument("--sections", default="intersect,render,adjoint,batch",
                    help="extra single-GPU sections in the same line: intersect (2^24-ray kernel, both layouts), "
                         "render (plain one-scene renderer on the frame), adjoint (forward/backward cost), "
                         "batch (64-scene batch vs plain); '' for none")
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


def profile_value(name, key):
    """A `key: value` line of a committed ncu summary (profiles/<name>.md),
    or None."""
    p = os.path.join(ROOT, "profiles", name + ".md")
    if os.path.exists(p):
        with open(p) as f:
            for line in f:
                if line.startswith(key + ":"):
                    return float(line.split(":", 1)[1])
    return None


def load_traffic(layout, num_rays):
    """DRAM bytes (read + write) of one full-size traversal launch of the
    intersection API, from the committed ncu summary of the kernel: its line
    `dram_bytes_per_ray: X` (measured on a smaller capture, scaled by the
    rays of this launch), or None."""
    kernel_layout = {"bvh": "bvh2", "qbvh": "bvh4"}[layout]
    v = profile_value(f"trace_closest_{kernel_layout}_intersect", "dram_bytes_per_ray")
    return None if v is None else int(v * num_rays)


def frame_config(world, triangles):
    """The headline workload: identical in both arms."""
    return {"workload": f"full path tracer: {triangles:,}-triangle fBm heightfield + 64 level-5 icospheres "
                        "(diffuse / diffuse-mirror), spherical area light + constant environment 0.5, "
                        f"{FRAME_W}x{FRAME_H}, 64 spp, pt.mis, max depth 16, Russian roulette after depth 4",
            "resolution": [FRAME_W, FRAME_H], "spp": 64, "technique": "pt.mis",
            "max_path_vertices": FRAME_MAX_PV, "rr_depth": FRAME_RR, "triangles": triangles,
            "rays": "every ray traced: camera, bounce and shadow rays",
            "l2": "path state and film far larger than L2 (126 MB); no flush",
            "parallelism": f"replicas x{world}"}


# --------------------------------------------------------------- reference --

def reference_render_rate(prims, samples_per_chunk, min_seconds, max_chunks, threads=None):
    """The reference's OpenMP pt.mis (oracle/_ref, float build, its `mt`
    scheduler and `bvh` scene) on the host cores: chunks of
    `samples_per_chunk` samples until `min_seconds` have passed (at most
    `max_chunks`); rays counted by the harness's counting scene."""
    import oracle
    threads = threads or os.cpu_count() or 1
    sess = oracle.RefRenderSession(prims, "pt.mis", rr_depth=FRAME_RR, max_path_vertices=FRAME_MAX_PV, seed=1)
    secs = rays = samples = 0
    chunks = 0
    while chunks < max_chunks and (chunks == 0 or secs < min_seconds):
        t, r, _ = sess.render(samples_per_chunk, threads=threads)
        secs += t
        rays += r
        samples += samples_per_chunk
        chunks += 1
    build = sess.build_seconds
    sess.close()
    return {"Mrays_per_s": rays / secs / 1e6, "Msamples_per_s": samples / secs / 1e6, "rays_per_sample": rays / samples,
            "seconds": secs, "samples": samples, "cores": threads, "build_seconds": build}


def cpu_reference_rate(pos, faces, rays, budget_s=12.0, threads=None, want_hits=False):
    """The reference's own BVHScene (oracle/_ref, compiled from the reference
    sources) on the host cores: Mrays/s over a bounded sample of `rays`, and
    with `want_hits` its hit ids and distances for the rays it traced."""
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
    ids, ts = [], []
    while t_total < budget_s and done < rays.shape[0]:
        m = min(n, rays.shape[0] - done)
        t0 = time.perf_counter()
        out = trace(rays[done:done + m])
        t_total += time.perf_counter() - t0
        if want_hits:
            ids.append(out["tri_id"])
            ts.append(out["t"])
        done += m
        n = min(n * 2, 1 << 22)
    hits = (np.concatenate(ids), np.concatenate(ts)) if want_hits else None
    return done / t_total / 1e6, kind, threads, done, t_total, hits


def run_reference_arm(args):
    """The reference's own renderer on the host cores, on the headline
    frame's scene and configuration: each step renders a bounded sample of
    the frame (a quarter of a sample per pixel, uniform raster positions as
    the reference samples them)."""
    rank, world, _ = dist_env()
    if rank != 0:
        return
    import oracle
    from lightmetrica_b200 import scenes
    prims = scenes.terrain_spheres(FRAME_W, FRAME_H)
    tris = scenes.num_triangles(prims)
    threads = os.cpu_count() or 1
    if not oracle.ref_available("f"):
        print(json.dumps({"impl": "reference", "unavailable": "reference harness (oracle/_ref) not built"}),
              flush=True)
        return
    sess = oracle.RefRenderSession(prims, "pt.mis", rr_depth=FRAME_RR, max_path_vertices=FRAME_MAX_PV, seed=1)
    sample = REF_SAMPLES_PER_STEP
    for _ in range(args.warmup):
        sess.render(sample, threads=threads)
    secs, rays = [], 0
    for _ in range(args.steps):
        t, r, _ = sess.render(sample, threads=threads)
        secs.append(t)
        rays += r
    build = sess.build_seconds
    sess.close()
    total = sum(secs)
    value = rays / total / 1e6
    line = {
        "impl": "reference", "metric": FRAME_METRIC, "value": round(value, 4),
        "unit": "Mrays/s", "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": round(1e3 * total / args.steps, 3), "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded; no public scene exists for this workload)",
        "config": frame_config(world, tris),
        "Msamples_per_s": round(sample * args.steps / total / 1e6, 4),
        "rays_per_sample": round(rays / (sample * args.steps), 4),
        "cpu_baseline": {"value": round(value, 4), "unit": "Mrays/s", "cores": threads, "kind": "reference",
                         "sample": f"{sample:,} samples per step (a quarter spp of the {FRAME_W}x{FRAME_H} frame, "
                                   f"uniform raster positions), the reference's mt scheduler with {threads} threads; "
                                   f"BVHScene built once ({build:.1f} s, untimed)"},
        "e2e": {"value": round(value, 4), "unit": "Mrays/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


# ---------------------------------------------------------------- ours ------

def _sum_over_ranks(value, dev, world):
    if world == 1:
        return float(value)
    import torch
    t = torch.tensor([float(value)], dtype=torch.float64, device=dev)
    torch.distributed.all_reduce(t)
    return float(t[0])


def _batch_launches(cfg, stats, bounces):
    """Kernels one batch render launches (captured or direct): per wave
    k_wave_begin, init, the camera-vertex shadow pass, `bounces` x (bounce
    prep, closest hit, shade, shadow), splat, k_wave_end, plus one setup
    kernel; stream mode: six kernels per iteration."""
    if cfg["mode"] == "stream":
        return 6 * stats["waves"] + 1
    return stats["waves"] * (5 + 4 * bounces) + 1


def frame_roofline(prof_count, prof_time, layout="bvh"):
    """Roofline of the dominant kernel of the frame, the closest-hit
    traversal of the path queues (and, beside it, the shadow traversal):
    algorithmic bytes per ray (32 B ray + 16 B hit + 32 B per binary-node
    slab test, 24 B for a quantised node, + 48 B per TriAccel test, the
    tests counted on the same samples by the counting kernel) over the
    launches' summed device time."""
    peak, peak_kind = measured_peaks()
    out = {}
    for kind in ("closest", "shadow"):
        c, t = prof_count[kind], prof_time[kind]
        rays = c["rays"]
        if rays == 0 or t["trace_ms"] <= 0:
            continue
        nb = c["node_tests"] / rays
        tb = c["tri_tests"] / rays
        bpr = RAY_IO_BYTES + node_bytes(layout, kind == "shadow") * nb + TRI_BYTES * tb
        achieved = bpr * rays / (t["trace_ms"] / 1e3) / 1e9
        out[kind] = {"achieved": round(achieved, 1), "frac": round(achieved / peak, 4),
                     "bytes_per_ray": round(bpr, 2), "node_tests_per_ray": round(nb, 3),
                     "tri_tests_per_ray": round(tb, 4), "rays": rays, "launches": t["launches"],
                     "avg_launch_ms": round(t["trace_ms"] / max(1, t["launches"]), 4),
                     "share_of_frame": round(t["trace_ms"] / prof_time["render_ms"], 4)}
    main = out["closest"]
    traffic_per_ray = profile_value("pathtrace_terrain_1080p_batched", "closest_dram_bytes_per_ray")
    return {"bound": "latency", "denominator": "hbm", "kernel": "k_trace_persistent (closest hit, path queues)",
            "achieved": main["achieved"], "peak": peak, "unit": "GB/s", "frac": main["frac"],
            "traffic": None if traffic_per_ray is None else int(traffic_per_ray * main["rays"] / main["launches"]),
            "peak_source": peak_kind,
            "why_not_hbm": "the tree and triangles (~250 MB) mostly hit in L2; each ray's walk is a chain of "
                           "dependent node fetches with a third of the lanes active, so the kernel is bound by "
                           "fetch latency and divergence, not DRAM bandwidth",
            "kernels": out}


def run_ours(args):
    import torch
    rank, world, local = dist_env()
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    if world > 1:
        import torch.distributed as dist
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=120), device_id=dev)
    from lightmetrica_b200 import create_renderer, create_scene, native, scenes
    from lightmetrica_b200.batch import SceneBatch
    from lightmetrica_b200.distributed import max_over_ranks

    W, H, S = FRAME_W, FRAME_H, args.render_spp
    t0 = time.perf_counter()
    prims = scenes.terrain_spheres(W, H)
    gen_s = time.perf_counter() - t0
    tris = scenes.num_triangles(prims)
    scene = create_scene("bvh")
    scene.load(prims)
    scene.configure({})
    scene.build()
    info = scene.info()
    r = create_renderer("pt.mis")
    r.configure({"rr_depth": FRAME_RR, "max_path_vertices": FRAME_MAX_PV, "sampler": {"rng_seed": 1}})
    n = W * H * S
    batch = SceneBatch([scene])
    tuned, tune_s = None, 0.0
    if not args.no_autotune:
        t0 = time.perf_counter()
        tuned = batch.autotune([r], [n], sample_fraction=1.0 / 8)
        tune_s = time.perf_counter() - t0
    if args.frame_layout:
        batch.configure(layout=args.frame_layout)
    stream = torch.cuda.current_stream(dev)
    film = torch.zeros(W * H * 3, dtype=torch.float32, device=dev)

    # Measurement renders (untimed): slab / TriAccel tests of every ray, then
    # the device time of every traversal launch, on the same samples.
    prof_count = batch.profile([r], [n], [film], count_tests=True)
    prof_time = batch.profile([r], [n], [film], count_tests=False)

    # Every step renders a whole frame of fresh samples (rank-disjoint).
    base = (rank * (args.warmup + args.steps + 64)) * n

    def frame(k, stats):
        batch.render_device([r], [n], [film], stats=stats, sample_offsets=base + k * n)
        return batch.last_stats["rays_traced"] if stats else 0

    for w in range(args.warmup):
        frame(w, False)
    torch.cuda.synchronize(dev)
    if world > 1:
        torch.distributed.barrier()
    torch.cuda.synchronize(dev)
    clocks = ClockSampler(local)
    clocks.start()
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    t_start = torch.cuda.Event(enable_timing=True)
    t_end = torch.cuda.Event(enable_timing=True)
    rays = 0
    t_start.record(stream)
    for k in range(args.steps):
        ev[k][0].record(stream)
        rays += frame(args.warmup + k, True)
        ev[k][1].record(stream)
    t_end.record(stream)
    torch.cuda.synchronize(dev)
    if world > 1:
        torch.distributed.barrier()
    torch.cuda.synchronize(dev)
    clk = clocks.stop()
    stats = batch.last_stats
    total_ms = max_over_ranks(t_start.elapsed_time(t_end), device=dev)
    frame_ms = [a.elapsed_time(b) for a, b in ev]
    all_rays = _sum_over_ranks(rays, dev, world)
    value = all_rays / (total_ms / 1e3) / 1e6
    samples_per_s = world * n * args.steps / (total_ms / 1e3)

    # End to end through SceneBatch.render: render parameters in, the
    # rescaled film out to a host array (copies inside the timed region).
    e2e = None
    if not args.no_e2e:
        out = [np.empty((H, W, 3), np.float32)]
        steps = max(3, args.steps // 4)
        batch.render([r], [n], sample_offsets=base, out=out)
        if world > 1:
            torch.distributed.barrier()
        e_rays = 0
        t0 = time.perf_counter()
        for k in range(steps):
            batch.render([r], [n], sample_offsets=base + (args.warmup + args.steps + k) * n, out=out)
            e_rays += batch.last_stats["rays_traced"]
        e2e_s = max_over_ranks(time.perf_counter() - t0, device=dev)
        e_all = _sum_over_ranks(e_rays, dev, world)
        e2e = {"value": round(e_all / e2e_s / 1e6, 3), "unit": "Mrays/s",
               "h2d_bytes_per_step": ctypes.sizeof(native.RenderParams), "d2h_bytes_per_step": W * H * 3 * 4,
               "steps": steps, "api": "SceneBatch.render -> lmgpu_batch_render (host film, rescaled)",
               "inputs": "the render parameters of the step (the scene stays resident in HBM)"}

    frame_layout = batch.config["layout"]
    roofline = frame_roofline(prof_count, prof_time, frame_layout)
    launches = _batch_launches(batch.config, stats, FRAME_MAX_PV - 1) * args.steps
    batch.close()

    rel = None
    if not args.no_render_parity and world == 1:
        rel = _terrain_parity(r, frame_layout)
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        try:
            c = reference_render_rate(prims, W * H, min_seconds=10.0, max_chunks=8)
            cpu = {"value": round(c["Mrays_per_s"], 4), "unit": "Mrays/s", "cores": c["cores"], "kind": "reference",
                   "Msamples_per_s": round(c["Msamples_per_s"], 4), "rays_per_sample": round(c["rays_per_sample"], 4),
                   "sample": f"{c['samples']:,} samples (whole-spp passes of the {W}x{H} frame, {c['seconds']:.1f} s), "
                             f"the reference's mt scheduler + pt.mis with {c['cores']} threads; BVHScene built once "
                             f"({c['build_seconds']:.1f} s, untimed)"}
        except Exception as e:      # a reported baseline only; never fails the bench
            cpu = {"unavailable": str(e)[:200]}
    scene.close()

    sections = run_sections(args, dev, rank, world)

    if rank == 0:
        line = {
            "metric": FRAME_METRIC, "value": round(value, 3),
            "unit": "Mrays/s", "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": round(total_ms / args.steps, 4), "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32",
            "data": "synthetic (seeded; no public scene exists for this workload)",
            "config": frame_config(world, tris),
            "spp_per_s": round(samples_per_s / (W * H), 3), "Msamples_per_s": round(samples_per_s / 1e6, 2),
            "rays_per_sample": round(all_rays / (world * n * args.steps), 4),
            "frame_ms": {"avg": round(sum(frame_ms) / len(frame_ms), 3), "min": round(min(frame_ms), 3),
                         "max": round(max(frame_ms), 3)},
            "relMSE_vs_fp64_reference": rel,
            "relMSE_case": "the same scene and camera at 96x54 through the same batch path and node layout, 65,536 spp, against "
                           "the reference's double-precision pt.mis at 16,384 spp (tests/golden); the full frame at "
                           "4096 spp would take the reference ~5 h on the host cores",
            "e2e": e2e,
            "gpu_launches": launches,
            "roofline": roofline,
            "cpu_baseline": cpu,
            "clocks": clk,
            "batch": {"config": batch_config_str(tuned), "autotune_seconds": round(tune_s, 2),
                      "waves_per_frame": stats["waves"], "max_bounces_run": stats["max_bounces_run"]},
            "scene": {"bvh_nodes": info["num_nodes"], "bvh_depth": info["max_depth"],
                      "build_seconds": round(info["build_seconds"], 3), "generation_seconds": round(gen_s, 2)},
        }
        if sections:
            line["sections"] = sections
        print(json.dumps(line), flush=True)
    if world > 1:
        torch.distributed.barrier()
        torch.distributed.destroy_process_group()


def batch_config_str(tuned):
    return "default (not autotuned)" if tuned is None else {k: v for k, v in tuned.items()}


def _terrain_parity(r, layout="bvh"):
    """relMSE of the terrain scene at 96 x 54 (65,536 spp, through the batch
    path with the headline's node layout) against the reference's FP64 image
    of the same scene and camera."""
    from lightmetrica_b200 import create_scene, scenes
    from lightmetrica_b200.batch import SceneBatch
    gold = np.load(os.path.join(ROOT, "tests", "golden", "terrain_ref_mis_96x54.npz"))
    small = scenes.terrain_spheres(96, 54)
    sc = create_scene("bvh")
    sc.load(small)
    sc.configure({})
    sc.build()
    b = SceneBatch([sc])
    b.configure(layout=layout)
    img = b.render([r], [96 * 54 * 65536])[0]
    b.close()
    sc.close()
    ref = gold["film"].astype(np.float64)
    return float(np.mean((img - ref) ** 2 / (ref ** 2 + 1e-2)))


# ------------------------------------------------------------- sections ----

def intersect_section(args, dev, layout, cpu_baseline, want_ref_hits):
    """The ray-intersection kernel alone: 2^24 rays (origins U[-2,2]^3,
    directions uniform on the sphere) against 1,048,576 random triangles
    (centres U[-1,1]^3, edges N(0, 0.01^2)), closest hit. Layout "bvh" is the
    binary SAH tree that reproduces the reference BVHScene; "qbvh" its 4-wide
    collapse. One launch per step over the batch (512 MB of rays, larger
    than L2)."""
    import torch
    from lightmetrica_b200 import native
    from lightmetrica_b200.scene import Scene, soup_primitives
    from lightmetrica_b200.workloads import random_rays, random_soup, rays_soa

    pos, faces = random_soup(NUM_TRIS, seed=1)
    num_rays = 1 << args.rays_log2
    rays = random_rays(num_rays, seed=2)
    scene = Scene(layout)
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
    Hh = native.HitsSoA(*[hits[k].data_ptr() for k in ("tri_id", "t", "u", "v")])
    stream = torch.cuda.current_stream(dev)
    sptr = ctypes.c_void_p(stream.cuda_stream)
    L = native.lib()

    # Work per ray (slab tests, TriAccel tests), counted on the device; untimed.
    counters = torch.zeros(2, dtype=torch.int64, device=dev)
    native.check(L.lmgpu_intersect_counted(scene.handle, ctypes.byref(R), n, ctypes.byref(Hh),
                                           ctypes.c_void_p(counters.data_ptr()), sptr))
    scene.status(stream.cuda_stream)
    node_tests, tri_tests = int(counters[0]), int(counters[1])
    if layout == "bvh":
        bytes_per_ray = RAY_IO_BYTES + NODE_BYTES * node_tests / n + TRI_BYTES * tri_tests / n
    else:
        bytes_per_ray = RAY_IO_BYTES + NODE4_BYTES * (node_tests / 4) / n + TRI_BYTES * tri_tests / n
    hit_frac = float((hits["tri_id"] >= 0).float().mean())

    steps, warm = max(3, args.steps), max(3, args.warmup)
    for _ in range(warm):
        native.check(L.lmgpu_intersect(scene.handle, ctypes.byref(R), n, ctypes.byref(Hh), sptr))
    torch.cuda.synchronize(dev)
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(steps)]
    for k in range(steps):
        ev[k][0].record(stream)
        native.check(L.lmgpu_intersect(scene.handle, ctypes.byref(R), n, ctypes.byref(Hh), sptr))
        ev[k][1].record(stream)
    torch.cuda.synchronize(dev)
    scene.status(stream.cuda_stream)
    launch_ms = [a.elapsed_time(b) for a, b in ev]
    avg_ms = sum(launch_ms) / len(launch_ms)
    peak, peak_kind = measured_peaks()
    achieved = bytes_per_ray * n / (avg_ms / 1e3) / 1e9
    out = {"workload": f"ray-intersection: 2^{n.bit_length() - 1} rays x 1,048,576-triangle soup, closest hit",
           "layout": {"bvh": "binary SAH BVH (reference bvh, bit-exact)",
                      "qbvh": "4-wide collapse of the reference tree, 128 B nodes (bit-exact)"}[layout],
           "Mrays_per_s": round(n / (avg_ms / 1e3) / 1e6, 1),
           "kernel_ms": {"avg": round(avg_ms, 4), "min": round(min(launch_ms), 4), "max": round(max(launch_ms), 4)},
           "steps": steps, "hit_fraction": round(hit_frac, 4),
           "roofline": {"bound": "latency", "denominator": "hbm", "achieved": round(achieved, 1), "peak": peak,
                        "unit": "GB/s", "frac": round(achieved / peak, 4), "traffic": load_traffic(layout, n),
                        "peak_source": peak_kind, "bytes_per_ray": round(bytes_per_ray, 2),
                        "node_tests_per_ray": round(node_tests / n, 3), "tri_tests_per_ray": round(tri_tests / n, 4)},
           "bvh_nodes": info["num_nodes"], "bvh_depth": info["max_depth"],
           "build_seconds": round(info["build_seconds"], 3)}
    if layout == "qbvh":
        out["node_fetches_per_ray"] = round(node_tests / 4 / n, 3)
    if not args.no_e2e and layout == "bvh":
        out["e2e"] = run_e2e(args, scene, rays, hits, dev)
    ids = hits["tri_id"].cpu().numpy()
    tv = hits["t"].cpu().numpy()
    scene.close()
    if cpu_baseline:
        rate, kind, cores, done, secs, rh = cpu_reference_rate(pos, faces, rays, want_hits=want_ref_hits)
        out["cpu_baseline"] = {"value": round(rate, 4), "unit": "Mrays/s", "cores": cores, "kind": kind,
                               "sample": f"first {done} rays of the batch ({secs:.1f} s), reference BVHScene built once"}
        if rh is not None:
            hit = rh[0] >= 0
            out["vs_reference"] = {"rays_compared": int(done),
                                   "ids_bit_exact": bool(np.array_equal(ids[:done], rh[0])),
                                   "t_bit_equal": bool(np.array_equal(tv[:done][hit], rh[1][hit]))}
    return out, ids, tv


def run_e2e(args, scene, rays, hits, dev):
    """Same metric through the host-buffer entry point lmgpu_intersect_host:
    pinned AoS rays in, hit arrays out, copies inside the timed region."""
    import torch
    from lightmetrica_b200 import native
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
    t0 = time.perf_counter()
    for _ in range(e2e_steps):
        e2e_once()
    e2e_s = time.perf_counter() - t0
    assert np.array_equal(out_id.numpy(), hits["tri_id"].cpu().numpy()), "host and device paths disagree"
    return {"value": round(n * e2e_steps / e2e_s / 1e6, 3), "unit": "Mrays/s", "h2d_bytes_per_step": n * 32,
            "d2h_bytes_per_step": n * 16, "steps": e2e_steps}


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


def render_section(args, dev):
    """The plain one-scene wavefront renderer (lmgpu_render_device: the host
    reads each bounce's queue sizes back to size the next launch) on the
    headline frame, and end to end through the scheduler (host film)."""
    import torch
    from lightmetrica_b200 import create_renderer, create_scene, create_scheduler, native, scenes
    L = native.lib()
    W, H, S = FRAME_W, FRAME_H, args.render_spp
    prims = scenes.terrain_spheres(W, H)
    scene = create_scene("bvh")
    scene.load(prims)
    scene.configure({})
    scene.build()
    r = create_renderer("pt.mis")
    r.configure({"rr_depth": FRAME_RR, "max_path_vertices": FRAME_MAX_PV, "sampler": {"rng_seed": 1}})
    stream = torch.cuda.current_stream(dev)
    film = torch.zeros(W * H * 3, dtype=torch.float32, device=dev)
    n = W * H * S
    _timed_device_renders(L, scene, r, n, film, stream, 1, native)          # warm-up
    runs = _timed_device_renders(L, scene, r, n, film, stream, max(1, args.render_frames), native)
    scene.status(stream.cuda_stream)
    ms = sum(x[0] for x in runs) / len(runs)
    rays = sum(x[1] for x in runs) / len(runs)
    shadow = sum(x[2] for x in runs) / len(runs)
    sched = create_scheduler("mt")
    sched.configure({"num_samples": n})
    t0 = time.perf_counter()
    sched.render(r, scene)
    e2e_s = time.perf_counter() - t0
    scene.close()
    return {"workload": "the headline frame through the plain one-scene wavefront renderer (lmgpu_render_device)",
            "Mrays_per_s": round(rays / (ms / 1e3) / 1e6, 1), "spp_per_s": round(S / (ms / 1e3), 2),
            "Msamples_per_s": round(n / (ms / 1e3) / 1e6, 2), "ms_per_frame": round(ms, 2),
            "rays_per_frame": int(rays), "shadow_rays_per_frame": int(shadow), "frames_timed": len(runs),
            "waves_per_frame": runs[0][3],
            "e2e_scheduler": {"Mrays_per_s": round(rays / e2e_s / 1e6, 1), "seconds": round(e2e_s, 3),
                              "d2h_bytes_per_step": W * H * 3 * 4, "h2d_bytes_per_step": 0},
            "relMSE": "same samples and paths as the batched headline: its relMSE applies"}


def adjoint_section(args, dev):
    """Adjoint path replay on the Cornell box refined to 36,864 triangles
    (every triangle of the 36-triangle box split into 4^5), 512 x 512, 32
    spp, pt.mis (max depth 8, Russian roulette from depth 3): per-triangle
    albedo U[0.1, 0.9] (seed 1) against a target rendered with albedos of
    seed 2. Reports the backward / forward device-time ratio, and the forward
    image with the scene's own albedos against the wavefront renderer's image
    of the same samples (the renderer whose images are pinned to the
    reference's FP64 renders)."""
    import torch
    from lightmetrica_b200 import create_renderer, create_scene, create_scheduler, scenes
    from lightmetrica_b200.diff import DifferentiableRender, light_emission, triangle_albedo
    prims = scenes.cornell_refined(5, 512, 512)
    scene = create_scene("bvh")
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
    own = dr.forward(torch.from_numpy(triangle_albedo(prims)).to(dev), em).double().cpu().numpy()
    sched = create_scheduler("mt")
    sched.configure({"num_samples": 512 * 512 * 32, "film_fp64": True})
    wf = sched.render(r, scene).astype(np.float64)
    fwd_rel = float(np.mean((own - wf) ** 2 / (wf ** 2 + 1e-2)))
    scene.close()
    f, b = sum(fwd) / len(fwd), sum(bwd) / len(bwd)
    return {"workload": f"adjoint path replay: Cornell box refined to {T:,} triangles, 512x512, 32 spp, pt.mis, "
                        "max depth 8, RR from depth 3; d loss / d (per-triangle albedo, light emission)",
            "forward_ms": round(f, 3), "backward_ms": round(b, 3), "backward_over_forward": round(b / f, 3),
            "loss": loss, "grad_norm_albedo": float(da.norm()), "grad_emission": de.cpu().numpy().round(6).tolist(),
            "forward_relMSE_vs_wavefront": fwd_rel,
            "forward_relMSE_case": "forward image with the scene's own albedos against the wavefront renderer's "
                                   "image of the same samples (FP64 film)"}


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
    if "intersect" in names:
        cpu = rank == 0 and not args.no_cpu_baseline
        out["intersect"], ids, tv = intersect_section(args, dev, "bvh", cpu, want_ref_hits=cpu)
        q, qids, qt = intersect_section(args, dev, "qbvh", False, False)
        hit = ids >= 0
        q["bit_exact_vs_bvh"] = bool(np.array_equal(qids, ids) and np.array_equal(qt[hit], tv[hit]))
        out["intersect_qbvh"] = q
    if "render" in names:
        out["render_1080p_plain"] = render_section(args, dev)
    if "adjoint" in names:
        out["adjoint"] = adjoint_section(args, dev)
    if "batch" in names:
        out["batch64"] = batch_section(args, dev)
    return out


def main():
    args = parse()
    if args.impl == "reference":
        run_reference_arm(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
