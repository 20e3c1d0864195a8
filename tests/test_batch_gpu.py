"""Multi-scene batch (lmgpu_batch_*): every scene of a batch must render the
same paths as the one-scene renderer with the same parameters, whatever the
batch configuration (mode, BVH layout, wave size, shading grid, overlap
bounce, CUDA graph or direct launches). With FP64 films the two differ only in the order of the
film additions, so they agree to ~1e-12 relative.
"""
import ctypes

import numpy as np
import pytest

from lightmetrica_b200 import HDRBitmapFilm, create_renderer, create_scene, native, scenes
from lightmetrica_b200.batch import SceneBatch

pytestmark = pytest.mark.gpu


def build(prims, layout="bvh"):
    s = create_scene(layout)
    s.load(prims)
    s.configure({})
    s.build()
    return s


def renderer(technique, rr_depth, max_pv, seed):
    r = create_renderer(technique)
    r.configure({"rr_depth": rr_depth, "max_path_vertices": max_pv, "sampler": {"rng_seed": seed}})
    return r


def small_set(technique="pt.mis"):
    """Scenes of different sizes, depths, seeds and sample counts."""
    items = []
    items.append((scenes.cornell_box(64, 64), renderer(technique, 3, 9, 1), 64 * 64 * 16))
    items.append((scenes.cornell_box(48, 40, variant="mixed"), renderer(technique, 2, 6, 7), 48 * 40 * 24))
    for i in range(4):
        d = scenes.batch_scene(i, seed=11)
        d["prims"].camera.film = HDRBitmapFilm(40 + 8 * i, 32 + 8 * i)
        W, H = d["prims"].camera.film.width, d["prims"].camera.film.height
        items.append((d["prims"], renderer(technique, 4, d["max_path_vertices"], 3 + i), W * H * (4 + 2 * i)))
    return items


def plain_films(built, items):
    import torch
    out = []
    for sc, (prims, r, n) in zip(built, items):
        W, H = prims.camera.film.width, prims.camera.film.height
        f = torch.zeros(W * H * 3, dtype=torch.float64, device="cuda")
        p = r.params(n, film_fp64=True)
        st = native.RenderStats()
        native.check(native.lib().lmgpu_render_device(sc.handle, ctypes.byref(p), ctypes.c_void_p(f.data_ptr()),
                                                      ctypes.c_void_p(torch.cuda.current_stream().cuda_stream),
                                                      ctypes.byref(st)))
        out.append(f)
    torch.cuda.synchronize()
    return [f.cpu().numpy() for f in out]


def batch_films(batch, items):
    import torch
    films = [torch.zeros(p.camera.film.width * p.camera.film.height * 3, dtype=torch.float64, device="cuda")
             for p, _, _ in items]
    batch.render_device([r for _, r, _ in items], [n for _, _, n in items], films)
    torch.cuda.synchronize()
    return [f.cpu().numpy() for f in films]


def assert_same(got, want):
    for g, w in zip(got, want):
        assert w.max() > 0
        np.testing.assert_allclose(g, w, rtol=1e-9, atol=1e-12)


@pytest.mark.parametrize("layout", ["bvh", "bvh_qshadow"])
@pytest.mark.parametrize("technique", ["pt.mis", "pt.direct", "pt"])
def test_batch_matches_one_scene_renders(cuda, technique, layout):
    items = small_set(technique)
    built = [build(p) for p, _, _ in items]
    want = plain_films(built, items)
    batch = SceneBatch(built)
    batch.configure(layout=layout)
    assert_same(batch_films(batch, items), want)
    st = batch.last_stats
    assert st["paths"] == sum(n for _, _, n in items)
    assert st["rays_traced"] > st["paths"] // 2 and st["max_bounces_run"] >= 5
    batch.close()


@pytest.mark.parametrize("config", [
    dict(layout="qbvh"),
    dict(wave_paths=4096),                       # many waves, every wave spans scenes
    dict(wave_paths=1 << 20, shade_blocks_per_sm=2),
    dict(use_graph=False),
    dict(layout="qbvh", wave_paths=10000, use_graph=False),
    dict(mode="waves"),
    dict(mode="waves", wave_paths=4096),         # many waves, every wave spans scenes
    dict(mode="waves", layout="qbvh", wave_paths=10000, use_graph=False),
    dict(mode="stream", wave_paths=4096),        # slots recycled many times, across scenes
    dict(mode="overlap"),                        # one wave: head, no period, tail
    dict(mode="overlap", wave_paths=4096),       # many waves in both pools
    dict(mode="overlap", wave_paths=5000, overlap_bounce=1),    # the whole path loop is the tail
    dict(mode="overlap", wave_paths=6000, overlap_bounce=12),   # split past the last bounce
    dict(mode="overlap", layout="qbvh", wave_paths=4096, overlap_bounce=4, use_graph=False),  # two streams
    dict(layout="bvh_q16"),                      # quantised nodes: boxes only grow, so the same hits here
    dict(mode="waves", layout="bvh_q16", wave_paths=10000, use_graph=False),
    dict(layout="bvh_qshadow"),                  # float nodes for bounce rays, quantised for shadow rays
    dict(mode="overlap", layout="bvh_qshadow", wave_paths=4096),
    dict(mode="stream", layout="bvh_qshadow", wave_paths=4096),
])
def test_batch_configurations_agree(cuda, config):
    items = small_set()
    built = [build(p) for p, _, _ in items]
    want = plain_films(built, items)
    batch = SceneBatch(built)
    batch.configure(**config)
    assert_same(batch_films(batch, items), want)
    assert_same(batch_films(batch, items), want)     # graph replay with a fresh table
    batch.close()


def _shifted(prims, offset):
    """The same scene moved by `offset` (geometry by its primitives'
    transforms, and the camera)."""
    import dataclasses
    M = np.eye(4)
    M[:3, 3] = offset
    moved = dataclasses.replace(prims, primitives=[dataclasses.replace(p, transform=M) for p in prims.primitives])
    cam = prims.camera
    moved.camera = dataclasses.replace(cam, eye=tuple(np.add(cam.eye, offset)), center=tuple(np.add(cam.center, offset)))
    return moved


@pytest.mark.parametrize("layout", ["bvh_q16", "bvh_qshadow"])
def test_quantised_layouts_on_a_deep_tree(cuda, layout):
    """A 256 x 256-vertex terrain with level-3 spheres (a deep tree of tiny
    triangles, quantisation steps down to ~1e-6): every quantised box holds
    its float box, so the walks find the float tree's hits and the films
    equal the one-scene renderer's. Far from the origin this stops holding
    exactly (a scene 100 units away differed in 0.26 % of its pixels): the
    render triangle test's rounding there admits hits just outside a
    triangle's edges, and the wider quantised boxes let more of those
    through than the float boxes do."""
    prims = scenes.terrain_spheres(64, 36, grid=256, spheres=8, ico_level=3)
    items = [(prims, renderer("pt.mis", 4, 9, 2), 64 * 36 * 8)]
    built = [build(p) for p, _, _ in items]
    want = plain_films(built, items)
    batch = SceneBatch(built)
    batch.configure(layout=layout)
    assert_same(batch_films(batch, items), want)
    batch.close()


@pytest.mark.parametrize("layout", ["bvh", "qbvh"])
@pytest.mark.parametrize("offset", [(100.0, -70.0, 130.0), (1000.0, -700.0, 1300.0)], ids=["100", "1000"])
def test_batch_far_from_origin(cuda, offset, layout):
    """Far from the origin the coordinates' float spacing grows (1.2e-4 at
    1,300): the batch's walks must still find exactly the one-scene
    renderer's hits."""
    items = [(_shifted(scenes.cornell_box(48, 48, variant="mixed"), offset), renderer("pt.mis", 3, 9, 3), 48 * 48 * 16)]
    built = [build(p) for p, _, _ in items]
    want = plain_films(built, items)
    batch = SceneBatch(built)
    batch.configure(layout=layout)
    assert_same(batch_films(batch, items), want)
    batch.close()


@pytest.mark.parametrize("mode", ["waves", "stream", "overlap"])
def test_batch_unbounded_depth_tail(cuda, mode):
    """max_path_vertices = -1 (Russian roulette only): in wave mode the graph
    covers the first bounces and direct launches finish the deep tail
    (overlap mode runs such renders as waves); in stream mode every path
    simply lives until it ends."""
    items = [(scenes.cornell_box(32, 32, variant="mixed"), renderer("pt.mis", 1, -1, 5), 32 * 32 * 32),
             (scenes.cornell_box(24, 24), renderer("pt.mis", 1, -1, 6), 24 * 24 * 16)]
    built = [build(p) for p, _, _ in items]
    want = plain_films(built, items)
    batch = SceneBatch(built)
    batch.configure(wave_paths=8192, mode=mode)
    assert_same(batch_films(batch, items), want)
    batch.close()


def test_mode_statistics(cuda):
    """Stream and overlap modes count the same rays as wave mode (same
    paths); stream mode reports its iterations, overlap mode its waves."""
    items = small_set()
    built = [build(p) for p, _, _ in items]
    batch = SceneBatch(built)
    stats = {}
    for mode in ("waves", "stream", "overlap"):
        batch.configure(mode=mode, wave_paths=8192)
        batch_films(batch, items)
        stats[mode] = dict(batch.last_stats)
    for mode in ("stream", "overlap"):
        for k in ("rays_traced", "shadow_rays", "max_bounces_run", "paths"):
            assert stats[mode][k] == stats["waves"][k], (mode, k)
    assert stats["stream"]["waves"] > 8     # iterations
    assert stats["overlap"]["waves"] == stats["waves"]["waves"] == -(-stats["waves"]["paths"] // 8192)
    batch.close()


def test_batch_repeated_scene_and_sample_offsets(cuda):
    """One scene twice with disjoint sample ranges equals one render of both ranges."""
    import torch
    prims = scenes.cornell_box(32, 32)
    sc = build(prims)
    r = renderer("pt.mis", 3, 9, 2)
    n = 32 * 32 * 8
    batch = SceneBatch([sc, sc])
    p = (native.RenderParams * 2)(r.params(n, film_fp64=True), r.params(n, sample_offset=n, film_fp64=True))
    f = torch.zeros(32 * 32 * 3, dtype=torch.float64, device="cuda")
    ptrs = (ctypes.c_void_p * 2)(f.data_ptr(), f.data_ptr())
    native.check(native.lib().lmgpu_batch_render_device(batch.handle, p, ptrs, None, None))
    torch.cuda.synchronize()
    want = plain_films([sc], [(prims, r, 2 * n)])[0]
    np.testing.assert_allclose(f.cpu().numpy(), want, rtol=1e-9, atol=1e-12)
    batch.close()


def test_batch_autotune_keeps_results(cuda):
    items = small_set()
    built = [build(p) for p, _, _ in items]
    want = plain_films(built, items)
    batch = SceneBatch(built)
    cfg = batch.autotune([r for _, r, _ in items], [n for _, _, n in items], sample_fraction=0.25)
    assert cfg["layout"] in ("bvh", "qbvh", "bvh_q16", "bvh_qshadow") and cfg["trial_ms"] > 0 and cfg["mode"] in ("waves", "stream", "overlap")
    assert 0 <= cfg["overlap_bounce"] <= 5
    assert cfg["wave_paths"] in (1 << 21, 1 << 22, 1 << 23, 1 << 24, 1 << 25, 1 << 26, 1 << 27)
    assert_same(batch_films(batch, items), want)
    batch.close()


def test_batch_rescaled_render_matches_scheduler(cuda):
    from lightmetrica_b200 import create_scheduler
    items = small_set()[:3]
    built = [build(p) for p, _, _ in items]
    batch = SceneBatch(built)
    films = batch.render([r for _, r, _ in items], [n for _, _, n in items])
    for sc, (prims, r, n), f in zip(built, items, films):
        s = create_scheduler("mt")
        s.configure({"num_samples": n})
        np.testing.assert_allclose(f, s.render(r, sc), rtol=2e-4, atol=1e-5)
    batch.close()


def test_batch_errors(cuda):
    import torch
    L = native.lib()
    a, b = build(scenes.cornell_box(16, 16)), build(scenes.cornell_box(16, 16))
    naive = build(scenes.cornell_box(16, 16), layout="naive")
    h = ctypes.c_void_p()
    assert L.lmgpu_batch_create((ctypes.c_void_p * 1)(naive.handle.value), 1, ctypes.byref(h)) == native.ERR_INVALID
    assert L.lmgpu_batch_create(None, 0, ctypes.byref(h)) == native.ERR_INVALID
    batch = SceneBatch([a, b])
    f = torch.zeros(16 * 16 * 3, device="cuda")
    ptrs = (ctypes.c_void_p * 2)(f.data_ptr(), f.data_ptr())
    p = (native.RenderParams * 2)(renderer("pt.mis", 3, 9, 1).params(256), renderer("pt", 3, 9, 1).params(256))
    assert L.lmgpu_batch_render_device(batch.handle, p, ptrs, None, None) == native.ERR_INVALID
    assert b"one technique" in L.lmgpu_last_error()
    p[1] = renderer("pt.mis", 3, 9, 1).params(0)
    assert L.lmgpu_batch_render_device(batch.handle, p, ptrs, None, None) == native.ERR_INVALID
    with pytest.raises(native.LmgpuError):
        batch.configure(wave_paths=16)
    with pytest.raises(native.LmgpuError):
        batch.configure(mode="overlap", overlap_bounce=65)
    with pytest.raises(ValueError):
        batch.configure(mode="pipelined")
    with pytest.raises(ValueError):
        batch.configure(layout="naive")
    batch.close()


def test_batch_profile_counts_and_times(cuda):
    """lmgpu_batch_profile: the counting and the timed measurement renders
    trace the same paths as a plain render (films equal the one-scene
    renderer's), and report per-kind rays, launches, device times and the
    traversal work counts."""
    import torch
    items = small_set()
    built = [build(p) for p, _, _ in items]
    want = plain_films(built, items)
    batch = SceneBatch(built)
    rs, ns = [r for _, r, _ in items], [n for _, _, n in items]
    films = [torch.zeros(p.camera.film.width * p.camera.film.height * 3, dtype=torch.float64, device="cuda")
             for p, _, _ in items]
    counted = batch.profile(rs, ns, films, count_tests=True)
    assert_same([f.cpu().numpy() for f in films], want)
    for f in films:
        f.zero_()
    timed = batch.profile(rs, ns, films, count_tests=False)
    assert_same([f.cpu().numpy() for f in films], want)
    batch.render_device(rs, ns, films)
    st = batch.last_stats
    for k in ("closest", "shadow"):
        c, t = counted[k], timed[k]
        assert c["rays"] == t["rays"] > 0 and c["launches"] == t["launches"] > 0
        assert t["trace_ms"] > 0
        # Every ray tests at least the root box; the scenes are hit often.
        assert c["node_tests"] >= c["rays"] and c["tri_tests"] > 0
    assert counted["closest"]["rays"] + counted["shadow"]["rays"] == st["rays_traced"]
    assert counted["shadow"]["rays"] == st["shadow_rays"]
    assert timed["render_ms"] > timed["closest"]["trace_ms"] + timed["shadow"]["trace_ms"]
    batch.close()


def test_batch_films_match_reference_goldens(cuda, golden_dir):
    """The golden Cornell scenes rendered inside a batch together with other
    scenes: each of their films against the reference's double-precision
    pt.mis image (relMSE <= 1e-3, the bar of the one-scene image tests)."""
    import os
    ref = {v: np.load(os.path.join(golden_dir, f"cornell_{v}_ref_mis.npz"))["film"] for v in ("classic", "mixed")}
    spp = 16384
    items = [(scenes.cornell_box(128, 128, variant="classic"), renderer("pt.mis", 3, 9, 7), 128 * 128 * spp),
             (scenes.cornell_box(128, 128, variant="mixed"), renderer("pt.mis", 3, 9, 8), 128 * 128 * spp)]
    items += small_set()[2:4]
    built = [build(p) for p, _, _ in items]
    batch = SceneBatch(built)
    films = batch.render([r for _, r, _ in items], [n for _, _, n in items])
    for variant, f in zip(("classic", "mixed"), films[:2]):
        e = float(np.mean((f - ref[variant]) ** 2 / (ref[variant] ** 2 + 1e-2)))
        print(f"batch {variant}: relMSE {e:.3e}")
        assert np.isfinite(f).all() and e <= 1e-3
    for f in films[2:]:
        assert np.isfinite(f).all() and f.max() > 0
    batch.close()
