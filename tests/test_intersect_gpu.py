"""Parity of the sm_100a closest-hit kernels with the reference's BVHScene.

Bar: bit-exact triangle ids, t, u, v (integer/index work: no tolerance) for
the exact layouts (bvh = binary, qbvh = 4-wide collapse of the same tree) and
for naive vs the reference naive scene. Geometry reconstructed from the hit
(p, gn, sn, ss, st, uv) is compared within 1e-3, the reference tests'
EpsLarge for float (src/lightmetrica.test, base.math.h:78-82).
"""
import ctypes
import os

import numpy as np
import pytest

import oracle
from lightmetrica_b200 import native
from lightmetrica_b200.scene import Scene, soup_primitives
from lightmetrica_b200.workloads import FLT_MAX, random_rays, random_soup, rays_soa

pytestmark = pytest.mark.gpu

LAYOUTS = ["bvh", "qbvh"]


def gpu_scene(pos, faces, layout="bvh", normals=None, texcoords=None):
    s = Scene(layout)
    s.load(soup_primitives(pos, faces, normals, texcoords))
    s.configure({})
    s.build()
    return s


def _golden(golden_dir, name):
    return np.load(os.path.join(golden_dir, name))


@pytest.mark.parametrize("layout", LAYOUTS)
def test_soup_small_bit_exact_vs_reference(cuda, golden_dir, layout):
    d = _golden(golden_dir, "soup_small.npz")
    s = gpu_scene(d["positions"], d["faces"], layout)
    r = s.intersect_host(d["rays"])
    np.testing.assert_array_equal(r["tri_id"], d["bvh_tri_id"])
    hit = r["tri_id"] >= 0
    for k in ("t", "u", "v"):
        np.testing.assert_array_equal(r[k][hit], d[f"bvh_{k}"][hit])


@pytest.mark.parametrize("name", ["intersect_simple.npz", "intersect_simple2.npz", "consistency_random.npz",
                                  "soup_duplicates.npz"])
@pytest.mark.parametrize("layout,ref_kind", [("bvh", "bvh"), ("qbvh", "bvh"), ("naive", "naive")])
def test_reference_fixtures_ids_bit_exact(cuda, golden_dir, name, layout, ref_kind):
    d = _golden(golden_dir, name)
    s = gpu_scene(d["positions"], d["faces"], layout, d.get("normals"), d.get("texcoords"))
    r = s.intersect_host(d["rays"])
    np.testing.assert_array_equal(r["tri_id"], d[f"{ref_kind}_tri_id"])
    hit = r["tri_id"] >= 0
    np.testing.assert_array_equal(r["t"][hit], d[f"{ref_kind}_t"][hit])


@pytest.mark.parametrize("name", ["intersect_simple.npz", "intersect_simple2.npz", "consistency_random.npz"])
def test_hit_geometry_matches_reference(cuda, golden_dir, name):
    """Scene::Intersect's hit record (scene.cpp:101-149) within EpsLarge."""
    d = _golden(golden_dir, name)
    s = gpu_scene(d["positions"], d["faces"], "bvh", d.get("normals"), d.get("texcoords"))
    r = s.intersect_full_host(d["rays"])
    hit = d["bvh_tri_id"] >= 0
    assert (r["kind"][hit] == 1).all() and (r["kind"][~hit] == 0).all()
    keys = ["p", "gn", "sn", "ss", "st"] + (["uv"] if "texcoords" in d else [])
    for k in keys:
        np.testing.assert_allclose(r[k][hit], d[f"bvh_{k}"][hit], atol=1e-3, rtol=0, err_msg=k)


def test_simple_known_answers(cuda, golden_dir):
    """Intersect_Simple known answers: p = (x, y, 0), gn = sn = (0,0,1), uv = (x, y)."""
    d = _golden(golden_dir, "intersect_simple.npz")
    s = gpu_scene(d["positions"], d["faces"], "bvh", d["normals"], d["texcoords"])
    r = s.intersect_full_host(d["rays"])
    xs = np.array([0.1 * j for i in range(1, 10) for j in range(1, 10)])
    ys = np.array([0.1 * i for i in range(1, 10) for j in range(1, 10)])
    np.testing.assert_allclose(r["p"], np.stack([xs, ys, 0 * xs], 1), atol=1e-3)
    np.testing.assert_allclose(r["gn"], np.tile([0, 0, 1.0], (81, 1)), atol=1e-3)
    np.testing.assert_allclose(r["uv"], np.stack([xs, ys], 1), atol=1e-3)


@pytest.mark.parametrize("layout", LAYOUTS)
@pytest.mark.parametrize("ntris,sigma,nrays", [(262144, 0.02, 100000), (4096, 0.4, 50000)])
def test_random_soup_vs_oracle(cuda, layout, ntris, sigma, nrays):
    pos, faces = random_soup(ntris, seed=21, sigma=sigma)
    rays = random_rays(nrays, seed=22)
    o = oracle.OracleScene(pos, faces, "bvh").intersect(rays)
    r = gpu_scene(pos, faces, layout).intersect_host(rays)
    np.testing.assert_array_equal(r["tri_id"], o["tri_id"])
    hit = o["tri_id"] >= 0
    for k in ("t", "u", "v"):
        np.testing.assert_array_equal(r[k][hit], o[k][hit])


def test_device_api_and_counters_match_oracle(cuda):
    """lmgpu_intersect (device SoA buffers) and the reference work counters."""
    import torch
    pos, faces = random_soup(50000, seed=31, sigma=0.05)
    rays = random_rays(40000, seed=32)
    o = oracle.OracleScene(pos, faces, "bvh").intersect(rays)
    s = gpu_scene(pos, faces, "bvh")
    soa = {k: torch.from_numpy(v).to(cuda) for k, v in rays_soa(rays).items()}
    n = rays.shape[0]
    out = {"tri_id": torch.empty(n, dtype=torch.int32, device=cuda)}
    for k in ("t", "u", "v"):
        out[k] = torch.empty(n, dtype=torch.float32, device=cuda)
    counters = torch.zeros(2, dtype=torch.int64, device=cuda)
    R = native.RaysSoA(*[soa[k].data_ptr() for k in ("ox", "oy", "oz", "dx", "dy", "dz", "tmin", "tmax")])
    H = native.HitsSoA(*[out[k].data_ptr() for k in ("tri_id", "t", "u", "v")])
    stream = torch.cuda.current_stream().cuda_stream
    native.check(native.lib().lmgpu_intersect_counted(s.handle, ctypes.byref(R), n, ctypes.byref(H),
                                                      ctypes.c_void_p(counters.data_ptr()), ctypes.c_void_p(stream)))
    s.status(stream)
    np.testing.assert_array_equal(out["tri_id"].cpu().numpy(), o["tri_id"])
    assert int(counters[0]) == int(o["node_tests"].sum())
    assert int(counters[1]) == int(o["tri_tests"].sum())
    # Plain device entry point gives the same answer.
    out2 = torch.full((n,), -7, dtype=torch.int32, device=cuda)
    s.intersect_device({k: soa[k].data_ptr() for k in soa}, {"tri_id": out2.data_ptr()}, n, stream)
    s.status(stream)
    np.testing.assert_array_equal(out2.cpu().numpy(), o["tri_id"])


def test_occluded_equals_closest_hit_exists(cuda):
    import torch
    pos, faces = random_soup(20000, seed=41, sigma=0.08)
    rays = random_rays(30000, seed=42)
    rays[:, 7] = np.random.default_rng(3).uniform(0.1, 4.0, rays.shape[0]).astype(np.float32)
    o = oracle.OracleScene(pos, faces, "bvh").intersect(rays)
    for layout in ("bvh", "qbvh", "naive"):
        s = gpu_scene(pos, faces, layout)
        soa = {k: torch.from_numpy(v).to(cuda) for k, v in rays_soa(rays).items()}
        occ = torch.zeros(rays.shape[0], dtype=torch.uint8, device=cuda)
        s.occluded_device({k: soa[k].data_ptr() for k in soa}, occ.data_ptr(), rays.shape[0],
                          torch.cuda.current_stream().cuda_stream)
        s.status(torch.cuda.current_stream().cuda_stream)
        np.testing.assert_array_equal(occ.cpu().numpy().astype(bool), o["tri_id"] >= 0)


def test_edge_cases(cuda):
    # Axis-aligned rays with zero direction components over a cube of shared
    # edges (exact ties between neighbouring triangles), rays with
    # tmin > tmax, rays starting on a face, and a degenerate triangle.
    cube = np.array([[x, y, z] for x in (0, 1) for y in (0, 1) for z in (0, 1)], np.float32)
    quads = [(0, 1, 3, 2), (4, 6, 7, 5), (0, 4, 5, 1), (2, 3, 7, 6), (0, 2, 6, 4), (1, 5, 7, 3)]
    f = []
    for a, b, c, d in quads:
        f += [[a, b, c], [a, c, d]]
    pos = np.concatenate([cube, np.array([[0.5, 0.5, 0.5], [0.5, 0.5, 0.5], [0.6, 0.6, 0.6]], np.float32)])
    faces = np.array(f + [[8, 9, 10]], np.uint32)
    rng = np.random.default_rng(5)
    rays = []
    for _ in range(3000):
        o = rng.choice([-0.5, 0.0, 0.25, 0.5, 1.0, 1.5], 3)
        d = np.zeros(3)
        d[rng.integers(0, 3)] = rng.choice([-1.0, 1.0])
        if rng.random() < 0.3:
            d[rng.integers(0, 3)] = rng.choice([-1.0, 0.5, 1.0])
        if not d.any():
            d[0] = 1.0
        tmin, tmax = (0.0, FLT_MAX) if rng.random() < 0.8 else (2.0, 1.0)
        rays.append([*o, *d, tmin, tmax])
    rays = np.array(rays, np.float32)
    ref = oracle.RefScene(pos, faces, "bvh").intersect(rays) if oracle.ref_available("f") else None
    o = oracle.OracleScene(pos, faces, "bvh").intersect(rays)
    if ref is not None:
        np.testing.assert_array_equal(o["tri_id"], ref["tri_id"])
    for layout in LAYOUTS:
        r = gpu_scene(pos, faces, layout).intersect_host(rays)
        np.testing.assert_array_equal(r["tri_id"], o["tri_id"])
        hit = o["tri_id"] >= 0
        np.testing.assert_array_equal(r["t"][hit], o["t"][hit])
    assert not (o["tri_id"] == 12).any()  # degenerate triangle never hit


def test_empty_and_single_triangle_scenes(cuda):
    rays = random_rays(1000, seed=51)
    empty = gpu_scene(np.zeros((0, 3), np.float32), np.zeros((0, 3), np.uint32))
    assert (empty.intersect_host(rays)["tri_id"] == -1).all()
    pos = np.array([[-1, -1, 0], [1, -1, 0], [0, 1, 0]], np.float32)
    faces = np.array([[0, 1, 2]], np.uint32)
    o = oracle.OracleScene(pos, faces).intersect(rays)
    r = gpu_scene(pos, faces).intersect_host(rays)
    np.testing.assert_array_equal(r["tri_id"], o["tri_id"])


def test_large_scene_layouts_agree(cuda):
    """Benchmark-scale property check: 1,048,576-triangle soup, 2^22 rays:
    the binary and 4-wide layouts agree bit for bit, and a 20k-ray sample
    agrees with the oracle."""
    pos, faces = random_soup(1 << 20, seed=1)
    rays = random_rays(1 << 22, seed=2)
    a = gpu_scene(pos, faces, "bvh").intersect_host(rays)
    b = gpu_scene(pos, faces, "qbvh").intersect_host(rays)
    np.testing.assert_array_equal(a["tri_id"], b["tri_id"])
    np.testing.assert_array_equal(a["t"], b["t"])
    frac = (a["tri_id"] >= 0).mean()
    assert 0.15 < frac < 0.35
    sample = rays[:: (1 << 22) // 20000][:20000]
    o = oracle.OracleScene(pos, faces).intersect(sample)
    np.testing.assert_array_equal(a["tri_id"][:: (1 << 22) // 20000][:20000], o["tri_id"])


def test_host_pipeline_matches_device_path(cuda):
    """lmgpu_intersect_host overlaps copies and traversal of 1M-ray chunks on
    two streams; each launch must use its own work counter."""
    import torch
    pos, faces = random_soup(1 << 18, seed=61, sigma=0.02)
    rays = random_rays(5 * (1 << 20) + 12345, seed=62)
    s = gpu_scene(pos, faces, "bvh")
    for _ in range(3):
        a = s.intersect_host(rays)
        soa = {k: torch.from_numpy(v).to(cuda) for k, v in rays_soa(rays).items()}
        out = torch.empty(rays.shape[0], dtype=torch.int32, device=cuda)
        s.intersect_device({k: soa[k].data_ptr() for k in soa}, {"tri_id": out.data_ptr()}, rays.shape[0],
                           torch.cuda.current_stream().cuda_stream)
        s.status(torch.cuda.current_stream().cuda_stream)
        np.testing.assert_array_equal(a["tri_id"], out.cpu().numpy())


@pytest.mark.parametrize("pinned_in,pinned_out", [(True, False), (False, True), (True, True)])
def test_host_pipeline_pinned_and_pageable_buffers(cuda, pinned_in, pinned_out):
    """Page-locked caller buffers go straight to the copy engines; pageable
    ones through the pipeline's pinned staging (rays in, hits out, or both).
    Same hits either way."""
    import ctypes
    import torch
    from lightmetrica_b200 import native
    pos, faces = random_soup(1 << 16, seed=63, sigma=0.03)
    rays = random_rays(5 * (1 << 20) + 777, seed=64)
    n = rays.shape[0]
    s = gpu_scene(pos, faces, "bvh")
    want = s.intersect_host(rays)                  # pageable in and out
    rin = torch.from_numpy(rays).pin_memory() if pinned_in else torch.from_numpy(rays.copy())
    outs = [torch.empty(n, dtype=dt) for dt in (torch.int32, torch.float32, torch.float32, torch.float32)]
    if pinned_out:
        outs = [o.pin_memory() for o in outs]
    native.check(native.lib().lmgpu_intersect_host(s.handle, rin.data_ptr(), n, *[o.data_ptr() for o in outs]))
    np.testing.assert_array_equal(outs[0].numpy(), want["tri_id"])
    for o, k in zip(outs[1:], ("t", "u", "v")):
        np.testing.assert_array_equal(o.numpy(), want[k])



@pytest.mark.skipif(not oracle.ref_available("f"), reason="reference harness (oracle/_ref) not built")
def test_full_benchmark_batch_bit_exact_vs_reference(cuda):
    """All 2^24 rays of the intersection benchmark against the reference's
    own BVHScene (oracle/_ref, its float build, on all host threads): ids
    bit-exact and hit distances bit-equal, for the binary layout and its
    4-wide collapse."""
    pos, faces = random_soup(1 << 20, seed=1)
    rays = random_rays(1 << 24, seed=2)
    want = oracle.RefScene(pos, faces, "bvh").intersect(rays, threads=os.cpu_count() or 1)
    hit = want["tri_id"] >= 0
    assert 0.15 < hit.mean() < 0.35
    for layout in LAYOUTS:
        got = gpu_scene(pos, faces, layout).intersect_host(rays)
        np.testing.assert_array_equal(got["tri_id"], want["tri_id"])
        np.testing.assert_array_equal(got["t"][hit], want["t"][hit])


def test_stack_bound_overflow_is_reported_and_recoverable(cuda):
    """A scene whose traversal stack bound (max_stack_entries) is below what
    its walks need: the kernels flag the overflow in the scene's status word
    and return (no trap), the call reports LMGPU_ERR_STACK_OVERFLOW, and the
    status is cleared: the next call on the same scene succeeds when its rays
    need no stack, and the same rays succeed on a scene with the automatic
    bound."""
    import torch
    pos, faces = random_soup(50000, seed=71, sigma=0.05)
    rays = random_rays(20000, seed=72)
    for layout in LAYOUTS:
        s = Scene(layout)
        s.load(soup_primitives(pos, faces))
        s.configure({"max_stack_entries": 2})
        s.build()
        with pytest.raises(native.LmgpuError) as e:
            s.intersect_host(rays)
        assert e.value.code == native.ERR_STACK_OVERFLOW
        # Device entry point: the status word carries it to lmgpu_scene_status.
        soa = {k: torch.from_numpy(v).to(cuda) for k, v in rays_soa(rays).items()}
        out = torch.empty(rays.shape[0], dtype=torch.int32, device=cuda)
        stream = torch.cuda.current_stream().cuda_stream
        s.intersect_device({k: soa[k].data_ptr() for k in soa}, {"tri_id": out.data_ptr()}, rays.shape[0], stream)
        with pytest.raises(native.LmgpuError) as e:
            s.status(stream)
        assert e.value.code == native.ERR_STACK_OVERFLOW
        s.status(stream)                              # cleared
        # Rays that miss the root box need no stack: the next call succeeds.
        away = rays.copy()
        away[:, 0:3] = 10.0
        away[:, 3:6] = np.array([1.0, 0.0, 0.0], np.float32)
        r = s.intersect_host(away)
        assert (r["tri_id"] == -1).all()
        ok = gpu_scene(pos, faces, layout).intersect_host(rays)
        o = oracle.OracleScene(pos, faces, "bvh").intersect(rays)
        np.testing.assert_array_equal(ok["tri_id"], o["tri_id"])
        s.close()


def test_stack_bound_overflow_in_a_render(cuda):
    """The same bound in the path tracer: the render's traversal kernels flag
    the overflow and lmgpu_render reports LMGPU_ERR_STACK_OVERFLOW; a render
    of the scene with the automatic bound then succeeds."""
    from lightmetrica_b200 import create_renderer, create_scheduler, scenes
    prims = scenes.cornell_refined(3, 32, 32)
    r = create_renderer("pt.mis")
    r.configure({"rr_depth": 3, "max_path_vertices": 6, "sampler": {"rng_seed": 1}})
    sched = create_scheduler("mt")
    sched.configure({"num_samples": 32 * 32 * 4})
    capped = Scene("bvh")
    capped.load(prims)
    capped.configure({"max_stack_entries": 1})
    capped.build()
    with pytest.raises(native.LmgpuError) as e:
        sched.render(r, capped)
    assert e.value.code == native.ERR_STACK_OVERFLOW
    capped.close()
    s = Scene("bvh")
    s.load(prims)
    s.configure({})
    s.build()
    assert sched.render(r, s).max() > 0
    s.close()
