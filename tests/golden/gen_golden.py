"""Generates the golden fixtures in this directory from the reference's own
code (oracle/_ref, built from the reference sources by oracle/build_ref.sh).

Run from the repository root, with LM_REFERENCE_ROOT naming the reference
source tree (oracle/_ref is built from it first):
    LM_REFERENCE_ROOT=<lightmetrica checkout> python tests/golden/gen_golden.py

Fixtures:
  intersect_simple.npz     reference test Intersect_Simple
                           (src/lightmetrica.test/test.scene.intersection.cpp:117-151)
  intersect_simple2.npz    reference test Intersect_Simple2 (:153-187)
  consistency_random.npz   reference test Consistency (:190-266) on
                           StubTriangleMesh_Random (stub.trianglemesh.h:184-225)
  soup_small.npz           seeded triangle soup with the ray-intersection
                           benchmark's distributions (4096 tris, edge sigma
                           0.16, 8192 rays);
                           reference BVHScene tri ids, t and (u, v)
  soup_duplicates.npz      1024 triangles, each repeated three times (exact
                           ties), 4096 rays; reference bvh and naive ids and t
  cornell_{classic,mixed}_ref_mis.npz
                           the reference's double-precision pt.mis image of
                           lightmetrica_b200.scenes.cornell_box(128, 128,
                           variant) (4096 / 16384 spp)
  cornell_c1_256_ref_mis.npz
                           the reference's double-precision pt.mis image of
                           scenes.cornell_box(256, 256) at max depth 8 (4096 spp)
  terrain_ref_mis_96x54.npz
                           the reference's double-precision pt.mis image of
                           scenes.terrain_spheres at 96 x 54 (16384 spp)
  ref_scene_literals.json  the XML scene literals of the reference's Primitives
                           and BPT tests (inputs of tests/test_sceneio.py)
Each fixture stores the inputs with the reference outputs for every scene
type the reference builds here (bvh, qbvh, naive).
"""
from __future__ import annotations

import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

import oracle  # noqa: E402
from lightmetrica_b200.workloads import random_rays, random_soup, FLT_MAX  # noqa: E402

OUT = os.path.dirname(os.path.abspath(__file__))
TYPES = ("bvh", "qbvh", "naive")


def _grid_rays(origin_fn, dir_fn):
    rays = []
    for i in range(1, 10):
        y = np.float32(0.1) * np.float32(i)
        for j in range(1, 10):
            x = np.float32(0.1) * np.float32(j)
            o = origin_fn(x, y)
            d = dir_fn(x, y, o)
            rays.append([*o, *d, 0.0, FLT_MAX])
    return np.asarray(rays, np.float32)


def _run_all(name, pos, faces, normals, texcoords, rays, extra=None):
    out = dict(positions=pos, faces=faces, rays=rays)
    if normals is not None:
        out["normals"] = normals
    if texcoords is not None:
        out["texcoords"] = texcoords
    for typ in TYPES:
        s = oracle.RefScene(pos, faces, typ, normals=normals, texcoords=texcoords)
        r = s.intersect(rays, geom=True)
        for k in ("tri_id", "t", "p", "gn", "sn", "ss", "st", "uv"):
            out[f"{typ}_{k}"] = r[k]
    if extra:
        out.update(extra)
    np.savez_compressed(os.path.join(OUT, name), **out)
    print("wrote", name, {k: v.shape for k, v in out.items()})


def main():
    if not oracle.ref_available("f"):
        raise SystemExit("oracle/_ref/liblmref_f.so missing: run oracle/build_ref.sh first")

    # Intersect_Simple: two z-planes, rays from (0,0,1) towards (x,y,0)
    ps = np.array([0, 0, 0, 1, 0, 0, 1, 1, 0, 0, 1, 0, 0, 0, -1, 1, 0, -1, 1, 1, -1, 0, 1, -1], np.float32).reshape(-1, 3)
    ns = np.tile(np.array([0, 0, 1], np.float32), (8, 1))
    ts = np.array([0, 0, 1, 0, 1, 1, 0, 1] * 2, np.float32).reshape(-1, 2)
    fs = np.array([0, 1, 2, 0, 2, 3, 4, 5, 6, 4, 6, 7], np.uint32).reshape(-1, 3)

    def d_simple(x, y, o):
        d = np.array([x, y, 0], np.float64) - np.asarray(o, np.float64)
        return (d / np.linalg.norm(d)).astype(np.float32)
    rays = _grid_rays(lambda x, y: np.array([0, 0, 1], np.float32), d_simple)
    _run_all("intersect_simple.npz", ps, fs, ns, ts, rays)

    # Intersect_Simple2: slanted plane x = -z, vertical rays
    ps2 = np.array([0, 0, 0, 1, 0, -1, 1, 1, -1, 0, 1, 0], np.float32).reshape(-1, 3)
    n2 = (np.array([1, 0, 1], np.float64) / np.sqrt(2.0)).astype(np.float32)
    ns2 = np.tile(n2, (4, 1))
    ts2 = np.array([0, 0, 1, 0, 1, 1, 0, 1], np.float32).reshape(-1, 2)
    fs2 = np.array([0, 1, 2, 0, 2, 3], np.uint32).reshape(-1, 3)
    rays2 = _grid_rays(lambda x, y: np.array([x, y, 1], np.float32), lambda x, y, o: np.array([0, 0, -1], np.float32))
    _run_all("intersect_simple2.npz", ps2, fs2, ns2, ts2, rays2)

    # Consistency: 1000 random triangles in [0,1]^3, vertical rays
    pr, nr = oracle.stub_random_mesh()
    fr = np.arange(3000, dtype=np.uint32).reshape(-1, 3)
    rays3 = _grid_rays(lambda x, y: np.array([x, y, 1], np.float32), lambda x, y, o: np.array([0, 0, -1], np.float32))
    _run_all("consistency_random.npz", pr, fr, nr, None, rays3)

    # Benchmark-distribution soup, small: ids, t and barycentrics (uv = b
    # because the harness assigns corner texcoords (0,0),(1,0),(0,1)). Edge
    # sigma is scaled by sqrt(1M / 4096) = 16 so that the hit rate matches the
    # 1M-triangle benchmark scene's (about a quarter of the rays).
    pos, faces = random_soup(4096, seed=11, sigma=0.16)
    rays4 = random_rays(8192, seed=12)
    s = oracle.RefScene(pos, faces, "bvh")
    r = s.intersect(rays4, geom=True)
    np.savez_compressed(os.path.join(OUT, "soup_small.npz"), positions=pos, faces=faces, rays=rays4,
                        bvh_tri_id=r["tri_id"], bvh_t=r["t"], bvh_u=r["uv"][:, 0], bvh_v=r["uv"][:, 1])
    print("wrote soup_small.npz hits", int((r["tri_id"] >= 0).sum()))

    # Exact ties: every triangle appears three times. The reference keeps the
    # last of equal-t hits in leaf order (t <= maxT is accepted,
    # scene.bvh.cpp:416-427), so the returned id pins the partition order
    # (std::partition, scene.bvh.cpp:375) and the naive scan order.
    base, _ = random_soup(1024, seed=13, sigma=0.16)
    tri = base.reshape(-1, 3, 3)
    dup = np.repeat(tri, 3, axis=0).reshape(-1, 3).astype(np.float32)
    fd = np.arange(dup.shape[0], dtype=np.uint32).reshape(-1, 3)
    rays5 = random_rays(4096, seed=14)
    out = dict(positions=dup, faces=fd, rays=rays5)
    for typ in ("bvh", "naive"):
        s = oracle.RefScene(dup, fd, typ)
        r = s.intersect(rays5, geom=True)
        out[f"{typ}_tri_id"] = r["tri_id"]
        out[f"{typ}_t"] = r["t"]
    np.savez_compressed(os.path.join(OUT, "soup_duplicates.npz"), **out)
    print("wrote soup_duplicates.npz hits", int((out["bvh_tri_id"] >= 0).sum()))


IMAGE_SPP = {"classic": 4096, "mixed": 16384}


def images(variants=("classic", "mixed")):
    """Image oracles: the reference's own pt.mis in double precision
    (oracle/_ref/liblmref_d.so), 128 x 128, max_path_vertices 9 (max depth
    8), rr_depth 3, rng standardmt seed 1, uniform raster sampling with the
    `mt` scheduler, at IMAGE_SPP samples per pixel on average (the mixed
    scene's mirror caustics carry ~4x the per-sample variance, so it gets 4x
    the samples)."""
    from lightmetrica_b200 import scenes
    for variant in variants:
        spp = IMAGE_SPP[variant]
        prims = scenes.cornell_box(128, 128, variant=variant)
        film, secs = oracle.ref_render(prims, "pt.mis", spp=spp, rr_depth=3, max_path_vertices=9, seed=1)
        np.savez_compressed(os.path.join(OUT, f"cornell_{variant}_ref_mis.npz"), film=film,
                            spp=spp, rr_depth=3, max_path_vertices=9, seconds=secs)
        print("wrote", variant, "image", f"{spp} spp {secs:.1f} s", film.mean(axis=(0, 1)))


def c1_image(spp: int = 4096):
    """Image oracle of the plain path-tracer configuration: the Cornell box
    (scenes.cornell_box "classic": 10 wall, 24 box and 2 light triangles,
    Le (17, 12, 4)) at exactly 256 x 256, 40 degree field of view, max depth
    8 (max_path_vertices 9), Russian roulette from vertex 3 (rr_depth 3),
    seed 1: the reference's double-precision pt.mis at 4096 spp."""
    from lightmetrica_b200 import scenes
    prims = scenes.cornell_box(256, 256, variant="classic")
    film, secs = oracle.ref_render(prims, "pt.mis", spp=spp, rr_depth=3, max_path_vertices=9, seed=1)
    np.savez_compressed(os.path.join(OUT, "cornell_c1_256_ref_mis.npz"), film=film, spp=spp, rr_depth=3,
                        max_path_vertices=9, seconds=secs)
    print("wrote C1 image", f"{spp} spp {secs:.1f} s", film.mean(axis=(0, 1)))


def terrain_image(spp: int = 16384):
    """Image oracle of the full path-tracer scene (scenes.terrain_spheres: a
    1024 x 1024-vertex fBm heightfield, 64 level-5 icospheres, a spherical
    area light, a constant environment; 3.4M triangles), scaled down to
    96 x 54 pixels with the same camera: the reference's double-precision
    pt.mis, max_path_vertices 17 (max depth 16), rr_depth 5 (Russian roulette
    after depth 4), at 16384 spp (two independent 4096-spp renders of it
    differ by relMSE 8.2e-4, so 16384 spp leaves ~1e-4 of noise)."""
    from lightmetrica_b200 import scenes
    prims = scenes.terrain_spheres(96, 54)
    film, secs = oracle.ref_render(prims, "pt.mis", spp=spp, rr_depth=5, max_path_vertices=17, seed=1)
    np.savez_compressed(os.path.join(OUT, "terrain_ref_mis_96x54.npz"), film=film, spp=spp, rr_depth=5,
                        max_path_vertices=17, seconds=secs)
    print("wrote terrain image", f"{spp} spp {secs:.1f} s", film.mean(axis=(0, 1)))


def scene_literals(reference_root: str | None = None):
    """The XML scene literals of the reference's own Primitives and BPT tests
    (test.primitives.cpp: SceneNode_Success, _WithTransformByMatrix,
    _WithTransform; test.bpt.mis.cpp: SceneFile), extracted verbatim as test
    inputs; the expected values live in tests/test_sceneio.py with the
    reference assertions they restate."""
    import json
    import re
    reference_root = reference_root or oracle.reference_root(required=True)
    out = {}
    for fname, names in (("test.primitives.cpp", ("SceneNode_Success", "SceneNode_Success_WithTransformByMatrix",
                                                   "SceneNode_Success_WithTransform")),
                         ("test.bpt.mis.cpp", ("SceneFile",))):
        src = open(os.path.join(reference_root, "src", "lightmetrica.test", fname)).read()
        for name in names:
            m = re.search(r"const std::string " + name + r" = LM_TEST_MULTILINE_LITERAL\((.*?)\n\t\);", src, re.S)
            if not m:
                raise RuntimeError(f"literal {name} not found in {fname}")
            out[f"{fname}:{name}"] = m.group(1).strip()
    with open(os.path.join(OUT, "ref_scene_literals.json"), "w") as f:
        json.dump(out, f, indent=1)
    print("wrote", len(out), "scene literals")


if __name__ == "__main__":
    main()
    scene_literals()
    if oracle.ref_available("d"):
        images()
        c1_image()
        terrain_image()
