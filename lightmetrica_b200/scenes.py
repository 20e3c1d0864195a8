"""Procedural scenes of the benchmark configurations, built as lightmetrica
Primitives (seeded; the reference ships no scene files for them).

* ``cornell_box``: unit cube [0,1]^3 with the front face (z = 1) open
  (5 quads = 10 triangles), two inner boxes of 12 triangles each, a
  2-triangle ceiling light of emission (17, 12, 4); Lambertian red / green /
  white walls; pinhole camera with 40 degree vertical field of view.
* ``cornell_refined``: the same box with every triangle split 4:1 at its edge
  midpoints `levels` times (36 * 4^levels triangles).
* ``terrain_spheres``: a fBm heightfield of n x n vertices, icospheres
  subdivided `ico_level` times, Lambertian / diffuse-mirror materials, one
  spherical area light and a constant environment.

Every mesh carries per-vertex normals whose orientation agrees with its
triangle winding (the reference BSDFs are one-sided w.r.t. the shading
normal and the light emits on the front side only).
"""
from __future__ import annotations

import numpy as np

from .scene import (AreaLight, ConstantEnvironmentLight, DiffuseBSDF, DiffuseMirrorBSDF, HDRBitmapFilm,
                    PerfectMirrorBSDF, PerspectiveCamera, Primitive, Primitives, TriangleMesh)

RED = (0.63, 0.065, 0.05)
GREEN = (0.14, 0.45, 0.09)
WHITE = (0.73, 0.73, 0.73)
LIGHT_LE = (17.0, 12.0, 4.0)


def _quad(a, b, c, d, normal):
    """Two triangles (a, b, c), (a, c, d) wound so that their geometric
    normal agrees with `normal`."""
    p = np.array([a, b, c, d], np.float64)
    n = np.asarray(normal, np.float64)
    g = np.cross(p[1] - p[0], p[2] - p[0])
    if np.dot(g, n) < 0:
        p = p[[0, 3, 2, 1]]
    return p.astype(np.float32), np.tile(n / np.linalg.norm(n), (4, 1)).astype(np.float32), \
        np.array([[0, 1, 2], [0, 2, 3]], np.uint32)


def _mesh(quads):
    P, N, F = [], [], []
    base = 0
    for p, n, f in quads:
        P.append(p)
        N.append(n)
        F.append(f + base)
        base += p.shape[0]
    return TriangleMesh(np.concatenate(P), np.concatenate(F), np.concatenate(N))


def _box(center, size, angle_deg):
    """Axis-aligned box rotated about y; 6 faces, outward normals."""
    cx, cy, cz = center
    sx, sy, sz = size
    th = np.radians(angle_deg)
    R = np.array([[np.cos(th), 0, np.sin(th)], [0, 1, 0], [-np.sin(th), 0, np.cos(th)]])

    def P(x, y, z):
        v = R @ np.array([x * sx / 2, y * sy / 2, z * sz / 2])
        return v + np.array([cx, cy + sy / 2, cz])

    faces = []
    for axis in range(3):
        for s in (-1, 1):
            corners = []
            for u, v in ((-1, -1), (1, -1), (1, 1), (-1, 1)):
                c = [0, 0, 0]
                c[axis] = s
                c[(axis + 1) % 3] = u
                c[(axis + 2) % 3] = v
                corners.append(P(*c))
            n = np.zeros(3)
            n[axis] = s
            faces.append(_quad(*corners, R @ n))
    return _mesh(faces)


def cornell_box(width: int = 256, height: int = 256, fovy: float = 40.0, variant: str = "classic") -> Primitives:
    """variant "classic": all Lambertian. variant "mixed": the tall box is a
    perfect mirror, the short box diffuse-mirror, and a constant environment
    of 0.5 shines in through the open front face."""
    white, red, green = DiffuseBSDF(WHITE), DiffuseBSDF(RED), DiffuseBSDF(GREEN)
    prims = Primitives()
    # Walls (normals into the box): floor, ceiling, back, left (red), right (green).
    prims.add(Primitive(mesh=_mesh([_quad((0, 0, 0), (1, 0, 0), (1, 0, 1), (0, 0, 1), (0, 1, 0)),
                                    _quad((0, 1, 0), (1, 1, 0), (1, 1, 1), (0, 1, 1), (0, -1, 0)),
                                    _quad((0, 0, 0), (1, 0, 0), (1, 1, 0), (0, 1, 0), (0, 0, 1))]), bsdf=white))
    prims.add(Primitive(mesh=_mesh([_quad((0, 0, 0), (0, 1, 0), (0, 1, 1), (0, 0, 1), (1, 0, 0))]), bsdf=red))
    prims.add(Primitive(mesh=_mesh([_quad((1, 0, 0), (1, 1, 0), (1, 1, 1), (1, 0, 1), (-1, 0, 0))]), bsdf=green))
    # Short and tall inner boxes.
    short_bsdf, tall_bsdf = white, white
    if variant == "mixed":
        short_bsdf = DiffuseMirrorBSDF((0.8, 0.75, 0.6))
        tall_bsdf = PerfectMirrorBSDF((0.9, 0.9, 0.9))
        prims.environment_light = ConstantEnvironmentLight((0.5, 0.5, 0.5))
    prims.add(Primitive(mesh=_box((0.33, 0.0, 0.62), (0.30, 0.30, 0.30), -17.0), bsdf=short_bsdf))
    prims.add(Primitive(mesh=_box((0.68, 0.0, 0.35), (0.30, 0.60, 0.30), 17.0), bsdf=tall_bsdf))
    # Ceiling light, just below the ceiling, emitting downwards.
    y = 1.0 - 1e-3
    prims.add(Primitive(mesh=_mesh([_quad((0.37, y, 0.40), (0.63, y, 0.40), (0.63, y, 0.60), (0.37, y, 0.60),
                                          (0, -1, 0))]),
                        bsdf=DiffuseBSDF((0.0, 0.0, 0.0)), light=AreaLight(LIGHT_LE)))
    prims.camera = PerspectiveCamera(fovy=fovy, eye=(0.5, 0.5, 2.44), center=(0.5, 0.5, 0.0), up=(0, 1, 0),
                                     film=HDRBitmapFilm(width, height))
    return prims


def subdivide(mesh: TriangleMesh, levels: int) -> TriangleMesh:
    """4:1 midpoint subdivision of every triangle (vertices per triangle,
    normals interpolated and renormalised)."""
    P = mesh.positions[mesh.faces].astype(np.float64)      # (T, 3, 3)
    Nn = mesh.normals[mesh.faces].astype(np.float64)
    for _ in range(levels):
        a, b, c = P[:, 0], P[:, 1], P[:, 2]
        ab, bc, ca = (a + b) / 2, (b + c) / 2, (c + a) / 2
        na, nb, nc = Nn[:, 0], Nn[:, 1], Nn[:, 2]
        nab, nbc, nca = (na + nb) / 2, (nb + nc) / 2, (nc + na) / 2
        P = np.concatenate([np.stack([a, ab, ca], 1), np.stack([ab, b, bc], 1),
                            np.stack([ca, bc, c], 1), np.stack([ab, bc, ca], 1)])
        Nn = np.concatenate([np.stack([na, nab, nca], 1), np.stack([nab, nb, nbc], 1),
                             np.stack([nca, nbc, nc], 1), np.stack([nab, nbc, nca], 1)])
        Nn /= np.linalg.norm(Nn, axis=2, keepdims=True)
    T = P.shape[0]
    return TriangleMesh(P.reshape(-1, 3).astype(np.float32), np.arange(3 * T, dtype=np.uint32).reshape(-1, 3),
                        Nn.reshape(-1, 3).astype(np.float32))


def cornell_refined(levels: int = 5, width: int = 512, height: int = 512) -> Primitives:
    base = cornell_box(width, height)
    for p in base.primitives:
        p.mesh = subdivide(p.mesh, levels)
    return base


# ---------------------------------------------------------------- terrain --

def heightfield(n: int = 1024, extent: float = 4.0, amplitude: float = 0.1, octaves: int = 4, seed: int = 7):
    """fBm heightfield of n x n vertices over [-extent, extent]^2 (xz),
    2 (n - 1)^2 triangles, normals from central differences."""
    rng = np.random.default_rng(seed)
    table = rng.random(1024).astype(np.float64)
    perm = rng.permutation(1024).astype(np.float64)
    lin = np.linspace(-extent, extent, n)
    X, Z = np.meshgrid(lin, lin, indexing="xy")
    H = np.zeros_like(X)
    freq, amp = 1.0, 1.0
    for _ in range(octaves):
        xi = X * freq
        zi = Z * freq
        ix, iz = np.floor(xi).astype(np.int64), np.floor(zi).astype(np.int64)
        fx, fz = xi - ix, zi - iz
        ux, uz = fx * fx * (3 - 2 * fx), fz * fz * (3 - 2 * fz)

        def h(i, j):
            return table[(perm[(j % 1024)].astype(np.int64) + i) % 1024]
        n00, n10, n01, n11 = h(ix, iz), h(ix + 1, iz), h(ix, iz + 1), h(ix + 1, iz + 1)
        H += amp * ((n00 * (1 - ux) + n10 * ux) * (1 - uz) + (n01 * (1 - ux) + n11 * ux) * uz - 0.5)
        freq *= 2.0
        amp *= 0.5
    H *= amplitude / 0.5
    P = np.stack([X, H, Z], -1).reshape(-1, 3)
    dx = np.gradient(H, lin, axis=1)
    dz = np.gradient(H, lin, axis=0)
    Nn = np.stack([-dx, np.ones_like(H), -dz], -1).reshape(-1, 3)
    Nn /= np.linalg.norm(Nn, axis=1, keepdims=True)
    i = np.arange(n - 1)
    I, J = np.meshgrid(i, i, indexing="xy")
    v00 = (J * n + I).reshape(-1)
    v10, v01, v11 = v00 + 1, v00 + n, v00 + n + 1
    F = np.concatenate([np.stack([v00, v01, v11], 1), np.stack([v00, v11, v10], 1)]).astype(np.uint32)
    return TriangleMesh(P.astype(np.float32), F, Nn.astype(np.float32))


def icosphere(level: int):
    """Unit icosphere: 20 * 4^level triangles, shared vertices, outward normals."""
    t = (1.0 + 5 ** 0.5) / 2.0
    V = [(-1, t, 0), (1, t, 0), (-1, -t, 0), (1, -t, 0), (0, -1, t), (0, 1, t), (0, -1, -t), (0, 1, -t),
         (t, 0, -1), (t, 0, 1), (-t, 0, -1), (-t, 0, 1)]
    F = [(0, 11, 5), (0, 5, 1), (0, 1, 7), (0, 7, 10), (0, 10, 11), (1, 5, 9), (5, 11, 4), (11, 10, 2),
         (10, 7, 6), (7, 1, 8), (3, 9, 4), (3, 4, 2), (3, 2, 6), (3, 6, 8), (3, 8, 9), (4, 9, 5), (2, 4, 11),
         (6, 2, 10), (8, 6, 7), (9, 8, 1)]
    V = np.array(V, np.float64)
    V /= np.linalg.norm(V, axis=1, keepdims=True)
    F = np.array(F, np.int64)
    for _ in range(level):
        edges = np.concatenate([F[:, [0, 1]], F[:, [1, 2]], F[:, [2, 0]]])
        key = np.sort(edges, axis=1)
        uniq, inv = np.unique(key, axis=0, return_inverse=True)
        mid = (V[uniq[:, 0]] + V[uniq[:, 1]]) / 2
        mid /= np.linalg.norm(mid, axis=1, keepdims=True)
        m = inv.reshape(3, -1).T + V.shape[0]
        V = np.concatenate([V, mid])
        a, b, c = F[:, 0], F[:, 1], F[:, 2]
        ab, bc, ca = m[:, 0], m[:, 1], m[:, 2]
        F = np.concatenate([np.stack([a, ab, ca], 1), np.stack([b, bc, ab], 1), np.stack([c, ca, bc], 1),
                            np.stack([ab, bc, ca], 1)])
    # Orient every face outwards.
    g = np.cross(V[F[:, 1]] - V[F[:, 0]], V[F[:, 2]] - V[F[:, 0]])
    flip = np.einsum("ij,ij->i", g, V[F[:, 0]]) < 0
    F[flip] = F[flip][:, [0, 2, 1]]
    return V.astype(np.float32), F.astype(np.uint32)


def terrain_spheres(width: int = 1920, height: int = 1080, grid: int = 1024, spheres: int = 64, ico_level: int = 5,
                    env: float = 0.5, seed: int = 3) -> Primitives:
    rng = np.random.default_rng(seed)
    prims = Primitives()
    prims.add(Primitive(mesh=heightfield(grid, seed=seed + 4), bsdf=DiffuseBSDF((0.5, 0.5, 0.5))))
    V, F = icosphere(ico_level)
    for k in range(spheres):
        r = rng.uniform(0.15, 0.45)
        c = np.array([rng.uniform(-3.2, 3.2), 0.0, rng.uniform(-3.2, 3.2)])
        c[1] = r + rng.uniform(0.05, 0.6)
        albedo = tuple(rng.uniform(0.2, 0.8, 3))
        bsdf = DiffuseBSDF(albedo) if k % 2 == 0 else DiffuseMirrorBSDF(albedo)
        prims.add(Primitive(mesh=TriangleMesh((V * r + c).astype(np.float32), F, V.copy()), bsdf=bsdf))
    # Spherical area light (icosphere level 2), emitting outwards.
    LV, LF = icosphere(2)
    lc = np.array([0.0, 3.0, 0.0])
    prims.add(Primitive(mesh=TriangleMesh((LV * 0.5 + lc).astype(np.float32), LF, LV.copy()),
                        bsdf=DiffuseBSDF((0.0, 0.0, 0.0)), light=AreaLight((40.0, 36.0, 30.0))))
    prims.environment_light = ConstantEnvironmentLight((env, env, env))
    prims.camera = PerspectiveCamera(fovy=45.0, eye=(0.0, 2.6, 6.2), center=(0.0, 0.2, 0.0), up=(0, 1, 0),
                                     film=HDRBitmapFilm(width, height))
    return prims


def num_triangles(prims: Primitives) -> int:
    return int(sum(p.mesh.faces.shape[0] for p in prims.primitives if p.mesh is not None))


# ----------------------------------------------------------- batch set ----

BATCH_RESOLUTIONS = (128, 256, 512, 1024)


def batch_scene(index: int, seed: int = 5) -> dict:
    """Scene `index` of the seeded multi-scene set: a random-triangle soup or
    a fBm heightfield with a log-uniform triangle count in [1k, 200k], a
    square film from {128, 256, 512, 1024}, 4-64 spp, max depth 8-16, half
    its triangles Lambertian and half perfect mirror, a 2-triangle area light
    and a constant environment of 0.3. Returns {"prims", "spp",
    "max_path_vertices", "kind", "triangles"}."""
    rng = np.random.default_rng([seed, index])
    tris = int(round(np.exp(rng.uniform(np.log(1e3), np.log(2e5)))))
    res = int(rng.choice(BATCH_RESOLUTIONS))
    spp = int(rng.choice((4, 8, 16, 32, 64)))
    depth = int(rng.integers(8, 17))
    kind = "soup" if index % 2 == 0 else "heightfield"
    albedo = tuple(rng.uniform(0.2, 0.8, 3))
    prims = Primitives()
    if kind == "soup":
        # Triangle size grows as the count falls, so that coverage stays comparable.
        sigma = 0.01 * np.sqrt(float(1 << 20) / tris)
        c = rng.uniform(-1.0, 1.0, size=(tris, 3))
        e1 = rng.normal(0.0, sigma, size=(tris, 3))
        e2 = rng.normal(0.0, sigma, size=(tris, 3))
        v0 = c - (e1 + e2) / 3.0
        P = np.stack([v0, v0 + e1, v0 + e2], axis=1).astype(np.float32)
        half = tris // 2
        for part, bsdf in ((P[:half], DiffuseBSDF(albedo)), (P[half:], PerfectMirrorBSDF((0.9, 0.9, 0.9)))):
            k = part.shape[0]
            if k == 0:
                continue
            prims.add(Primitive(mesh=TriangleMesh(part.reshape(-1, 3), np.arange(3 * k, dtype=np.uint32).reshape(-1, 3)),
                                bsdf=bsdf))
        light_y, light_half, eye, center = 1.6, 0.5, (0.0, 0.6, 3.4), (0.0, 0.0, 0.0)
    else:
        n = max(2, int(round(np.sqrt(tris / 2.0))) + 1)
        hf = heightfield(n, extent=2.0, amplitude=0.25, seed=int(rng.integers(1 << 30)))
        F = hf.faces
        half = F.shape[0] // 2
        prims.add(Primitive(mesh=TriangleMesh(hf.positions, F[:half], hf.normals), bsdf=DiffuseBSDF(albedo)))
        prims.add(Primitive(mesh=TriangleMesh(hf.positions, F[half:], hf.normals), bsdf=PerfectMirrorBSDF((0.9, 0.9, 0.9))))
        light_y, light_half, eye, center = 1.5, 0.6, (0.0, 1.6, 3.2), (0.0, 0.0, 0.0)
    lp, ln, lf = _quad((-light_half, light_y, -light_half), (light_half, light_y, -light_half),
                       (light_half, light_y, light_half), (-light_half, light_y, light_half), (0, -1, 0))
    prims.add(Primitive(mesh=TriangleMesh(lp, lf, ln), bsdf=DiffuseBSDF((0.0, 0.0, 0.0)), light=AreaLight((12.0, 12.0, 12.0))))
    prims.environment_light = ConstantEnvironmentLight((0.3, 0.3, 0.3))
    prims.camera = PerspectiveCamera(fovy=45.0, eye=eye, center=center, up=(0, 1, 0), film=HDRBitmapFilm(res, res))
    return {"prims": prims, "spp": spp, "max_path_vertices": depth + 1, "kind": kind, "triangles": num_triangles(prims)}
