"""ORACLE — test infrastructure, not product code.

ctypes bindings for
  * ``liblmoracle.so`` — the plain-C restatement of lightmetrica's scene
    accelerator and path tracer (lmoracle.c, lmoracle_pt.c), and
  * ``_ref/liblmref_{f,d}.so`` — the reference's own hot-path sources compiled
    unmodified with this directory's stand-ins (build_ref.sh).

Only ``tests/``, ``__graft_entry__.smoke()`` and ``bench.py``'s CPU-baseline
legs may import this package, and only as the checker or the timed CPU
baseline. The product package ``lightmetrica_b200`` never imports it.
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
_ORACLE_SO = os.path.join(HERE, "liblmoracle.so")
_REF_SO = {"f": os.path.join(HERE, "_ref", "liblmref_f.so"),
           "d": os.path.join(HERE, "_ref", "liblmref_d.so")}

_P = ctypes.c_void_p
_I = ctypes.c_int
_LL = ctypes.c_longlong


def build(reference_root: str = "/root/reference") -> None:
    """Compile the C restatement and, when the reference tree is present, the
    reference harness (oracle/_ref). Building the checker is not using it."""
    subprocess.run(["bash", os.path.join(HERE, "build_oracle.sh")], check=True)
    if os.path.isdir(os.path.join(reference_root, "src", "liblightmetrica")):
        subprocess.run(["bash", os.path.join(HERE, "build_ref.sh"), reference_root], check=True)


def _ptr(a):
    return None if a is None else a.ctypes.data


_lib = None


def lib():
    """The C restatement (liblmoracle.so)."""
    global _lib
    if _lib is None:
        if not os.path.exists(_ORACLE_SO):
            subprocess.run(["bash", os.path.join(HERE, "build_oracle.sh")], check=True)
        L = ctypes.CDLL(_ORACLE_SO)
        L.orc_scene_create.restype = _P
        L.orc_scene_create.argtypes = [_I, _P, _I, _P, _I]
        L.orc_scene_destroy.argtypes = [_P]
        L.orc_intersect.restype = _LL
        L.orc_intersect.argtypes = [_P, _LL, _P, _P, _P, _P, _P, _P, _P]
        L.orc_scene_stats.argtypes = [_P, ctypes.POINTER(_LL), ctypes.POINTER(_LL), ctypes.POINTER(ctypes.c_int32)]
        L.orc_scene_tri_order.restype = _P
        L.orc_scene_tri_order.argtypes = [_P]
        _bind_pt(L)
        _lib = L
    return _lib


def _bind_pt(L):
    """Path-tracer restatement entry points (lmoracle_pt.c), when present."""
    if hasattr(L, "orc_render"):
        L.orc_render.restype = _I
        L.orc_render.argtypes = [_P, _P, _P]


class OracleScene:
    """Reference-exact BVH (kind='bvh') or brute force (kind='naive') over
    world-space triangles; triangle i is TriAccel index i."""

    def __init__(self, positions, faces, kind: str = "bvh"):
        self.positions = np.ascontiguousarray(positions, np.float32).reshape(-1)
        self.faces = np.ascontiguousarray(faces, np.uint32).reshape(-1)
        k = {"bvh": 0, "naive": 1}[kind]
        self.h = lib().orc_scene_create(k, _ptr(self.positions), self.positions.size // 3,
                                        _ptr(self.faces), self.faces.size // 3)

    def __del__(self):
        if getattr(self, "h", None):
            lib().orc_scene_destroy(self.h)
            self.h = None

    def intersect(self, rays):
        """rays: (n, 8) float32 AoS (o, d, minT, maxT)."""
        rays = np.ascontiguousarray(rays, np.float32).reshape(-1, 8)
        n = rays.shape[0]
        out = {k: np.zeros(n, np.float32) for k in ("t", "u", "v")}
        out["tri_id"] = np.zeros(n, np.int32)
        out["node_tests"] = np.zeros(n, np.int32)
        out["tri_tests"] = np.zeros(n, np.int32)
        lib().orc_intersect(self.h, n, _ptr(rays), _ptr(out["tri_id"]), _ptr(out["t"]), _ptr(out["u"]),
                            _ptr(out["v"]), _ptr(out["node_tests"]), _ptr(out["tri_tests"]))
        return out

    def stats(self):
        nodes, leaves, depth = _LL(), _LL(), ctypes.c_int32()
        lib().orc_scene_stats(self.h, ctypes.byref(nodes), ctypes.byref(leaves), ctypes.byref(depth))
        return {"nodes": nodes.value, "leaves": leaves.value, "max_depth": depth.value}

    def tri_order(self):
        p = lib().orc_scene_tri_order(self.h)
        n = self.faces.size // 3
        return np.ctypeslib.as_array(ctypes.cast(p, ctypes.POINTER(ctypes.c_int32)), shape=(n,)).copy()


_refs = {}


def ref_available(precision: str = "f") -> bool:
    return os.path.exists(_REF_SO[precision])


def ref(precision: str = "f"):
    """The reference's own code (oracle/_ref), float ('f') or double ('d')."""
    if precision not in _refs:
        L = ctypes.CDLL(_REF_SO[precision])
        L.lmref_scene_create.restype = _P
        L.lmref_scene_create.argtypes = [ctypes.c_char_p, _P, _I, _P, _P, _P, _I, ctypes.POINTER(ctypes.c_double)]
        L.lmref_scene_destroy.argtypes = [_P]
        L.lmref_intersect.restype = _LL
        L.lmref_intersect.argtypes = [_P, _LL, _P, _P, _P, _P, _I]
        L.lmref_stub_random_mesh.argtypes = [_P, _P]
        _bind_ref_render(L)
        _refs[precision] = L
    return _refs[precision]


def _bind_ref_render(L):
    if hasattr(L, "lmref_render"):
        L.lmref_render.restype = ctypes.c_double
        L.lmref_render.argtypes = [_P, _P, _P]


class RefScene:
    """The reference's Scene component ('bvh', 'qbvh', 'naive') built through
    its own Build() over identity-transform primitives."""

    def __init__(self, positions, faces, kind: str = "bvh", normals=None, texcoords=None,
                 precision: str = "f"):
        self.L = ref(precision)
        self.positions = np.ascontiguousarray(positions, np.float32).reshape(-1)
        self.faces = np.ascontiguousarray(faces, np.uint32).reshape(-1)
        self.normals = None if normals is None else np.ascontiguousarray(normals, np.float32).reshape(-1)
        self.texcoords = None if texcoords is None else np.ascontiguousarray(texcoords, np.float32).reshape(-1)
        bt = ctypes.c_double()
        self.h = self.L.lmref_scene_create(kind.encode(), _ptr(self.positions), self.positions.size // 3,
                                           _ptr(self.normals), _ptr(self.texcoords), _ptr(self.faces),
                                           self.faces.size // 3, ctypes.byref(bt))
        if not self.h:
            raise RuntimeError(f"reference scene '{kind}' failed to build")
        self.build_seconds = bt.value

    def __del__(self):
        if getattr(self, "h", None):
            self.L.lmref_scene_destroy(self.h)
            self.h = None

    def intersect(self, rays, geom: bool = False, threads: int = 1):
        rays = np.ascontiguousarray(rays, np.float32).reshape(-1, 8)
        n = rays.shape[0]
        ids = np.zeros(n, np.int32)
        t = np.zeros(n, np.float32)
        g = np.zeros((n, 17), np.float32) if geom else None
        self.L.lmref_intersect(self.h, n, _ptr(rays), _ptr(ids), _ptr(t), _ptr(g), threads)
        out = {"tri_id": ids, "t": t}
        if geom:
            out.update(p=g[:, 0:3], gn=g[:, 3:6], sn=g[:, 6:9], ss=g[:, 9:12], st=g[:, 12:15], uv=g[:, 15:17])
        return out


def stub_random_mesh():
    """The reference test fixture StubTriangleMesh_Random (1000 triangles)."""
    p = np.zeros(9000, np.float32)
    n = np.zeros(9000, np.float32)
    ref("f").lmref_stub_random_mesh(_ptr(p), _ptr(n))
    return p.reshape(-1, 3), n.reshape(-1, 3)
