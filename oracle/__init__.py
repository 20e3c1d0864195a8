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


def reference_root(required: bool = False):
    """The lightmetrica source tree named by the environment variable
    LM_REFERENCE_ROOT (a checkout of hi2p-perim/lightmetrica), or None when it
    is unset. With `required`, an unset or wrong variable raises."""
    root = os.environ.get("LM_REFERENCE_ROOT")
    ok = bool(root) and os.path.isdir(os.path.join(root, "src", "liblightmetrica"))
    if required and not ok:
        raise RuntimeError("set LM_REFERENCE_ROOT to a lightmetrica source tree (it holds src/liblightmetrica); "
                           f"got {root!r}")
    return root if ok else None


def build(reference_root_dir: str | None = None) -> None:
    """Compile the C restatement and, when a reference tree is given (the
    argument, or LM_REFERENCE_ROOT), the reference harness (oracle/_ref) and
    the product's lightmetrica plugin built against the reference headers
    (oracle/_ref/plugin.gpu.so). Without one, oracle/_ref keeps what an
    earlier build left there. Building the checker is not using it."""
    subprocess.run(["bash", os.path.join(HERE, "build_oracle.sh")], check=True)
    root = reference_root_dir or reference_root()
    if root and os.path.isdir(os.path.join(root, "src", "liblightmetrica")):
        subprocess.run(["bash", os.path.join(HERE, "build_ref.sh"), root], check=True)
        subprocess.run(["bash", os.path.join(HERE, "build_plugin.sh"), root], check=True)
    else:
        print("oracle: LM_REFERENCE_ROOT is unset (or holds no src/liblightmetrica); "
              "oracle/_ref not rebuilt", flush=True)


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


PLUGIN_SO = os.path.join(HERE, "_ref", "plugin.gpu.so")
_plugins_loaded = set()


def plugin_available() -> bool:
    return os.path.exists(PLUGIN_SO) and ref_available("f")


def load_plugin(path: str = PLUGIN_SO) -> None:
    """Loads a lightmetrica plugin into the float reference build the way the
    reference does (dlopen, then its exported LM_Plugin_CreateInstance): its
    components become available to RefScene and ref_render by name."""
    if path in _plugins_loaded:
        return
    L = ref("f")
    L.lmref_load_plugin.restype = ctypes.c_int
    L.lmref_load_plugin.argtypes = [ctypes.c_char_p, ctypes.POINTER(ctypes.c_char_p)]
    err = ctypes.c_char_p()
    if L.lmref_load_plugin(path.encode(), ctypes.byref(err)) != 0:
        raise RuntimeError(f"plugin {path} failed to load: {err.value.decode() if err.value else ''}")
    _plugins_loaded.add(path)


def stub_random_mesh():
    """The reference test fixture StubTriangleMesh_Random (1000 triangles)."""
    p = np.zeros(9000, np.float32)
    n = np.zeros(9000, np.float32)
    ref("f").lmref_stub_random_mesh(_ptr(p), _ptr(n))
    return p.reshape(-1, 3), n.reshape(-1, 3)


# ------------------------------------------------------------ rendering ----

class _RefRenderDesc(ctypes.Structure):
    _fields_ = [("num_prims", ctypes.c_int), ("positions", ctypes.POINTER(ctypes.c_void_p)),
                ("normals", ctypes.POINTER(ctypes.c_void_p)), ("faces", ctypes.POINTER(ctypes.c_void_p)),
                ("num_vertices", ctypes.c_void_p), ("num_faces", ctypes.c_void_p), ("material", ctypes.c_void_p),
                ("light", ctypes.c_void_p), ("num_materials", ctypes.c_int), ("mat_type", ctypes.c_void_p),
                ("mat_R", ctypes.c_void_p), ("num_lights", ctypes.c_int), ("light_Le", ctypes.c_void_p),
                ("has_env", ctypes.c_int), ("env_Le", ctypes.c_float * 3), ("eye", ctypes.c_float * 3),
                ("center", ctypes.c_float * 3), ("up", ctypes.c_float * 3), ("fovy", ctypes.c_float),
                ("width", ctypes.c_int), ("height", ctypes.c_int), ("renderer", ctypes.c_char_p),
                ("rr_depth", ctypes.c_int), ("max_path_vertices", ctypes.c_int), ("seed", ctypes.c_int),
                ("num_samples", ctypes.c_longlong), ("num_threads", ctypes.c_int),
                ("samples_per_block", ctypes.c_longlong), ("scene_type", ctypes.c_char_p),
                ("sched_type", ctypes.c_char_p)]


def flatten_primitives(prims):
    """World-space arrays of a lightmetrica_b200 Primitives description:
    per primitive positions/normals/faces, material (type, R) and light
    indices in first-use order, like the GPU scene description."""
    out = {"pos": [], "nrm": [], "faces": [], "mat": [], "light": []}
    mats, mat_index, lights, light_index = [], {}, [], {}
    for p in prims.primitives:
        m = p.mesh
        pos = m.positions.astype(np.float64)
        nrm = m.normals.astype(np.float64) if m.normals is not None else None
        if p.transform is not None:
            T = np.asarray(p.transform, np.float64).reshape(4, 4)
            pos = pos @ T[:3, :3].T + T[:3, 3]
            if nrm is not None:
                nrm = nrm @ np.linalg.inv(T[:3, :3])
        if nrm is None:
            nrm = np.zeros_like(pos)
            f = m.faces.astype(np.int64)
            g = np.cross(pos[f[:, 1]] - pos[f[:, 0]], pos[f[:, 2]] - pos[f[:, 0]])
            for c in range(3):
                nrm[f[:, c]] = g
        out["pos"].append(np.ascontiguousarray(pos, np.float32).reshape(-1))
        out["nrm"].append(np.ascontiguousarray(nrm, np.float32).reshape(-1))
        out["faces"].append(np.ascontiguousarray(m.faces, np.uint32).reshape(-1))
        if p.bsdf is not None:
            if id(p.bsdf) not in mat_index:
                mat_index[id(p.bsdf)] = len(mats)
                mats.append(p.bsdf)
            out["mat"].append(mat_index[id(p.bsdf)])
        else:
            out["mat"].append(-1)
        if p.light is not None:
            if id(p.light) not in light_index:
                light_index[id(p.light)] = len(lights)
                lights.append(p.light)
            out["light"].append(light_index[id(p.light)])
        else:
            out["light"].append(-1)
    out["mats"] = mats
    out["lights"] = lights
    return out


def _ref_desc(prims, renderer, num_samples, spp, rr_depth, max_path_vertices, seed, threads, samples_per_block,
              scene_type, sched_type):
    """The harness's flat scene description of `prims`, with the arrays it
    points into (keep them alive while the description is in use)."""
    fl = flatten_primitives(prims)
    cam = prims.camera
    W, H = cam.film.width, cam.film.height
    n = len(prims.primitives)
    keep = []

    def ptrs(arrs):
        a = (ctypes.c_void_p * n)(*[x.ctypes.data for x in arrs])
        keep.append(a)
        return a
    keep += [fl]
    nv = np.array([x.size // 3 for x in fl["pos"]], np.int32)
    nf = np.array([x.size // 3 for x in fl["faces"]], np.int32)
    mat = np.array(fl["mat"], np.int32)
    lig = np.array(fl["light"], np.int32)
    mt = np.array([m.kind for m in fl["mats"]] or [0], np.int32)
    mR = np.array([np.broadcast_to(np.asarray(m.reflectance, np.float32), (3,)) for m in fl["mats"]] or [[0, 0, 0]],
                  np.float32).reshape(-1)
    lLe = np.array([np.broadcast_to(np.asarray(l.luminance, np.float32), (3,)) for l in fl["lights"]] or [[0, 0, 0]],
                   np.float32).reshape(-1)
    keep += [nv, nf, mat, lig, mt, mR, lLe]
    d = _RefRenderDesc()
    d.num_prims = n
    d.positions = ptrs(fl["pos"])
    d.normals = ptrs(fl["nrm"])
    d.faces = ptrs(fl["faces"])
    d.num_vertices, d.num_faces, d.material, d.light = nv.ctypes.data, nf.ctypes.data, mat.ctypes.data, lig.ctypes.data
    d.num_materials = len(fl["mats"])
    d.mat_type, d.mat_R = mt.ctypes.data, mR.ctypes.data
    d.num_lights = len(fl["lights"])
    d.light_Le = lLe.ctypes.data
    if prims.environment_light is not None:
        d.has_env = 1
        le = np.broadcast_to(np.asarray(prims.environment_light.luminance, np.float32), (3,))
        for c in range(3):
            d.env_Le[c] = float(le[c])
    for c in range(3):
        d.eye[c], d.center[c], d.up[c] = cam.eye[c], cam.center[c], cam.up[c]
    d.fovy = cam.fovy
    d.width, d.height = W, H
    d.renderer = renderer.encode()
    d.rr_depth, d.max_path_vertices, d.seed = rr_depth, max_path_vertices, seed
    d.num_samples = int(num_samples if num_samples is not None else spp * W * H)
    d.num_threads = int(threads or os.cpu_count() or 1)
    d.samples_per_block = samples_per_block
    d.scene_type = scene_type.encode()
    d.sched_type = sched_type.encode()
    keep += [d.renderer, d.scene_type, d.sched_type]
    return d, keep


def _ref_error(L, code):
    L.lmref_last_error.restype = ctypes.c_char_p
    return f"reference render failed ({code}): {L.lmref_last_error().decode(errors='replace')}"


def ref_render(prims, renderer="pt", num_samples=None, spp=16, rr_depth=1, max_path_vertices=-1, seed=1,
               threads=None, precision="d", samples_per_block=100, scene_type="bvh", sched_type="mt"):
    """Renders `prims` with the reference's own component wiring (oracle/_ref):
    renderer `renderer`, scheduler `sched_type` (the reference's "mt") and
    accelerator `scene_type` (the reference's "bvh"); a loaded plugin's
    components ("plugin.gpu", "gpu.pt.mis", "gpu") can take any of the three
    slots. Returns (film (H, W, 3) float32, render seconds)."""
    L = ref(precision)
    if not hasattr(L, "lmref_render"):
        raise RuntimeError("reference harness built without the renderer")
    L.lmref_render.restype = ctypes.c_double
    L.lmref_render.argtypes = [ctypes.POINTER(_RefRenderDesc), ctypes.c_void_p, ctypes.POINTER(ctypes.c_double)]
    d, keep = _ref_desc(prims, renderer, num_samples, spp, rr_depth, max_path_vertices, seed, threads,
                        samples_per_block, scene_type, sched_type)
    cam = prims.camera
    film = np.zeros((cam.film.height, cam.film.width, 3), np.float32)
    bt = ctypes.c_double()
    secs = L.lmref_render(ctypes.byref(d), film.ctypes.data, ctypes.byref(bt))
    del keep
    if secs < 0:
        raise RuntimeError(_ref_error(L, secs))
    return film, secs


class RefRenderSession:
    """The reference's renderer (oracle/_ref, its own `mt` scheduler and
    `bvh` scene) built once and rendered several times: the timed CPU
    baseline of the path tracer. The scene is wrapped in the harness's
    counting scene, so every render reports the rays it traced (camera,
    bounce and shadow rays: every Scene::Intersect, scene.cpp:67-72).
    Successive renders continue the renderer's sampler (fresh samples)."""

    def __init__(self, prims, renderer="pt.mis", rr_depth=1, max_path_vertices=-1, seed=1, precision="f",
                 samples_per_block=100):
        L = ref(precision)
        if not hasattr(L, "lmref_session_create"):
            raise RuntimeError("reference harness built without render sessions")
        L.lmref_session_create.restype = ctypes.c_void_p
        L.lmref_session_create.argtypes = [ctypes.POINTER(_RefRenderDesc), ctypes.POINTER(ctypes.c_double),
                                           ctypes.POINTER(ctypes.c_int)]
        L.lmref_session_render.restype = ctypes.c_double
        L.lmref_session_render.argtypes = [ctypes.c_void_p, ctypes.c_longlong, ctypes.c_int, ctypes.c_void_p,
                                           ctypes.POINTER(ctypes.c_longlong)]
        L.lmref_session_destroy.argtypes = [ctypes.c_void_p]
        self._L = L
        d, keep = _ref_desc(prims, renderer, 1, 1, rr_depth, max_path_vertices, seed, None, samples_per_block,
                            "harness.counting", "mt")
        bt, st = ctypes.c_double(), ctypes.c_int()
        self._h = L.lmref_session_create(ctypes.byref(d), ctypes.byref(bt), ctypes.byref(st))
        del keep
        if not self._h:
            raise RuntimeError(_ref_error(L, st.value))
        self.build_seconds = bt.value
        self.width, self.height = prims.camera.film.width, prims.camera.film.height

    def render(self, num_samples: int, threads=None, film: bool = False):
        """Renders `num_samples` samples; returns (seconds of sched.Render,
        rays traced, rescaled film (H, W, 3) or None)."""
        out = np.zeros((self.height, self.width, 3), np.float32) if film else None
        rays = ctypes.c_longlong()
        secs = self._L.lmref_session_render(self._h, int(num_samples), int(threads or os.cpu_count() or 1),
                                            None if out is None else out.ctypes.data, ctypes.byref(rays))
        if secs < 0:
            raise RuntimeError(_ref_error(self._L, secs))
        return secs, rays.value, out

    def close(self):
        if self._h:
            self._L.lmref_session_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class _OrcPtDesc(ctypes.Structure):
    _fields_ = [("num_tris", ctypes.c_int), ("pos", ctypes.c_void_p), ("nrm", ctypes.c_void_p),
                ("tri_mat", ctypes.c_void_p), ("tri_light", ctypes.c_void_p), ("num_mats", ctypes.c_int),
                ("mat_type", ctypes.c_void_p), ("mat_R", ctypes.c_void_p), ("tri_albedo", ctypes.c_void_p),
                ("num_lights", ctypes.c_int), ("light_Le", ctypes.c_void_p), ("has_env", ctypes.c_int),
                ("env_Le", ctypes.c_float * 3), ("eye", ctypes.c_float * 3), ("center", ctypes.c_float * 3),
                ("up", ctypes.c_float * 3), ("fovy", ctypes.c_float), ("width", ctypes.c_int),
                ("height", ctypes.c_int), ("technique", ctypes.c_int), ("rr_depth", ctypes.c_int),
                ("max_pv", ctypes.c_int), ("sampling", ctypes.c_int), ("seed", ctypes.c_uint64),
                ("sample_begin", ctypes.c_int64), ("sample_end", ctypes.c_int64)]


_TECH = {"pt": 0, "pt.direct": 1, "pt.mis": 2}


def _pt_desc(prims, technique, rr_depth, max_path_vertices, seed, sampling, tri_albedo, light_Le):
    fl = flatten_primitives(prims)
    pos, nrm, tmat, tlight = [], [], [], []
    for k in range(len(fl["pos"])):
        P = fl["pos"][k].reshape(-1, 3)
        Nn = fl["nrm"][k].reshape(-1, 3)
        F = fl["faces"][k].reshape(-1, 3).astype(np.int64)
        pos.append(P[F].reshape(-1))
        nrm.append(Nn[F].reshape(-1))
        tmat.append(np.full(F.shape[0], fl["mat"][k], np.int32))
        tlight.append(np.full(F.shape[0], fl["light"][k], np.int32))
    keep = dict(pos=np.ascontiguousarray(np.concatenate(pos), np.float32),
                nrm=np.ascontiguousarray(np.concatenate(nrm), np.float32),
                tmat=np.concatenate(tmat), tlight=np.concatenate(tlight),
                mt=np.array([m.kind for m in fl["mats"]] or [0], np.int32),
                mR=np.array([np.broadcast_to(np.asarray(m.reflectance, np.float32), (3,)) for m in fl["mats"]]
                            or [[0, 0, 0]], np.float32).reshape(-1))
    if light_Le is None:
        light_Le = np.array([np.broadcast_to(np.asarray(l.luminance, np.float32), (3,)) for l in fl["lights"]]
                            or [[0, 0, 0]], np.float32)
    keep["lLe"] = np.ascontiguousarray(light_Le, np.float32).reshape(-1)
    if tri_albedo is not None:
        keep["alb"] = np.ascontiguousarray(tri_albedo, np.float32).reshape(-1)
    d = _OrcPtDesc()
    d.num_tris = keep["tmat"].size
    d.pos, d.nrm = keep["pos"].ctypes.data, keep["nrm"].ctypes.data
    d.tri_mat, d.tri_light = keep["tmat"].ctypes.data, keep["tlight"].ctypes.data
    d.num_mats = len(fl["mats"])
    d.mat_type, d.mat_R = keep["mt"].ctypes.data, keep["mR"].ctypes.data
    d.tri_albedo = keep["alb"].ctypes.data if "alb" in keep else None
    d.num_lights = len(fl["lights"])
    d.light_Le = keep["lLe"].ctypes.data
    if prims.environment_light is not None:
        d.has_env = 1
        le = np.broadcast_to(np.asarray(prims.environment_light.luminance, np.float32), (3,))
        for c in range(3):
            d.env_Le[c] = float(le[c])
    cam = prims.camera
    for c in range(3):
        d.eye[c], d.center[c], d.up[c] = cam.eye[c], cam.center[c], cam.up[c]
    d.fovy = cam.fovy
    d.width, d.height = cam.film.width, cam.film.height
    d.technique = _TECH[technique]
    d.rr_depth, d.max_pv = rr_depth, max_path_vertices
    d.sampling = 0 if sampling == "stratified" else 1
    d.seed = seed
    return d, keep


def _split_run(fn, d, total, threads, out_arrays):
    """Runs fn(desc copy, *per-thread outputs) over [0, total) samples on
    `threads` Python threads (ctypes releases the GIL) and sums the outputs."""
    import threading
    threads = max(1, min(threads or os.cpu_count() or 1, total))
    parts = [[np.zeros_like(a, dtype=np.float64) for a in out_arrays] for _ in range(threads)]
    descs = []
    for t in range(threads):
        dd = _OrcPtDesc()
        ctypes.pointer(dd)[0] = d
        dd.sample_begin = total * t // threads
        dd.sample_end = total * (t + 1) // threads
        descs.append(dd)
    ths = [threading.Thread(target=fn, args=(descs[t], parts[t])) for t in range(threads)]
    for th in ths:
        th.start()
    for th in ths:
        th.join()
    return [sum(p[i] for p in parts) for i in range(len(out_arrays))]


def oracle_render(prims, technique="pt.mis", spp=16, rr_depth=1, max_path_vertices=-1, seed=1,
                  sampling="stratified", threads=None, tri_albedo=None, light_Le=None):
    """The C restatement's render (double), rescaled like the reference film:
    (H, W, 3) float64."""
    L = lib()
    L.orc_render.restype = ctypes.c_int64
    L.orc_render.argtypes = [ctypes.POINTER(_OrcPtDesc), ctypes.c_void_p]
    d, keep = _pt_desc(prims, technique, rr_depth, max_path_vertices, seed, sampling, tri_albedo, light_Le)
    W, H = prims.camera.film.width, prims.camera.film.height
    total = W * H * spp

    def run(dd, outs):
        L.orc_render(ctypes.byref(dd), outs[0].ctypes.data)
    film, = _split_run(run, d, total, threads, [np.zeros(W * H * 3)])
    return (film * (W * H / total)).reshape(H, W, 3)


def oracle_render_range(prims, sample_begin, sample_end, technique="pt.mis", rr_depth=1, max_path_vertices=-1,
                        seed=1, sampling="stratified"):
    """The C restatement's un-rescaled film (W*H*3 float64 sums) of the
    samples [sample_begin, sample_end) only, one thread."""
    L = lib()
    L.orc_render.restype = ctypes.c_int64
    L.orc_render.argtypes = [ctypes.POINTER(_OrcPtDesc), ctypes.c_void_p]
    d, keep = _pt_desc(prims, technique, rr_depth, max_path_vertices, seed, sampling, None, None)
    W, H = prims.camera.film.width, prims.camera.film.height
    film = np.zeros(W * H * 3)
    d.sample_begin = int(sample_begin)
    d.sample_end = int(sample_end)
    L.orc_render(ctypes.byref(d), film.ctypes.data)
    return film


def oracle_grad(prims, dL_dimage, technique="pt.mis", spp=16, rr_depth=1, max_path_vertices=-1, seed=1,
                sampling="stratified", threads=None, tri_albedo=None, light_Le=None):
    """FP64 reference gradient of a loss with image gradient dL_dimage
    ((H, W, 3), w.r.t. the rescaled film) w.r.t. per-triangle albedo and
    area-light emission: returns (d_albedo (T, 3), d_Le (lights, 3))."""
    L = lib()
    L.orc_render_grad.restype = ctypes.c_int64
    L.orc_render_grad.argtypes = [ctypes.POINTER(_OrcPtDesc), ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p]
    d, keep = _pt_desc(prims, technique, rr_depth, max_path_vertices, seed, sampling, tri_albedo, light_Le)
    W, H = prims.camera.film.width, prims.camera.film.height
    total = W * H * spp
    g = np.ascontiguousarray(np.asarray(dL_dimage, np.float64).reshape(-1) * (W * H / total))
    T = d.num_tris
    nl = max(1, d.num_lights)

    def run(dd, outs):
        L.orc_render_grad(ctypes.byref(dd), g.ctypes.data, outs[0].ctypes.data, outs[1].ctypes.data)
    ga, gl = _split_run(run, d, total, threads, [np.zeros(3 * T), np.zeros(3 * nl)])
    return ga.reshape(T, 3), gl.reshape(nl, 3)[:d.num_lights]


# ------------------------------------------------ component evaluation ----
# The oracle's camera, sampling and BSDF functions (lmoracle_pt.c) for
# given inputs, in float64.

BSDF_TYPES = {"diffuse": 0, "mirror": 1, "diffuse_mirror": 2}


def _components():
    """liblmoracle with the component entry points' signatures declared."""
    L = lib()
    if not getattr(L, "_components_bound", False):
        P, I = ctypes.c_void_p, ctypes.c_int
        L.orc_eval_disk.argtypes = [P, I, P]
        L.orc_eval_cosine.argtypes = [P, I, P]
        L.orc_camera_rays.argtypes = [ctypes.POINTER(_OrcPtDesc), P, I, P, P]
        L.orc_camera_rays.restype = I
        L.orc_camera_raster.argtypes = [ctypes.POINTER(_OrcPtDesc), P, I, P, P]
        L.orc_camera_raster.restype = I
        L.orc_bsdf_sample.argtypes = [I, P, P, P, P, I, P, P, P, P]
        L.orc_bsdf_eval.argtypes = [I, P, P, P, P, I, P, P]
        L._components_bound = True
    return L


def _f64(a, cols):
    return np.ascontiguousarray(np.asarray(a, dtype=np.float64).reshape(-1, cols))


def eval_disk(u):
    """UniformConcentricDiskSample of u (n x 2) -> (n x 2)."""
    u = _f64(u, 2)
    out = np.empty_like(u)
    _components().orc_eval_disk(_ptr(u), u.shape[0], _ptr(out))
    return out


def eval_cosine(u):
    """CosineSampleHemisphere of u (n x 2) -> (n x 3)."""
    u = _f64(u, 2)
    out = np.empty((u.shape[0], 3))
    _components().orc_eval_cosine(_ptr(u), u.shape[0], _ptr(out))
    return out


def _camera_desc(eye, center, up, fovy, width, height):
    d = _OrcPtDesc()
    d.eye[:], d.center[:], d.up[:] = list(map(float, eye)), list(map(float, center)), list(map(float, up))
    d.fovy, d.width, d.height = float(fovy), int(width), int(height)
    return d


def light_sample(prims, u):
    """The C restatement's light sample (scene.cpp:79-86, light.area.cpp:146-179,
    light.env.const.cpp:194-203) of the scene's lights for (u0, u1) (n x 2):
    (points (n x 7: position, normal, area pdf times the selection
    probability), light index (n))."""
    L = lib()
    L.orc_light_sample.restype = ctypes.c_int
    L.orc_light_sample.argtypes = [ctypes.POINTER(_OrcPtDesc), ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p,
                                   ctypes.c_void_p]
    d, keep = _pt_desc(prims, "pt.mis", 1, -1, 1, "stratified", None, None)
    uu = _f64(u, 2)
    out, light = np.empty((uu.shape[0], 7)), np.empty(uu.shape[0], dtype=np.int32)
    if not L.orc_light_sample(ctypes.byref(d), _ptr(uu), uu.shape[0], _ptr(out), _ptr(light)):
        raise ValueError("scene setup failed")
    return out, light


def camera_rays(raster, eye, center, up, fovy, width, height):
    """Raster positions (n x 2) -> (origins and directions (n x 6), pdf (n))."""
    r = _f64(raster, 2)
    rays, pdf = np.empty((r.shape[0], 6)), np.empty(r.shape[0])
    d = _camera_desc(eye, center, up, fovy, width, height)
    if not _components().orc_camera_rays(ctypes.byref(d), _ptr(r), r.shape[0], _ptr(rays), _ptr(pdf)):
        raise ValueError("degenerate camera")
    return rays, pdf


def camera_raster(rays, eye, center, up, fovy, width, height):
    """Rays (n x 6: origin, direction) -> (raster (n x 2), valid (n))."""
    r = _f64(rays, 6)
    raster, valid = np.empty((r.shape[0], 2)), np.empty(r.shape[0], dtype=np.int32)
    d = _camera_desc(eye, center, up, fovy, width, height)
    if not _components().orc_camera_raster(ctypes.byref(d), _ptr(r), r.shape[0], _ptr(raster), _ptr(valid)):
        raise ValueError("degenerate camera")
    return raster, valid.astype(bool)


def bsdf_sample(bsdf, R, frames, wi, u):
    """SampleAndEstimateDirection: frames (n x 6: gn, sn), wi (n x 3), u (n x 3)
    -> dict of wo, weight (n x 3), pdf (n), specular (n)."""
    f, w, uu = _f64(frames, 6), _f64(wi, 3), _f64(u, 3)
    n = f.shape[0]
    R = _f64(R, 3)
    out = {"wo": np.empty((n, 3)), "weight": np.empty((n, 3)), "pdf": np.empty(n), "specular": np.empty(n, dtype=np.int32)}
    _components().orc_bsdf_sample(BSDF_TYPES[bsdf], _ptr(R), _ptr(f), _ptr(w), _ptr(uu), n,
                          _ptr(out["wo"]), _ptr(out["weight"]), _ptr(out["pdf"]), _ptr(out["specular"]))
    out["specular"] = out["specular"].astype(bool)
    return out


def bsdf_eval(bsdf, R, frames, wi, wo):
    """EvaluateDirection / EvaluateDirectionPDF (NonDelta): -> (f (n x 3), pdf (n))."""
    f, a, b = _f64(frames, 6), _f64(wi, 3), _f64(wo, 3)
    n = f.shape[0]
    R = _f64(R, 3)
    fs, pdf = np.empty((n, 3)), np.empty(n)
    _components().orc_bsdf_eval(BSDF_TYPES[bsdf], _ptr(R), _ptr(f), _ptr(a), _ptr(b), n,
                        _ptr(fs), _ptr(pdf))
    return fs, pdf
