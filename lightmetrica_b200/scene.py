"""Scene side of the component mirror: meshes, primitives, BSDF / light /
camera descriptors and the Scene component (reference scene.h:47-191).
"""
from __future__ import annotations

import ctypes
from dataclasses import dataclass, field
from typing import List, Optional

import numpy as np

from . import native as N


# ------------------------------------------------------------- assets ------

@dataclass
class TriangleMesh:
    """Reference TriangleMesh (trianglemesh.h:34-84): positions/normals
    (3 per vertex), texcoords (2 per vertex), faces (3 indices per triangle)."""
    positions: np.ndarray
    faces: np.ndarray
    normals: Optional[np.ndarray] = None
    texcoords: Optional[np.ndarray] = None

    def __post_init__(self):
        self.positions = np.ascontiguousarray(self.positions, np.float32).reshape(-1, 3)
        self.faces = np.ascontiguousarray(self.faces, np.uint32).reshape(-1, 3)
        if self.normals is not None:
            self.normals = np.ascontiguousarray(self.normals, np.float32).reshape(-1, 3)
        if self.texcoords is not None:
            self.texcoords = np.ascontiguousarray(self.texcoords, np.float32).reshape(-1, 2)

    def num_faces(self) -> int:
        return int(self.faces.shape[0])


@dataclass
class DiffuseBSDF:
    """Reference `diffuse` (diffuse.cpp): Lambertian, diffuse_reflectance R."""
    reflectance: tuple = (1.0, 1.0, 1.0)
    kind: int = N.BSDF_DIFFUSE


@dataclass
class PerfectMirrorBSDF:
    """Reference `mirror` (mirror.cpp): perfect specular reflection."""
    reflectance: tuple = (1.0, 1.0, 1.0)
    kind: int = N.BSDF_MIRROR


@dataclass
class DiffuseMirrorBSDF:
    """Reference `plugin.diffusemirror` (diffusemirror.cpp): 50/50 mixture."""
    reflectance: tuple = (1.0, 1.0, 1.0)
    kind: int = N.BSDF_DIFFUSE_MIRROR


@dataclass
class AreaLight:
    """Reference `area` light (light.area.cpp): emits `luminance` from the
    front side (w.r.t. the shading normal) of its primitives."""
    luminance: tuple = (1.0, 1.0, 1.0)


@dataclass
class ConstantEnvironmentLight:
    """Reference `env.const` (light.env.const.cpp)."""
    luminance: tuple = (1.0, 1.0, 1.0)


@dataclass
class HDRBitmapFilm:
    """Reference `hdr` film (hdrfilm.cpp): W x H x 3, row y = 0 first."""
    width: int
    height: int
    data: Optional[np.ndarray] = None
    image_type: str = "radiancehdr"        # or "openexr" (hdrfilm.cpp:88-107)

    def internal_data(self) -> np.ndarray:
        if self.data is None:
            self.data = np.zeros((self.height, self.width, 3), np.float32)
        return self.data

    def allocate(self, width: int, height: int) -> None:
        """HDRBitmapFilm::Allocate (hdrfilm.cpp:327-332): zeroed W x H."""
        self.width, self.height = int(width), int(height)
        self.data = np.zeros((self.height, self.width, 3), np.float32)

    def pixel_of(self, raster) -> int:
        """Pixel index of a raster position in [0,1]^2, or -1 outside it:
        int(r * W) in float arithmetic, clamped to the film
        (hdrfilm.cpp:151-163)."""
        rx, ry = np.float32(raster[0]), np.float32(raster[1])
        if rx < 0 or rx > 1 or ry < 0 or ry > 1:
            return -1
        x = min(max(int(rx * np.float32(self.width)), 0), self.width - 1)
        y = min(max(int(ry * np.float32(self.height)), 0), self.height - 1)
        return y * self.width + x

    def record_contribution(self, raster, contribution) -> bool:
        """HDRBitmapFilm::RecordContribution (hdrfilm.cpp:129-149): sets the pixel."""
        i = self.pixel_of(raster)
        if i < 0:
            return False
        self.internal_data().reshape(-1, 3)[i] = np.asarray(contribution, np.float32)
        return True

    def accumulate_contribution(self, raster, contribution) -> bool:
        """HDRBitmapFilm::AccumulateContribution(rasterPos, contrb)
        (hdrfilm.cpp:151-171): adds to the pixel; a position outside [0,1]^2
        is ignored (the reference logs a warning)."""
        i = self.pixel_of(raster)
        if i < 0:
            return False
        self.internal_data().reshape(-1, 3)[i] += np.asarray(contribution, np.float32)
        return True

    def accumulate_film(self, other: "HDRBitmapFilm") -> bool:
        """HDRBitmapFilm::AccumulateContribution(film) (hdrfilm.cpp:173-197):
        adds another film of the same size (else ignored, as the reference)."""
        if other.width != self.width or other.height != self.height:
            return False
        self.internal_data()[...] += other.internal_data()
        return True

    def rescale(self, weight: float) -> None:
        """HDRBitmapFilm::Rescale (hdrfilm.cpp:334-341)."""
        self.internal_data()[...] *= np.float32(weight)

    def clone(self) -> "HDRBitmapFilm":
        return HDRBitmapFilm(self.width, self.height, self.internal_data().copy(), self.image_type)

    def rescale_and_save(self, path: str, weight: float = 1.0) -> str:
        """HDRBitmapFilm::RescaleAndSave (hdrfilm.cpp:199-304); returns the
        path written (see film_io for the naming rules)."""
        from .film_io import save_film
        return save_film(self.internal_data(), path, self.image_type, weight)

    def save(self, path: str) -> str:
        return self.rescale_and_save(path, 1.0)


@dataclass
class PerspectiveCamera:
    """Reference `perspective` camera (perspectivecamera.cpp) placed by a
    LookAt transform."""
    fovy: float
    eye: tuple
    center: tuple
    up: tuple
    film: HDRBitmapFilm = None


@dataclass
class Primitive:
    """Reference Primitive (primitive.h:39-60)."""
    mesh: Optional[TriangleMesh] = None
    transform: Optional[np.ndarray] = None   # 4x4, applied as M @ (x, y, z, 1)
    bsdf: object = None
    light: Optional[AreaLight] = None


@dataclass
class Primitives:
    """Reference Primitives (primitives.h:43-139): the flattened scene."""
    primitives: List[Primitive] = field(default_factory=list)
    camera: Optional[PerspectiveCamera] = None
    environment_light: Optional[ConstantEnvironmentLight] = None

    def add(self, p: Primitive) -> "Primitives":
        self.primitives.append(p)
        return self

    def main_camera(self):
        return self.camera

    def num_lights(self) -> int:
        lights = {id(p.light) for p in self.primitives if p.light is not None}
        return len(lights) + (1 if self.environment_light is not None else 0)


# -------------------------------------------------------------- scene -----

_LAYOUTS = {"bvh": N.LAYOUT_BVH2, "qbvh": N.LAYOUT_BVH4, "naive": N.LAYOUT_NAIVE,
            "plugin.gpu": N.LAYOUT_BVH2, "plugin.gpu.bvh4": N.LAYOUT_BVH4}


class Scene:
    """GPU implementation of the reference Scene component. `impl` names the
    accelerator: "bvh" (binary, bit-identical to the reference BVHScene),
    "qbvh" (4-wide collapse of the same tree, also bit-identical) or "naive"."""

    def __init__(self, impl: str = "bvh"):
        if impl not in _LAYOUTS:
            raise ValueError(f"unknown scene type '{impl}'")
        self.impl = impl
        self.layout = _LAYOUTS[impl]
        self.primitives: Optional[Primitives] = None
        self.build_threads = 0
        self.max_stack_entries = 0
        self.render_tree = N.RENDER_TREE_SAH
        self.handle = None
        self._keep = []

    # reference Scene::Load (scene.cpp:42-45)
    def load(self, primitives: Primitives) -> None:
        self.primitives = primitives

    # reference Scene::Configure: the GPU scene reads `build_threads`,
    # `max_stack_entries` (the traversal stack bound per ray, 0 = automatic)
    # and `render_tree` ("sah": renders traverse a second tree built for
    # traversal cost, the default; "reference": the reference's tree).
    def configure(self, node: Optional[dict] = None) -> bool:
        node = node or {}
        self.build_threads = int(node.get("build_threads", 0))
        self.max_stack_entries = int(node.get("max_stack_entries", 0))
        if self.max_stack_entries < 0:
            raise ValueError("max_stack_entries must be >= 0")
        tree = node.get("render_tree", "sah")
        if tree not in ("sah", "reference"):
            raise ValueError("render_tree must be 'sah' or 'reference'")
        self.render_tree = N.RENDER_TREE_SAH if tree == "sah" else N.RENDER_TREE_REFERENCE
        return True

    def build(self) -> bool:
        """Scene::Build: host BVH build + upload. Raises LmgpuError on failure."""
        if self.primitives is None:
            raise RuntimeError("Scene.build() before Scene.load()")
        desc, keep = self._describe()
        h = ctypes.c_void_p()
        N.check(N.lib().lmgpu_scene_create(ctypes.byref(desc), ctypes.byref(h)))
        self.close()
        self.handle = h
        self._keep = keep
        return True

    def close(self):
        if self.handle is not None and self.handle.value:
            N.lib().lmgpu_scene_destroy(self.handle)
        self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def info(self) -> dict:
        inf = N.SceneInfo()
        N.check(N.lib().lmgpu_scene_info(self.handle, ctypes.byref(inf)))
        return {"num_triangles": inf.num_triangles, "num_nodes": inf.num_nodes, "num_leaves": inf.num_leaves,
                "max_depth": inf.max_depth, "layout": inf.layout, "device_bytes": inf.device_bytes,
                "build_seconds": inf.build_seconds,
                "bounds_min": list(inf.bounds_min), "bounds_max": list(inf.bounds_max),
                "render_tree": "sah" if inf.render_tree == N.RENDER_TREE_SAH else "reference",
                "render_max_depth": inf.render_max_depth, "render_num_nodes": inf.render_num_nodes,
                "render_num_leaves": inf.render_num_leaves, "render_build_seconds": inf.render_build_seconds}

    def get_aabb_triangles(self):
        i = self.info()
        return np.array(i["bounds_min"], np.float32), np.array(i["bounds_max"], np.float32)

    def main_camera(self):
        return self.primitives.camera if self.primitives else None

    # ---- queries
    def intersect_host(self, rays_aos: np.ndarray) -> dict:
        """Closest hits for host AoS rays (n, 8): o, d, minT, maxT."""
        rays = np.ascontiguousarray(rays_aos, np.float32).reshape(-1, 8)
        n = rays.shape[0]
        out = {"tri_id": np.empty(n, np.int32), "t": np.empty(n, np.float32),
               "u": np.empty(n, np.float32), "v": np.empty(n, np.float32)}
        N.check(N.lib().lmgpu_intersect_host(self.handle, rays.ctypes.data, n, out["tri_id"].ctypes.data,
                                             out["t"].ctypes.data, out["u"].ctypes.data, out["v"].ctypes.data))
        return out

    def intersect_full_host(self, rays_aos: np.ndarray) -> dict:
        """Scene::Intersect with the full hit record (p, gn, sn, ss, st, uv)."""
        rays = np.ascontiguousarray(rays_aos, np.float32).reshape(-1, 8)
        n = rays.shape[0]
        ids = np.empty(n, np.int32)
        t = np.empty(n, np.float32)
        g = np.empty((n, 17), np.float32)
        kind = np.empty(n, np.int32)
        N.check(N.lib().lmgpu_intersect_full_host(self.handle, rays.ctypes.data, n, ids.ctypes.data,
                                                  t.ctypes.data, g.ctypes.data, kind.ctypes.data))
        return {"tri_id": ids, "t": t, "kind": kind, "p": g[:, 0:3], "gn": g[:, 3:6], "sn": g[:, 6:9],
                "ss": g[:, 9:12], "st": g[:, 12:15], "uv": g[:, 15:17]}

    def intersect_device(self, rays: dict, hits: dict, n: int, stream: int = 0) -> None:
        """Asynchronous batch query on device buffers. `rays` maps ox..tmax and
        `hits` maps tri_id/t/u/v to device pointers (ints)."""
        R = N.RaysSoA(*[rays[k] for k in ("ox", "oy", "oz", "dx", "dy", "dz", "tmin", "tmax")])
        H = N.HitsSoA(*[hits.get(k) for k in ("tri_id", "t", "u", "v")])
        N.check(N.lib().lmgpu_intersect(self.handle, ctypes.byref(R), n, ctypes.byref(H), ctypes.c_void_p(stream)))

    def occluded_device(self, rays: dict, occluded_ptr: int, n: int, stream: int = 0) -> None:
        R = N.RaysSoA(*[rays[k] for k in ("ox", "oy", "oz", "dx", "dy", "dz", "tmin", "tmax")])
        N.check(N.lib().lmgpu_occluded(self.handle, ctypes.byref(R), n, ctypes.c_void_p(occluded_ptr),
                                       ctypes.c_void_p(stream)))

    def status(self, stream: int = 0) -> None:
        """Raises if a kernel flagged a device error (stack/queue overflow, timeout)."""
        N.check(N.lib().lmgpu_scene_status(self.handle, ctypes.c_void_p(stream)))

    # ---- description marshalling
    def _describe(self):
        P = self.primitives
        keep = []
        mats, mat_index = [], {}
        lights, light_index = [], {}
        prims = (N.PrimitiveDesc * max(1, len(P.primitives)))()
        for i, p in enumerate(P.primitives):
            d = prims[i]
            m = p.mesh
            if m is not None:
                arrs = [m.positions, m.faces]
                d.positions = m.positions.ctypes.data_as(ctypes.POINTER(ctypes.c_float))
                d.faces = m.faces.ctypes.data_as(ctypes.POINTER(ctypes.c_uint32))
                d.num_vertices = m.positions.shape[0]
                d.num_faces = m.faces.shape[0]
                if m.normals is not None:
                    d.normals = m.normals.ctypes.data_as(ctypes.POINTER(ctypes.c_float))
                    arrs.append(m.normals)
                if m.texcoords is not None:
                    d.texcoords = m.texcoords.ctypes.data_as(ctypes.POINTER(ctypes.c_float))
                    arrs.append(m.texcoords)
                keep += arrs
            if p.transform is not None:
                tr = np.ascontiguousarray(np.asarray(p.transform, np.float32).reshape(4, 4).T).reshape(-1)
                keep.append(tr)
                d.transform = tr.ctypes.data_as(ctypes.POINTER(ctypes.c_float))
            if p.bsdf is not None:
                if id(p.bsdf) not in mat_index:
                    mat_index[id(p.bsdf)] = len(mats)
                    mats.append(p.bsdf)
                d.material = mat_index[id(p.bsdf)]
            else:
                d.material = -1
            if p.light is not None:
                if id(p.light) not in light_index:
                    light_index[id(p.light)] = len(lights)
                    lights.append(p.light)
                d.area_light = light_index[id(p.light)]
            else:
                d.area_light = -1
        mat_arr = (N.MaterialDesc * max(1, len(mats)))()
        for i, m in enumerate(mats):
            mat_arr[i].type = m.kind
            for c in range(3):
                mat_arr[i].reflectance[c] = float(np.broadcast_to(np.asarray(m.reflectance, np.float32), (3,))[c])
        light_arr = (N.AreaLightDesc * max(1, len(lights)))()
        for i, L in enumerate(lights):
            for c in range(3):
                light_arr[i].luminance[c] = float(np.broadcast_to(np.asarray(L.luminance, np.float32), (3,))[c])
        desc = N.SceneDesc()
        desc.primitives = prims
        desc.num_primitives = len(P.primitives)
        desc.materials = mat_arr
        desc.num_materials = len(mats)
        desc.area_lights = light_arr
        desc.num_area_lights = len(lights)
        if P.environment_light is not None:
            desc.has_env_light = 1
            le = np.broadcast_to(np.asarray(P.environment_light.luminance, np.float32), (3,))
            for c in range(3):
                desc.env_luminance[c] = float(le[c])
        cam = P.camera
        if cam is not None:
            desc.has_camera = 1
            for c in range(3):
                desc.camera_eye[c] = float(cam.eye[c])
                desc.camera_center[c] = float(cam.center[c])
                desc.camera_up[c] = float(cam.up[c])
            desc.camera_fovy_degrees = float(cam.fovy)
            desc.film_width = cam.film.width
            desc.film_height = cam.film.height
        desc.layout = self.layout
        desc.build_threads = self.build_threads
        desc.max_stack_entries = self.max_stack_entries
        desc.render_tree = self.render_tree
        keep += [prims, mat_arr, light_arr]
        return desc, keep


def create_scene(impl: str = "bvh") -> Scene:
    """ComponentFactory::Create<Scene>(impl)."""
    return Scene(impl)


def soup_primitives(positions: np.ndarray, faces: np.ndarray, normals=None, texcoords=None) -> Primitives:
    """One identity-transform primitive over world-space triangles."""
    return Primitives(primitives=[Primitive(mesh=TriangleMesh(positions, faces, normals, texcoords))])
