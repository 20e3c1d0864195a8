"""Scene ingestion: lightmetrica's XML scene documents -> Primitives plus
the renderer and scheduler configuration, so that the reference's scene
files render through this package end to end.

Document (main.cpp:255-612): a root element `lightmetrica` (or the older
`nanon`) with `assets`, `scene`, `renderer` and `render_scheduler`.

* Assets (assets.cpp:150-310): groups `triangle_meshes`, `bsdfs`, `films`,
  `cameras`, `lights`, `textures`, each asset with a unique `id` and a
  `type`; other elements refer to an asset with `ref="id"`.
  - triangle_mesh `raw` (rawmesh.cpp:65-89): `positions`, `normals` and
    `faces` required, `texcoords` optional; `obj` (objmesh.cpp): `path`,
    relative to the document, read by `load_obj` below.
  - bsdf `diffuse` (diffuse.cpp:68-107): `diffuse_reflectance` with a
    `color` child or a `texture` reference (a plain value is accepted too,
    as older documents write it); `mirror` (mirror.cpp:64):
    `specular_reflectance`, default 1; `plugin.diffusemirror`
    (diffusemirror.cpp:49): `diffuse_reflectance`, default 1.
  - texture `constant` (constanttexture.cpp:40): `color`, default 1.
  - light `area` (light.area.cpp:89) and `env.const`
    (light.env.const.cpp:84): `luminance` required.
  - camera `perspective` (perspectivecamera.cpp:101-140): `film` reference,
    `fovy` required.
  - film `hdr` (hdrfilm.cpp:84-107): `width`, `height`, `imagetype`
    (`radiancehdr` default, or `openexr`).
* Scene nodes (primitives.cpp:251-416): `scene/root` and nested `node`
  elements; each node's world transform is parent * local (`transform`),
  or its `global_transform` alone. A transform is a column-major `matrix`,
  a `lookat` (position, center, up), or translate * rotate(angle, axis) *
  scale. A node with a `triangle_mesh` needs a `bsdf`; `camera` and
  `light` exclude each other; leaf nodes have no children; `id` attributes
  are unique. The first camera is the main camera; a light without a mesh
  is the environment (`env.const`).

Transform arithmetic is float32, as in the reference's single-precision
build (math.transform.inl: Translate, Rotate, Scale, LookAt).
"""
from __future__ import annotations

import os
import xml.etree.ElementTree as ET
from dataclasses import dataclass, field
from typing import Dict, Optional

import numpy as np

from .scene import (AreaLight, ConstantEnvironmentLight, DiffuseBSDF, DiffuseMirrorBSDF, HDRBitmapFilm,
                    PerfectMirrorBSDF, PerspectiveCamera, Primitive, Primitives, TriangleMesh)

F = np.float32
ROOT_NAMES = ("lightmetrica", "nanon")
ASSET_GROUPS = {"triangle_meshes": "triangle_mesh", "bsdfs": "bsdf", "films": "film", "cameras": "camera",
                "lights": "light", "textures": "texture"}


class SceneFormatError(ValueError):
    pass


@dataclass
class SceneDocument:
    primitives: Primitives
    scene_type: str = "bvh"
    renderer_type: str = "pt"
    renderer_config: dict = field(default_factory=dict)
    scheduler_type: str = "mt"
    scheduler_config: dict = field(default_factory=dict)
    image_type: str = "radiancehdr"
    ids: Dict[str, int] = field(default_factory=dict)     # node id -> primitive index


# ------------------------------------------------------------ values ------

def _floats(elem, n: Optional[int] = None) -> np.ndarray:
    if elem is None or elem.text is None:
        raise SceneFormatError("missing value")
    v = np.array([float(x) for x in elem.text.split()], F)
    if n is not None and v.size != n:
        raise SceneFormatError(f"<{elem.tag}> needs {n} values, has {v.size}")
    return v


def _child(elem, name):
    return elem.find(name) if elem is not None else None


def _value(elem, name, n=None, default=None):
    c = _child(elem, name)
    if c is None:
        if default is None:
            raise SceneFormatError(f"missing <{name}> in <{elem.tag}>")
        return np.array(default, F)
    return _floats(c, n)


# ------------------------------------------------------- float32 math -----

def _dot(a, b):
    return F(F(F(a[0] * b[0]) + F(a[1] * b[1])) + F(a[2] * b[2]))


def _normalize(v):
    length = F(np.sqrt(_dot(v, v)))
    return np.array([F(x / length) for x in v], F)


def _cross(a, b):
    return np.array([F(F(a[1] * b[2]) - F(a[2] * b[1])), F(F(a[2] * b[0]) - F(a[0] * b[2])),
                     F(F(a[0] * b[1]) - F(a[1] * b[0]))], F)


def mat_mul(a: np.ndarray, b: np.ndarray) -> np.ndarray:
    """Row-major 4x4 float32 product a @ b, each result column formed as
    (c0 x + c1 y) + (c2 z + c3 w) from a's columns, like the reference's
    Mat4f * Vec4f."""
    a = np.asarray(a, F)
    b = np.asarray(b, F)
    out = np.zeros((4, 4), F)
    for j in range(4):
        x, y, z, w = b[:, j]
        for i in range(4):
            out[i, j] = F(F(F(a[i, 0] * x) + F(a[i, 1] * y)) + F(F(a[i, 2] * z) + F(a[i, 3] * w)))
    return out


def translate(v) -> np.ndarray:
    m = np.eye(4, dtype=F)
    m[:3, 3] = np.asarray(v, F)
    return m


def scale(v) -> np.ndarray:
    return np.diag(np.array([v[0], v[1], v[2], 1.0], F)).astype(F)


def rotate(angle_deg, axis) -> np.ndarray:
    """Rotation by angle_deg about axis (math.transform.inl Rotate, float)."""
    rad = F(F(angle_deg) * F(np.pi / 180.0))
    c, s = F(np.cos(rad)), F(np.sin(rad))
    a = _normalize(np.asarray(axis, F))
    t = np.array([F(F(1.0 - c) * x) for x in a], F)
    cols = [np.array([c, 0, 0], F) + a * t[0] + np.array([0, F(s * a[2]), F(-s * a[1])], F),
            np.array([0, c, 0], F) + a * t[1] + np.array([F(-s * a[2]), 0, F(s * a[0])], F),
            np.array([0, 0, c], F) + a * t[2] + np.array([F(s * a[1]), F(-s * a[0]), 0], F)]
    m = np.eye(4, dtype=F)
    for j in range(3):
        m[:3, j] = cols[j]
    return m


def look_at(eye, center, up) -> np.ndarray:
    eye, center, up = (np.asarray(v, F) for v in (eye, center, up))
    f = _normalize(center - eye)
    u = _normalize(up)
    s = _normalize(_cross(f, u))
    u = _cross(s, f)
    m = np.eye(4, dtype=F)
    m[0, :3], m[1, :3], m[2, :3] = s, u, -f
    m[0, 3], m[1, 3], m[2, 3] = -_dot(s, eye), -_dot(u, eye), _dot(f, eye)
    return m


def parse_transform(elem) -> np.ndarray:
    """PrimitivesImpl::ParseTransform (primitives.cpp:418-498): row-major 4x4."""
    mat = _child(elem, "matrix")
    if mat is not None:
        return _floats(mat, 16).reshape(4, 4).T.copy()      # the element is column-major
    la = _child(elem, "lookat")
    if la is not None:
        return look_at(_value(la, "position", 3), _value(la, "center", 3), _value(la, "up", 3))
    T = np.eye(4, dtype=F)
    R = np.eye(4, dtype=F)
    S = np.eye(4, dtype=F)
    if _child(elem, "translate") is not None:
        T = translate(_value(elem, "translate", 3))
    rot = _child(elem, "rotate")
    if rot is not None:
        if _child(rot, "matrix") is not None:
            R = _floats(_child(rot, "matrix"), 16).reshape(4, 4).T.copy()
        elif _child(rot, "quat") is not None:
            raise SceneFormatError("rotation by quaternion is not supported (nor by the reference)")
        else:
            R = rotate(float(_value(rot, "angle", 1)[0]), _value(rot, "axis", 3))
    if _child(elem, "scale") is not None:
        S = scale(_value(elem, "scale", 3))
    return mat_mul(mat_mul(T, R), S)


# ------------------------------------------------------------- meshes -----

def load_obj(path: str) -> TriangleMesh:
    """Wavefront obj: `v`, `vt`, `vn`, `f` (polygons fanned into triangles,
    indices 1-based or negative); vertices that share position, texture and
    normal indices are joined. Faces without normals get their flat face
    normal (vertices split per face), as the reference's importer flags
    (GenNormals | Triangulate | JoinIdenticalVertices, objmesh.cpp:151-156)
    ask. All objects of the file form one mesh."""
    V, VT, VN = [], [], []
    faces = []
    with open(path) as f:
        for line in f:
            p = line.split()
            if not p or p[0].startswith("#"):
                continue
            if p[0] == "v":
                V.append([float(x) for x in p[1:4]])
            elif p[0] == "vt":
                VT.append([float(x) for x in p[1:3]])
            elif p[0] == "vn":
                VN.append([float(x) for x in p[1:4]])
            elif p[0] == "f":
                corners = []
                for c in p[1:]:
                    ids = (c.split("/") + ["", ""])[:3]

                    def res(s, n):
                        if s == "":
                            return -1
                        i = int(s)
                        return i - 1 if i > 0 else n + i
                    corners.append((res(ids[0], len(V)), res(ids[1], len(VT)), res(ids[2], len(VN))))
                for k in range(1, len(corners) - 1):
                    faces.append((corners[0], corners[k], corners[k + 1]))
    V = np.array(V, np.float64).reshape(-1, 3)
    VT = np.array(VT, np.float64).reshape(-1, 2)
    VN = np.array(VN, np.float64).reshape(-1, 3)
    key_index = {}
    pos, nrm, uv, out_faces = [], [], [], []
    has_uv = all(c[1] >= 0 for f3 in faces for c in f3) and len(faces) > 0
    for fi, f3 in enumerate(faces):
        flat = None
        if any(c[2] < 0 for c in f3):
            a, b, c = (V[x[0]] for x in f3)
            n = np.cross(b - a, c - a)
            ln = np.linalg.norm(n)
            flat = n / ln if ln > 0 else np.array([0.0, 0.0, 1.0])
        tri = []
        for c in f3:
            key = (c[0], c[1] if has_uv else -1, c[2]) if flat is None else (c[0], c[1] if has_uv else -1, -2 - fi)
            if key not in key_index:
                key_index[key] = len(pos)
                pos.append(V[c[0]])
                nrm.append(VN[c[2]] if flat is None else flat)
                uv.append(VT[c[1]] if has_uv else (0.0, 0.0))
            tri.append(key_index[key])
        out_faces.append(tri)
    return TriangleMesh(np.array(pos, np.float32).reshape(-1, 3), np.array(out_faces, np.uint32).reshape(-1, 3),
                        np.array(nrm, np.float32).reshape(-1, 3),
                        np.array(uv, np.float32).reshape(-1, 2) if has_uv else None)


def _raw_mesh(elem) -> TriangleMesh:
    pos = _floats(_child(elem, "positions"))
    nrm = _floats(_child(elem, "normals")) if _child(elem, "normals") is not None else None
    if nrm is None:
        raise SceneFormatError("raw mesh needs <normals>")                 # rawmesh.cpp:74-78
    if _child(elem, "faces") is None:
        raise SceneFormatError("raw mesh needs <faces>")
    faces = np.array([int(x) for x in _child(elem, "faces").text.split()], np.int64)
    tc = _floats(_child(elem, "texcoords")) if _child(elem, "texcoords") is not None else None
    if pos.size % 3 or nrm.size != pos.size or faces.size % 3 or (tc is not None and tc.size * 3 != pos.size * 2):
        raise SceneFormatError("raw mesh arrays have inconsistent sizes")
    if faces.size and (faces.min() < 0 or faces.max() >= pos.size // 3):
        raise SceneFormatError("raw mesh face index out of range")
    return TriangleMesh(pos.reshape(-1, 3), faces.astype(np.uint32).reshape(-1, 3), nrm.reshape(-1, 3),
                        None if tc is None else tc.reshape(-1, 2))


# ------------------------------------------------------------- assets -----

class _Assets:
    def __init__(self, elem, base_dir):
        self.elems: Dict[str, ET.Element] = {}
        self.group_of: Dict[str, str] = {}
        self.objs: Dict[str, object] = {}
        self.base_dir = base_dir
        if elem is None:
            return
        for group in elem:
            if group.tag not in ASSET_GROUPS:
                raise SceneFormatError(f"unknown asset group <{group.tag}>")
            for a in group:
                if a.tag != ASSET_GROUPS[group.tag]:
                    raise SceneFormatError(f"invalid element <{a.tag}> in <{group.tag}>")
                aid = a.get("id")
                if not aid:
                    raise SceneFormatError("missing attribute 'id'")
                if aid in self.elems:
                    raise SceneFormatError(f"ID '{aid}' is already registered")
                self.elems[aid] = a
                self.group_of[aid] = a.tag

    def resolve(self, ref_elem, kind):
        if ref_elem is None:
            return None
        aid = ref_elem.get("ref")
        if aid is None:
            raise SceneFormatError(f"<{ref_elem.tag}> needs a 'ref' attribute")
        if aid not in self.elems:
            raise SceneFormatError(f"unknown asset '{aid}'")
        if self.group_of[aid] != kind:
            raise SceneFormatError(f"invalid reference to asset type '{self.group_of[aid]}' (expected '{kind}')")
        if aid not in self.objs:
            self.objs[aid] = self._load(self.elems[aid])
        return self.objs[aid]

    def _color(self, elem, name, default=None):
        node = _child(elem, name)
        if node is None:
            if default is None:
                raise SceneFormatError(f"missing <{name}>")
            return tuple(float(x) for x in default)
        if _child(node, "color") is not None and _child(node, "texture") is not None:
            raise SceneFormatError("'color' and 'texture' element cannot be used simultaneously")
        if _child(node, "color") is not None:
            return tuple(float(x) for x in _floats(_child(node, "color"), 3))
        if _child(node, "texture") is not None:
            tex = self.resolve(_child(node, "texture"), "texture")
            return tex
        return tuple(float(x) for x in _floats(node, 3))

    def _load(self, a):
        t = a.get("type")
        if a.tag == "triangle_mesh":
            if t == "raw":
                return _raw_mesh(a)
            if t == "obj":
                p = _child(a, "path")
                if p is None or not p.text:
                    raise SceneFormatError("obj mesh needs <path>")
                path = p.text.strip()
                return load_obj(path if os.path.isabs(path) else os.path.join(self.base_dir, path))
        elif a.tag == "texture":
            if t == "constant":
                return tuple(float(x) for x in _value(a, "color", 3, (1.0, 1.0, 1.0)))
        elif a.tag == "bsdf":
            if t == "diffuse":
                return DiffuseBSDF(self._color(a, "diffuse_reflectance"))
            if t == "mirror":
                return PerfectMirrorBSDF(self._color(a, "specular_reflectance", (1.0, 1.0, 1.0)))
            if t == "plugin.diffusemirror":
                return DiffuseMirrorBSDF(self._color(a, "diffuse_reflectance", (1.0, 1.0, 1.0)))
        elif a.tag == "light":
            if t == "area":
                return AreaLight(tuple(float(x) for x in _value(a, "luminance", 3)))
            if t == "env.const":
                return ConstantEnvironmentLight(tuple(float(x) for x in _value(a, "luminance", 3)))
        elif a.tag == "film":
            if t == "hdr":
                it = _child(a, "imagetype")
                kind = it.text.strip() if it is not None and it.text else "radiancehdr"
                if kind not in ("radiancehdr", "openexr"):
                    raise SceneFormatError(f"invalid image type '{kind}'")
                return HDRBitmapFilm(int(_value(a, "width", 1)[0]), int(_value(a, "height", 1)[0]), image_type=kind)
        elif a.tag == "camera":
            if t == "perspective":
                film = self.resolve(_child(a, "film"), "film")
                if film is None:
                    raise SceneFormatError("camera needs a <film> reference")
                return {"fovy": float(_value(a, "fovy", 1)[0]), "film": film}
        raise SceneFormatError(f"unsupported {a.tag} type '{t}'")


# -------------------------------------------------------------- nodes -----

def _camera_from_view(view: np.ndarray, spec: dict) -> PerspectiveCamera:
    """The camera's view matrix is its node's transform
    (perspectivecamera.cpp:174-183); eye / center / up reproduce it for a
    rigid (look-at) view."""
    inv = np.linalg.inv(view.astype(np.float64))
    eye = inv[:3, 3]
    forward = -view[2, :3].astype(np.float64)
    up = view[1, :3].astype(np.float64)
    return PerspectiveCamera(fovy=spec["fovy"], eye=tuple(eye), center=tuple(eye + forward), up=tuple(up),
                             film=spec["film"])


def _traverse(node, assets, parent, prims: Primitives, ids):
    tnode = _child(node, "transform")
    local = parse_transform(tnode) if tnode is not None else np.eye(4, dtype=F)
    g = _child(node, "global_transform")
    world = parse_transform(g) if g is not None else mat_mul(parent, local)
    cam_el, light_el, mesh_el = _child(node, "camera"), _child(node, "light"), _child(node, "triangle_mesh")
    if cam_el is not None and light_el is not None:
        raise SceneFormatError("'camera' and 'light' elements cannot be used in the same time")
    light = assets.resolve(light_el, "light") if light_el is not None else None
    made = False
    if cam_el is not None and prims.camera is None:
        # A look-at transform under an identity parent gives the camera's
        # position / center / up directly; anything else goes through the matrix.
        direct = tnode is not None and g is None and np.array_equal(parent, np.eye(4, dtype=F))
        look = _child(tnode, "lookat") if direct and _child(tnode, "matrix") is None else None
        spec = assets.resolve(cam_el, "camera")
        if look is not None:
            prims.camera = PerspectiveCamera(fovy=spec["fovy"], eye=tuple(_value(look, "position", 3)),
                                             center=tuple(_value(look, "center", 3)),
                                             up=tuple(_value(look, "up", 3)), film=spec["film"])
        else:
            prims.camera = _camera_from_view(world, spec)
        made = True
    if mesh_el is not None:
        if _child(node, "bsdf") is None:
            raise SceneFormatError("Missing 'bsdf' element")
        mesh = assets.resolve(mesh_el, "triangle_mesh")
        bsdf = assets.resolve(_child(node, "bsdf"), "bsdf")
        if isinstance(light, ConstantEnvironmentLight):
            raise SceneFormatError("an environment light cannot be attached to a mesh")
        identity = np.array_equal(world, np.eye(4, dtype=F))
        prims.add(Primitive(mesh=mesh, bsdf=bsdf, light=light, transform=None if identity else world.copy()))
        made = True
    elif light is not None:
        if not isinstance(light, ConstantEnvironmentLight):
            raise SceneFormatError("an area light needs a triangle mesh")
        prims.environment_light = light
        made = True
    nid = node.get("id")
    if made and nid:
        if nid in ids:
            raise SceneFormatError(f"ID '{nid}' for the node is already used")
        if mesh_el is not None:
            ids[nid] = len(prims.primitives) - 1
    is_leaf = cam_el is not None or light_el is not None or mesh_el is not None
    children = node.findall("node")
    if children and is_leaf:
        raise SceneFormatError("Leaf node cannot have children")
    for c in children:
        _traverse(c, assets, world, prims, ids)


def _config_dict(elem) -> dict:
    """Element tree -> nested dict of child name -> text or dict (attributes
    under '@type' etc.)."""
    out = {}
    if elem is None:
        return out
    for k, v in elem.attrib.items():
        out["@" + k] = v
    for c in elem:
        if len(c) or c.attrib:
            out[c.tag] = _config_dict(c)
            if c.text and c.text.strip():
                out[c.tag]["#text"] = c.text.strip()
        else:
            out[c.tag] = (c.text or "").strip()
    return out


def _num(v, cast):
    try:
        return cast(v)
    except (TypeError, ValueError):
        raise SceneFormatError(f"bad value '{v}'")


def load_scene(source: str, base_dir: Optional[str] = None) -> SceneDocument:
    """Parses a scene document from a file path or an XML string. Relative
    asset paths resolve against the file's directory (or base_dir)."""
    if source.lstrip().startswith("<"):
        root = ET.fromstring(source)
        base = base_dir or os.getcwd()
    else:
        root = ET.parse(source).getroot()
        base = base_dir or os.path.dirname(os.path.abspath(source))
    if root.tag in ROOT_NAMES:
        top = root
    elif root.tag == "scene":
        top = ET.Element("lightmetrica")
        top.append(root)
    else:
        raise SceneFormatError(f"unknown root element <{root.tag}>")
    for required in ("scene",):
        if top.find(required) is None:
            raise SceneFormatError(f"missing <{required}>")
    assets = _Assets(top.find("assets"), base)
    scene_el = top.find("scene")
    prims = Primitives()
    ids: Dict[str, int] = {}
    root_el = scene_el.find("root")
    if root_el is not None:
        _traverse(root_el, assets, np.eye(4, dtype=F), prims, ids)
    doc = SceneDocument(primitives=prims, scene_type=scene_el.get("type", "bvh"), ids=ids)
    if prims.camera is not None and prims.camera.film is not None:
        doc.image_type = prims.camera.film.image_type
    r = top.find("renderer")
    if r is not None:
        doc.renderer_type = r.get("type", "pt")
        d = _config_dict(r)
        cfg = {}
        if "rr_depth" in d:
            cfg["rr_depth"] = _num(d["rr_depth"], int)
        if "max_path_vertices" in d:
            cfg["max_path_vertices"] = _num(d["max_path_vertices"], int)
        if isinstance(d.get("sampler"), dict):
            s = d["sampler"]
            cfg["sampler"] = {"type": s.get("@type", "random")}
            if "rng_seed" in s:
                cfg["sampler"]["rng_seed"] = _num(s["rng_seed"], int)
        doc.renderer_config = cfg
    s = top.find("render_scheduler")
    if s is not None:
        doc.scheduler_type = s.get("type", "mt")
        d = _config_dict(s)
        cfg = {}
        for key, cast in (("num_samples", int), ("num_threads", int), ("samples_per_block", int),
                          ("samples_per_mpi_task", int), ("progress_image_interval", float)):
            if key in d:
                cfg[key] = _num(d[key], cast)
        doc.scheduler_config = cfg
    return doc


# ------------------------------------------------------------- export -----

def _fmt(v) -> str:
    return " ".join(repr(float(x)) for x in np.asarray(v, np.float64).reshape(-1))


def save_scene(prims: Primitives, path: Optional[str] = None, scene_type: str = "bvh", renderer: Optional[dict] = None,
               scheduler: Optional[dict] = None) -> str:
    """Writes Primitives as a scene document that load_scene (and the
    reference) reads back: raw meshes, one BSDF / light asset per primitive,
    nodes with column-major matrices. Returns the XML text (also written to
    `path` when given)."""
    L = ET.Element("lightmetrica", version="1.0.dev")
    A = ET.SubElement(L, "assets")
    groups = {g: ET.SubElement(A, g) for g in ("triangle_meshes", "bsdfs", "films", "cameras", "lights")}
    scene = ET.SubElement(L, "scene", type=scene_type)
    root = ET.SubElement(scene, "root")
    light_ids = {}
    if prims.camera is not None:
        cam, film = prims.camera, prims.camera.film
        f = ET.SubElement(groups["films"], "film", id="film", type="hdr")
        ET.SubElement(f, "width").text = str(film.width)
        ET.SubElement(f, "height").text = str(film.height)
        ET.SubElement(f, "imagetype").text = film.image_type
        c = ET.SubElement(groups["cameras"], "camera", id="camera", type="perspective")
        ET.SubElement(c, "film", ref="film")
        ET.SubElement(c, "fovy").text = repr(float(cam.fovy))
        n = ET.SubElement(root, "node", id="camera")
        la = ET.SubElement(ET.SubElement(n, "transform"), "lookat")
        ET.SubElement(la, "position").text = _fmt(cam.eye)
        ET.SubElement(la, "center").text = _fmt(cam.center)
        ET.SubElement(la, "up").text = _fmt(cam.up)
        ET.SubElement(n, "camera", ref="camera")
    for i, p in enumerate(prims.primitives):
        if p.mesh is None:
            continue
        m = ET.SubElement(groups["triangle_meshes"], "triangle_mesh", id=f"mesh{i}", type="raw")
        ET.SubElement(m, "positions").text = _fmt(p.mesh.positions)
        nrm = p.mesh.normals
        if nrm is None:                         # raw meshes require normals: face normals
            P = p.mesh.positions.astype(np.float64)
            nrm = np.zeros_like(P)
            for f3 in p.mesh.faces:
                a, b, c = P[f3]
                nrm[f3] = np.cross(b - a, c - a)
            ln = np.linalg.norm(nrm, axis=1, keepdims=True)
            nrm = nrm / np.where(ln > 0, ln, 1.0)
        ET.SubElement(m, "normals").text = _fmt(nrm)
        if p.mesh.texcoords is not None:
            ET.SubElement(m, "texcoords").text = _fmt(p.mesh.texcoords)
        ET.SubElement(m, "faces").text = " ".join(str(int(x)) for x in p.mesh.faces.reshape(-1))
        b = p.bsdf
        kind = {DiffuseBSDF: ("diffuse", "diffuse_reflectance"), PerfectMirrorBSDF: ("mirror", "specular_reflectance"),
                DiffuseMirrorBSDF: ("plugin.diffusemirror", "diffuse_reflectance")}[type(b)]
        be = ET.SubElement(groups["bsdfs"], "bsdf", id=f"bsdf{i}", type=kind[0])
        if kind[0] == "diffuse":
            ET.SubElement(ET.SubElement(be, kind[1]), "color").text = _fmt(np.broadcast_to(b.reflectance, (3,)))
        else:
            ET.SubElement(be, kind[1]).text = _fmt(np.broadcast_to(b.reflectance, (3,)))
        n = ET.SubElement(root, "node", id=f"prim{i}")
        if p.transform is not None:
            ET.SubElement(ET.SubElement(n, "transform"), "matrix").text = _fmt(np.asarray(p.transform, F).T)
        ET.SubElement(n, "triangle_mesh", ref=f"mesh{i}")
        ET.SubElement(n, "bsdf", ref=f"bsdf{i}")
        if p.light is not None:
            if id(p.light) not in light_ids:
                lid = f"light{len(light_ids)}"
                light_ids[id(p.light)] = lid
                le = ET.SubElement(groups["lights"], "light", id=lid, type="area")
                ET.SubElement(le, "luminance").text = _fmt(np.broadcast_to(p.light.luminance, (3,)))
            ET.SubElement(n, "light", ref=light_ids[id(p.light)])
    if prims.environment_light is not None:
        le = ET.SubElement(groups["lights"], "light", id="env", type="env.const")
        ET.SubElement(le, "luminance").text = _fmt(np.broadcast_to(prims.environment_light.luminance, (3,)))
        ET.SubElement(ET.SubElement(root, "node", id="environment"), "light", ref="env")
    if renderer:
        r = ET.SubElement(L, "renderer", type=renderer.get("type", "pt"))
        for k in ("rr_depth", "max_path_vertices"):
            if k in renderer:
                ET.SubElement(r, k).text = str(renderer[k])
        if "sampler" in renderer:
            se = ET.SubElement(r, "sampler", type="random")
            if "rng_seed" in renderer["sampler"]:
                ET.SubElement(se, "rng_seed").text = str(renderer["sampler"]["rng_seed"])
    if scheduler:
        s = ET.SubElement(L, "render_scheduler", type=scheduler.get("type", "mt"))
        for k, v in scheduler.items():
            if k != "type":
                ET.SubElement(s, k).text = str(v)
    text = ET.tostring(L, encoding="unicode")
    if path:
        with open(path, "w") as f:
            f.write(text)
    return text
