"""Scene ingestion (lightmetrica_b200.sceneio) on CPU.

Pinned by the reference's own Primitives tests (test.primitives.cpp: the
scene literals are read from tests/golden/ref_scene_literals.json, made by
gen_golden.py; the expected values restate that file's assertions) and by
its BPT test scene (test.bpt.mis.cpp), plus our own documents for the error
paths, obj meshes and the exporter's round trip.
"""
import json
import os

import numpy as np
import pytest

from lightmetrica_b200 import scenes
from lightmetrica_b200.scene import DiffuseBSDF, PerfectMirrorBSDF
from lightmetrica_b200.sceneio import SceneFormatError, load_obj, load_scene, look_at, mat_mul, rotate, save_scene

HERE = os.path.dirname(os.path.abspath(__file__))
LITERALS = json.load(open(os.path.join(HERE, "golden", "ref_scene_literals.json")))

# Stand-ins for the reference test's StubTriangleMesh / StubBSDF assets.
STUB_ASSETS = """
<assets>
  <triangle_meshes>
    <triangle_mesh id="mesh1" type="raw">
      <positions>0 0 0  1 0 0  0 1 0</positions><normals>0 0 1  0 0 1  0 0 1</normals><faces>0 1 2</faces>
    </triangle_mesh>
    <triangle_mesh id="mesh2" type="raw">
      <positions>0 0 1  1 0 1  0 1 1</positions><normals>0 0 1  0 0 1  0 0 1</normals><faces>0 1 2</faces>
    </triangle_mesh>
  </triangle_meshes>
  <bsdfs>
    <bsdf id="bsdf1" type="diffuse"><diffuse_reflectance><color>0.5 0.5 0.5</color></diffuse_reflectance></bsdf>
    <bsdf id="bsdf2" type="mirror"/>
  </bsdfs>
</assets>"""


def with_stubs(literal):
    return f"<lightmetrica version='1.0.dev'>{STUB_ASSETS}{literal}</lightmetrica>"


def test_reference_primitives_load():
    """PrimitivesTest.Load: two nodes by id, identity transforms."""
    doc = load_scene(with_stubs(LITERALS["test.primitives.cpp:SceneNode_Success"]))
    assert doc.scene_type == "stub"
    assert set(doc.ids) == {"node1", "node2"}
    p1, p2 = (doc.primitives.primitives[doc.ids[k]] for k in ("node1", "node2"))
    assert p1.transform is None and p2.transform is None       # identity
    assert isinstance(p1.bsdf, DiffuseBSDF) and isinstance(p2.bsdf, PerfectMirrorBSDF)
    np.testing.assert_array_equal(p2.mesh.positions[:, 2], 1.0)


def test_reference_transform_by_matrix():
    """PrimitivesTest.Load_WithTransformByMatrix: root translation (1, 2, 3)
    times the node's uniform scale 2 (column-major matrices)."""
    doc = load_scene(with_stubs(LITERALS["test.primitives.cpp:SceneNode_Success_WithTransformByMatrix"]))
    t = doc.primitives.primitives[doc.ids["node1"]].transform
    expected = np.array([[2, 0, 0, 1], [0, 2, 0, 2], [0, 0, 2, 3], [0, 0, 0, 1]], np.float32)
    np.testing.assert_allclose(t, expected, atol=1e-6)


def test_reference_transform_translate_rotate_scale():
    """PrimitivesTest.Load_WithTransform: T(1,1,1) R(45 deg, y) S(2) maps
    (1, 1, 1, 1) to (2 sqrt 2 + 1, 3, 1, 1)."""
    doc = load_scene(with_stubs(LITERALS["test.primitives.cpp:SceneNode_Success_WithTransform"]))
    t = doc.primitives.primitives[doc.ids["node1"]].transform
    np.testing.assert_allclose(t @ np.ones(4, np.float32), [2 * np.sqrt(2) + 1, 3, 1, 1], atol=1e-5)


def test_reference_bpt_scene_document():
    """The reference BPT test's scene: a look-at camera, a rotated and
    translated diffuse quad, and an area-light quad."""
    doc = load_scene(f"<lightmetrica version='1.0.dev'>{LITERALS['test.bpt.mis.cpp:SceneFile']}</lightmetrica>")
    P = doc.primitives
    assert doc.scene_type == "qbvh"
    cam = P.camera
    np.testing.assert_allclose(cam.eye, (0, 0.1, 0.3))
    np.testing.assert_allclose(cam.center, (0, 0.1, 0))
    assert cam.fovy == 45 and cam.film.width == 500 and cam.film.image_type == "radiancehdr"
    assert len(P.primitives) == 2
    wall, light = P.primitives
    assert wall.light is None and light.light is not None
    np.testing.assert_allclose(light.light.luminance, (2, 2, 2))
    np.testing.assert_allclose(wall.bsdf.reflectance, (0.9, 0.9, 0.9), rtol=1e-6)
    # The wall: translate (0, 0.1, -0.1) after a -90 degree turn about x:
    # the quad's corner (-0.1, 0, -0.1) lands at (-0.1, 0.1 - 0.1, -0.1).
    w = wall.transform @ np.array([-0.1, 0, -0.1, 1], np.float32)
    np.testing.assert_allclose(w[:3], [-0.1, 0.0, -0.1], atol=1e-6)
    li = light.transform @ np.array([0.1, 0, 0.1, 1], np.float32)
    np.testing.assert_allclose(li[:3], [0.1, 0.2, 0.1], atol=1e-7)


def test_float32_transform_math():
    r = rotate(90.0, (0, 0, 1))
    np.testing.assert_allclose(r[:3, :3] @ [1, 0, 0], [0, 1, 0], atol=1e-7)
    v = look_at((0, 0, 5), (0, 0, 0), (0, 1, 0))
    np.testing.assert_allclose(v @ [0, 0, 0, 1], [0, 0, -5, 1], atol=1e-6)
    a = np.arange(16, dtype=np.float32).reshape(4, 4)
    np.testing.assert_allclose(mat_mul(a, np.eye(4, dtype=np.float32)), a)
    np.testing.assert_allclose(mat_mul(a, a), a.astype(np.float64) @ a, rtol=1e-6)


def _doc(nodes, assets=STUB_ASSETS):
    return f"<lightmetrica>{assets}<scene type='bvh'><root>{nodes}</root></scene></lightmetrica>"


@pytest.mark.parametrize("nodes,msg", [
    ("<node><triangle_mesh ref='mesh1'/></node>", "bsdf"),
    ("<node><triangle_mesh ref='nope'/><bsdf ref='bsdf1'/></node>", "unknown asset"),
    ("<node><triangle_mesh ref='bsdf1'/><bsdf ref='bsdf1'/></node>", "expected"),
    ("<node id='a'><triangle_mesh ref='mesh1'/><bsdf ref='bsdf1'/></node>"
     "<node id='a'><triangle_mesh ref='mesh2'/><bsdf ref='bsdf1'/></node>", "already used"),
    ("<node><triangle_mesh ref='mesh1'/><bsdf ref='bsdf1'/><node/></node>", "Leaf node"),
])
def test_scene_errors(nodes, msg):
    with pytest.raises(SceneFormatError, match=msg):
        load_scene(_doc(nodes))


def test_asset_errors():
    bad_mesh = "<assets><triangle_meshes><triangle_mesh id='m' type='raw'><positions>0 0 0</positions>" \
               "<faces>0 0 0</faces></triangle_mesh></triangle_meshes><bsdfs><bsdf id='b' type='diffuse'>" \
               "<diffuse_reflectance><color>1 1 1</color></diffuse_reflectance></bsdf></bsdfs></assets>"
    with pytest.raises(SceneFormatError, match="normals"):
        load_scene(_doc("<node><triangle_mesh ref='m'/><bsdf ref='b'/></node>", bad_mesh))
    oob = bad_mesh.replace("<faces>0 0 0</faces>", "<faces>0 1 2</faces>").replace(
        "<positions>0 0 0</positions>", "<positions>0 0 0</positions><normals>0 0 1</normals>")
    with pytest.raises(SceneFormatError, match="out of range"):
        load_scene(_doc("<node><triangle_mesh ref='m'/><bsdf ref='b'/></node>", oob))
    dup = "<assets><bsdfs><bsdf id='b' type='mirror'/><bsdf id='b' type='mirror'/></bsdfs></assets>"
    with pytest.raises(SceneFormatError, match="already registered"):
        load_scene(_doc("", dup))
    with pytest.raises(SceneFormatError, match="root element"):
        load_scene("<other/>")


def test_environment_light_and_camera_matrix():
    assets = STUB_ASSETS.replace("</assets>", """
      <lights><light id='env' type='env.const'><luminance>0.5 0.5 0.5</luminance></light></lights>
      <films><film id='f' type='hdr'><width>8</width><height>4</height><imagetype>openexr</imagetype></film></films>
      <cameras><camera id='c' type='perspective'><film ref='f'/><fovy>30</fovy></camera></cameras>
    </assets>""")
    view = look_at((1, 2, 3), (0, 0, 0), (0, 1, 0))
    mat = " ".join(str(float(x)) for x in view.T.reshape(-1))
    doc = load_scene(_doc(f"<node><light ref='env'/></node><node><transform><matrix>{mat}</matrix></transform>"
                          "<camera ref='c'/></node>", assets))
    P = doc.primitives
    np.testing.assert_allclose(P.environment_light.luminance, (0.5, 0.5, 0.5))
    np.testing.assert_allclose(P.camera.eye, (1, 2, 3), atol=1e-5)
    d = np.asarray(P.camera.center) - np.asarray(P.camera.eye)
    np.testing.assert_allclose(d / np.linalg.norm(d), -np.array([1, 2, 3]) / np.sqrt(14), atol=1e-6)
    assert doc.image_type == "openexr"


def test_obj_meshes(tmp_path):
    path = tmp_path / "m.obj"
    path.write_text("# quad with normals and uvs, then a triangle without normals\n"
                    "v 0 0 0\nv 1 0 0\nv 1 1 0\nv 0 1 0\nv 0 0 1\n"
                    "vt 0 0\nvt 1 0\nvt 1 1\nvt 0 1\n"
                    "vn 0 0 1\n"
                    "f 1/1/1 2/2/1 3/3/1 4/4/1\n"
                    "f 1/1 2/2 -1/1\n")
    m = load_obj(str(path))
    assert m.faces.shape == (3, 3)
    # the quad's 4 corners are shared; the normal-less triangle gets 3 own vertices
    assert m.positions.shape[0] == 7
    np.testing.assert_allclose(m.normals[:4], [[0, 0, 1]] * 4)
    a, b, c = (m.positions[i] for i in m.faces[2])
    n = np.cross(b - a, c - a)
    np.testing.assert_allclose(m.normals[m.faces[2][0]], n / np.linalg.norm(n), atol=1e-6)
    assert m.texcoords is not None
    doc_text = _doc("<node><triangle_mesh ref='o'/><bsdf ref='bsdf1'/></node>",
                    STUB_ASSETS.replace("</triangle_meshes>",
                                        "<triangle_mesh id='o' type='obj'><path>m.obj</path></triangle_mesh>"
                                        "</triangle_meshes>"))
    scene_file = tmp_path / "s.xml"
    scene_file.write_text(doc_text)
    assert load_scene(str(scene_file)).primitives.primitives[0].mesh.faces.shape == (3, 3)


def test_export_round_trip():
    for variant in ("classic", "mixed"):
        P = scenes.cornell_box(32, 24, variant=variant)
        text = save_scene(P, renderer={"type": "pt.mis", "rr_depth": 3, "max_path_vertices": 9,
                                       "sampler": {"rng_seed": 7}},
                          scheduler={"type": "mt", "num_samples": 1000, "progress_image_interval": 2.5})
        doc = load_scene(text)
        Q = doc.primitives
        assert doc.renderer_type == "pt.mis" and doc.renderer_config["sampler"]["rng_seed"] == 7
        assert doc.scheduler_config == {"num_samples": 1000, "progress_image_interval": 2.5}
        assert len(Q.primitives) == len(P.primitives)
        for a, b in zip(P.primitives, Q.primitives):
            np.testing.assert_array_equal(a.mesh.positions, b.mesh.positions)
            np.testing.assert_array_equal(a.mesh.faces, b.mesh.faces)
            assert type(a.bsdf) is type(b.bsdf)
            assert (a.light is None) == (b.light is None)
        assert (P.environment_light is None) == (Q.environment_light is None)
        np.testing.assert_allclose(Q.camera.eye, P.camera.eye)
        assert (Q.camera.film.width, Q.camera.film.height) == (32, 24)
