"""The lightmetrica plugin (lightmetrica_b200/plugin/plugin.gpu.cpp), built
against the reference's headers and its plugin.common.cpp like the
reference's own plugins (oracle/build_plugin.sh), loads into the reference
build through the reference's plugin ABI and registers the "plugin.gpu"
scene, the "gpu.pt", "gpu.pt.direct", "gpu.pt.mis" renderers and the "gpu"
render process scheduler (CPU; building the scene and rendering need a GPU,
see test_plugin_gpu.py)."""
import ctypes

import numpy as np
import pytest

import oracle
from lightmetrica_b200 import scenes

pytestmark = pytest.mark.skipif(not oracle.plugin_available(), reason="reference tree not present: plugin not built")


def test_plugin_exports_the_reference_plugin_abi():
    lib = ctypes.CDLL(oracle.PLUGIN_SO)
    assert hasattr(lib, "LM_Plugin_CreateInstance") and hasattr(lib, "LM_Plugin_CheckRegistered")
    lib.LM_Plugin_CheckRegistered.restype = ctypes.c_bool
    lib.LM_Plugin_CheckRegistered.argtypes = [ctypes.c_char_p, ctypes.c_char_p]
    assert lib.LM_Plugin_CheckRegistered(b"plugin.gpu", b"scene")
    for r in (b"gpu.pt", b"gpu.pt.direct", b"gpu.pt.mis"):
        assert lib.LM_Plugin_CheckRegistered(r, b"renderer")
    assert lib.LM_Plugin_CheckRegistered(b"gpu", b"rendersched")
    assert not lib.LM_Plugin_CheckRegistered(b"plugin.gpu", b"renderer")
    assert not lib.LM_Plugin_CheckRegistered(b"bvh", b"scene")


def test_reference_factory_finds_the_plugin_scene():
    oracle.load_plugin()
    oracle.load_plugin()            # idempotent
    L = oracle.ref("f")
    L.lmref_component_available.restype = ctypes.c_int
    L.lmref_component_available.argtypes = [ctypes.c_char_p, ctypes.c_char_p]
    assert L.lmref_component_available(b"scene", b"plugin.gpu") == 1
    assert L.lmref_component_available(b"scene", b"bvh") == 1
    assert L.lmref_component_available(b"scene", b"plugin.nothing") == 0
    assert L.lmref_component_available(b"renderer", b"gpu.pt.mis") == 1
    assert L.lmref_component_available(b"rendersched", b"gpu") == 1
    assert L.lmref_component_available(b"rendersched", b"mt") == 1


def test_plugin_scheduler_hands_other_renderers_to_mt():
    """The "gpu" scheduler renders a reference renderer through the reference's
    own "mt" scheduler: the identical image (one thread, same seed)."""
    oracle.load_plugin()
    prims = scenes.cornell_box(16, 16, variant="mixed")
    kw = dict(spp=8, rr_depth=3, max_path_vertices=9, seed=5, threads=1, precision="f")
    want, _ = oracle.ref_render(prims, "pt.mis", scene_type="bvh", sched_type="mt", **kw)
    got, _ = oracle.ref_render(prims, "pt.mis", scene_type="bvh", sched_type="gpu", **kw)
    np.testing.assert_array_equal(got, want)


def test_plugin_renderer_needs_the_plugin_scene():
    """A GPU renderer over the reference's own "bvh" scene fails in Preprocess."""
    oracle.load_plugin()
    with pytest.raises(RuntimeError):
        oracle.ref_render(scenes.cornell_box(16, 16), "gpu.pt.mis", spp=4, threads=1, precision="f", scene_type="bvh",
                          sched_type="gpu")
