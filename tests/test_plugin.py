"""The lightmetrica plugin (lightmetrica_b200/plugin/plugin.gpu.cpp), built
against the reference's headers and its plugin.common.cpp like the
reference's own plugins (oracle/build_plugin.sh), loads into the reference
build through the reference's plugin ABI and registers the "plugin.gpu"
scene (CPU; building the scene needs a GPU, see test_plugin_gpu.py)."""
import ctypes

import pytest

import oracle

pytestmark = pytest.mark.skipif(not oracle.plugin_available(), reason="reference tree not present: plugin not built")


def test_plugin_exports_the_reference_plugin_abi():
    lib = ctypes.CDLL(oracle.PLUGIN_SO)
    assert hasattr(lib, "LM_Plugin_CreateInstance") and hasattr(lib, "LM_Plugin_CheckRegistered")
    lib.LM_Plugin_CheckRegistered.restype = ctypes.c_bool
    lib.LM_Plugin_CheckRegistered.argtypes = [ctypes.c_char_p, ctypes.c_char_p]
    assert lib.LM_Plugin_CheckRegistered(b"plugin.gpu", b"scene")
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
