"""Drop-in proof of the scene slot: the product's lightmetrica plugin
(plugin.gpu.so, built against the reference's headers) loaded into the
reference build through the reference's plugin ABI, then used by the
reference's own code.

* Scene::Intersect through the plugin's "plugin.gpu" scene equals the
  reference BVHScene ("bvh") bit for bit: triangle, t and the whole
  Intersection the reference's StoreIntersectionFromBarycentricCoords fills.
* The reference's own pt.mis renderer and mt scheduler (one thread, its own
  Mersenne-twister sampler) render the identical image over either scene.
"""
import numpy as np
import pytest

import oracle
from lightmetrica_b200 import scenes
from lightmetrica_b200.workloads import random_rays, random_soup

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not oracle.plugin_available(), reason="reference tree not present: plugin not built")]


def test_plugin_scene_equals_reference_bvh_bit_for_bit(cuda):
    oracle.load_plugin()
    pos, faces = random_soup(4096, seed=7, sigma=0.1)
    rays = random_rays(4000, seed=8)
    ref = oracle.RefScene(pos, faces, "bvh").intersect(rays, geom=True, threads=1)
    got = oracle.RefScene(pos, faces, "plugin.gpu").intersect(rays, geom=True, threads=4)
    assert (ref["tri_id"] >= 0).sum() > 400
    np.testing.assert_array_equal(got["tri_id"], ref["tri_id"])
    np.testing.assert_array_equal(got["t"], ref["t"])
    for k in ("p", "gn", "sn", "ss", "st", "uv"):
        np.testing.assert_array_equal(got[k], ref[k])


@pytest.mark.parametrize("renderer", ["pt.mis", "pt"])
def test_reference_renderer_over_the_plugin_scene(cuda, renderer):
    oracle.load_plugin()
    prims = scenes.cornell_box(16, 16, variant="mixed")
    kw = dict(spp=8, rr_depth=3, max_path_vertices=9, seed=5, threads=1, precision="f")
    want, _ = oracle.ref_render(prims, renderer, scene_type="bvh", **kw)
    got, _ = oracle.ref_render(prims, renderer, scene_type="plugin.gpu", **kw)
    assert want.max() > 0
    np.testing.assert_array_equal(got, want)
