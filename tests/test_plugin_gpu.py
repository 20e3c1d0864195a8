"""Drop-in proof of the scene slot: the product's lightmetrica plugin
(plugin.gpu.so, built against the reference's headers) loaded into the
reference build through the reference's plugin ABI, then used by the
reference's own code.

* Scene::Intersect through the plugin's "plugin.gpu" scene equals the
  reference BVHScene ("bvh") bit for bit: triangle, t and the whole
  Intersection the reference's StoreIntersectionFromBarycentricCoords fills.
* The reference's own pt.mis renderer and mt scheduler (one thread, its own
  Mersenne-twister sampler) render the identical image over either scene.
* The plugin's renderer ("gpu.pt.mis" ...) and scheduler ("gpu"), created
  and driven by the reference's own component wiring over a "plugin.gpu"
  scene whose BSDFs, lights and camera are the reference's objects: the
  image matches the reference's double-precision pt.mis (the golden images
  and bar of test_render_gpu.py) and the Python path's render of the same
  samples; the renderer also works under the reference's "mt" scheduler,
  and the scheduler hands other renderers to "mt".
"""
import os
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


RELMSE_BAR = 1e-3     # test_render_gpu.py: reference noise leaves this for the estimate


def relmse(x, r):
    return float(np.mean((x - r) ** 2 / (r ** 2 + 1e-2)))


def golden(golden_dir, variant):
    return np.load(os.path.join(golden_dir, f"cornell_{variant}_ref_mis.npz"))["film"]


GOLDEN_KW = dict(rr_depth=3, max_path_vertices=9, seed=7, precision="f")


@pytest.mark.parametrize("variant", ["classic", "mixed"])
def test_plugin_renderer_and_scheduler_match_reference(cuda, golden_dir, variant):
    from lightmetrica_b200 import create_renderer, create_scheduler, create_scene
    oracle.load_plugin()
    prims = scenes.cornell_box(128, 128, variant=variant)
    spp = 16384
    film, _ = oracle.ref_render(prims, "gpu.pt.mis", spp=spp, threads=1, scene_type="plugin.gpu", sched_type="gpu",
                                **GOLDEN_KW)
    assert np.isfinite(film).all()
    assert relmse(film, golden(golden_dir, variant)) <= RELMSE_BAR
    # The Python path with the same parameters draws the same samples: the
    # two differ only where the camera recovered from the reference's view
    # matrix rounds a ray differently.
    s = create_scene("bvh")
    s.load(prims)
    s.configure({})
    s.build()
    r = create_renderer("pt.mis")
    r.configure({"rr_depth": 3, "max_path_vertices": 9, "sampler": {"rng_seed": 7, "sampling": "uniform"}})
    sc = create_scheduler("mt")
    sc.configure({"num_samples": 128 * 128 * spp})
    want = sc.render(r, s)
    s.close()
    assert relmse(film, want) < 1e-5


def test_plugin_renderer_under_reference_mt_scheduler(cuda, golden_dir):
    """Four render processes count their samples and render them on the GPU
    when the reference's mt scheduler collects their films."""
    oracle.load_plugin()
    film, _ = oracle.ref_render(scenes.cornell_box(128, 128), "gpu.pt.mis", spp=16384, threads=4,
                                samples_per_block=1 << 20, scene_type="plugin.gpu", sched_type="mt", **GOLDEN_KW)
    assert relmse(film, golden(golden_dir, "classic")) <= RELMSE_BAR


@pytest.mark.parametrize("renderer", ["gpu.pt", "gpu.pt.direct"])
def test_plugin_pt_and_direct_renderers(cuda, golden_dir, renderer):
    oracle.load_plugin()
    spp = 65536 if renderer == "gpu.pt" else 16384
    film, _ = oracle.ref_render(scenes.cornell_box(128, 128), renderer, spp=spp, threads=1, scene_type="plugin.gpu",
                                sched_type="gpu", **GOLDEN_KW)
    assert relmse(film, golden(golden_dir, "classic")) <= RELMSE_BAR
