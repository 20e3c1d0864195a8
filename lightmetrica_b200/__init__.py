"""lightmetrica_b200 — B200-native scene accelerator and path tracer behind
lightmetrica's component interfaces.

The Python classes mirror the reference's component API for this path
(names, configuration keys and failure behaviour) so that code written
against lightmetrica's Scene / Renderer / RenderProcessScheduler reads the
same:

    scene = create_scene("bvh")            # ComponentFactory::Create<Scene>("bvh")
    scene.load(primitives)                 # Scene::Load(Primitives*)
    scene.configure({})                    # Scene::Configure(const ConfigNode&)
    scene.build()                          # Scene::Build()
    hits = scene.intersect_batch(rays)     # Scene::Intersect for a ray batch

    renderer = create_renderer("pt")       # "pt", "pt.direct", "pt.mis"
    renderer.configure({"rr_depth": 1, "max_path_vertices": 9, "sampler": {"rng_seed": 1}})
    sched = create_scheduler("mt")         # whole sample budget, one GPU call
    sched.configure({"num_samples": W * H * spp})
    sched.render(renderer, scene)          # film in scene.main_camera().film

All compute runs in lightmetrica_b200/_lib/liblmgpu.so (hand-written sm_100a
CUDA); there is no CPU fallback.
"""
from .scene import (AreaLight, ConstantEnvironmentLight, DiffuseBSDF, DiffuseMirrorBSDF, HDRBitmapFilm,
                    PerfectMirrorBSDF, PerspectiveCamera, Primitive, Primitives, Scene, TriangleMesh,
                    create_scene)
from .render import RenderProcessScheduler, Renderer, create_renderer, create_scheduler, release_render_memory
from . import native

__all__ = ["AreaLight", "ConstantEnvironmentLight", "DiffuseBSDF", "DiffuseMirrorBSDF", "HDRBitmapFilm",
           "PerfectMirrorBSDF", "PerspectiveCamera", "Primitive", "Primitives", "Scene", "TriangleMesh",
           "create_scene", "Renderer", "RenderProcessScheduler", "create_renderer", "create_scheduler",
           "release_render_memory", "native"]
