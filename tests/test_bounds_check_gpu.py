"""The bounds-checked build, liblmgpu_check.so (LMGPU_BOUNDS_CHECK=1).

It checks every tree reference on the device when a scene is built (internal
references below the node count, every leaf's TriRecord run ending inside
the triangle array) and every wavefront queue append against the queue's
capacity; a failed check sets a status word and skips the access, and the
call returns LMGPU_ERR_BOUNDS or LMGPU_ERR_QUEUE_OVERFLOW. Two things are
shown here, each in a child process that loads one library:

- on valid inputs the checked build reports no error and computes what the
  product library computes (bit-exact hits, the same films);
- each check fires and reaches the caller: LMGPU_CHECK_NODE_LIMIT and
  LMGPU_CHECK_QUEUE_LIMIT lower the limits the checks compare with (never
  the buffers), so every access stays inside memory while the check fails,
  and the next call without them succeeds.
"""
import ctypes
import json
import os
import subprocess
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)

from lightmetrica_b200 import native  # noqa: E402

SPP = 16


def _child(case, library, out_path, env_extra=None):
    env = dict(os.environ)
    env["LMGPU_LIBRARY"] = library
    env["PYTHONPATH"] = ROOT + os.pathsep + env.get("PYTHONPATH", "")
    env.update(env_extra or {})
    r = subprocess.run([sys.executable, os.path.abspath(__file__), case, out_path], env=env, cwd=ROOT,
                       capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stdout[-3000:] + r.stderr[-3000:]
    line = [x for x in r.stdout.splitlines() if x.startswith("{")][-1]
    return json.loads(line)


# ---------------------------------------------------------------- child side

def _build(prims, layout="bvh"):
    from lightmetrica_b200 import create_scene
    s = create_scene(layout)
    s.load(prims)
    s.configure({})
    s.build()
    return s


def _renderer(technique="pt.mis", seed=3):
    from lightmetrica_b200 import create_renderer
    r = create_renderer(technique)
    r.configure({"rr_depth": 3, "max_path_vertices": 9, "sampler": {"rng_seed": seed}})
    return r


def _render_device(scene, r, n):
    """lmgpu_render_device into an FP64 device film: (status, film)."""
    import torch
    W, H = scene.main_camera().film.width, scene.main_camera().film.height
    f = torch.zeros(W * H * 3, dtype=torch.float64, device="cuda")
    p = r.params(n, film_fp64=True)
    st = native.RenderStats()
    rc = native.lib().lmgpu_render_device(scene.handle, ctypes.byref(p), ctypes.c_void_p(f.data_ptr()),
                                          ctypes.c_void_p(torch.cuda.current_stream().cuda_stream), ctypes.byref(st))
    torch.cuda.synchronize()
    return rc, f.cpu().numpy()


def _batch_items():
    from lightmetrica_b200 import HDRBitmapFilm, scenes
    items = [(scenes.cornell_box(64, 64), _renderer("pt.mis", 1), 64 * 64 * SPP)]
    for i in range(2):
        d = scenes.batch_scene(i, seed=11)
        d["prims"].camera.film = HDRBitmapFilm(48, 40)
        items.append((d["prims"], _renderer("pt.mis", 5 + i), 48 * 40 * SPP))
    return items


def _batch_films(items, scenes_built):
    import torch
    from lightmetrica_b200.batch import SceneBatch
    b = SceneBatch(scenes_built)
    films = [torch.zeros(p.camera.film.width * p.camera.film.height * 3, dtype=torch.float64, device="cuda")
             for p, _, _ in items]
    b.render_device([r for _, r, _ in items], [n for _, _, n in items], films)
    torch.cuda.synchronize()
    b.close()
    return [f.cpu().numpy() for f in films]


def child_parity(out_path):
    """Hits of a 200k-triangle soup (both exact layouts), a one-scene
    render and a three-scene batch render."""
    from lightmetrica_b200 import scenes
    from lightmetrica_b200.scene import soup_primitives
    from lightmetrica_b200.workloads import random_rays, random_soup
    out = {}
    pos, faces = random_soup(200_000, seed=21)
    rays = random_rays(1 << 20, seed=22)
    for layout in ("bvh", "qbvh"):
        s = _build(soup_primitives(pos, faces), layout)
        h = s.intersect_host(rays)
        out[f"{layout}_tri_id"], out[f"{layout}_t"] = h["tri_id"], h["t"]
        s.close()
    sc = _build(scenes.cornell_box(64, 64, variant="mixed"))
    rc, out["film"] = _render_device(sc, _renderer(), 64 * 64 * SPP)
    native.check(rc)
    sc.close()
    items = _batch_items()
    built = [_build(p) for p, _, _ in items]
    for i, f in enumerate(_batch_films(items, built)):
        out[f"batch_{i}"] = f
    np.savez(out_path, **out)
    print(json.dumps({"library": os.path.basename(native.LIB_PATH)}))


def child_node_limit(out_path):
    """A node limit of 1 fails every tree with more than one node (the
    render tree of the Cornell box has several); without it the
    same scene builds and traces."""
    from lightmetrica_b200 import scenes
    res = {}
    try:
        _build(scenes.cornell_box(32, 32))
        res["limited"] = "built"
    except native.LmgpuError as e:
        res["limited"] = e.code
        res["message"] = str(e)
    del os.environ["LMGPU_CHECK_NODE_LIMIT"]
    sc = _build(scenes.cornell_box(32, 32))
    rc, film = _render_device(sc, _renderer(), 32 * 32 * 4)
    res["after"] = rc
    res["after_film_max"] = float(film.max())
    print(json.dumps(res))


def child_queue_limit(out_path):
    """Queues limited to 1000 slots (the workspace holds 65,536 paths): the
    one-scene render and a batch render report the overflow; the one-scene
    render without the limit succeeds."""
    from lightmetrica_b200 import scenes
    res = {}
    sc = _build(scenes.cornell_box(64, 64))
    res["render"], _ = _render_device(sc, _renderer(), 64 * 64 * SPP)
    res["render_message"] = native.lib().lmgpu_last_error().decode()
    items = _batch_items()
    built = [_build(p) for p, _, _ in items]
    try:
        _batch_films(items, built)
        res["batch"] = 0
    except native.LmgpuError as e:
        res["batch"] = e.code
    del os.environ["LMGPU_CHECK_QUEUE_LIMIT"]
    rc, film = _render_device(sc, _renderer(), 64 * 64 * SPP)
    res["after"] = rc
    res["after_film_max"] = float(film.max())
    print(json.dumps(res))


# ---------------------------------------------------------------- tests

pytestmark = pytest.mark.gpu


def test_checked_build_matches_product_on_valid_inputs(cuda, tmp_path):
    a, b = str(tmp_path / "product.npz"), str(tmp_path / "checked.npz")
    assert _child("parity", native.LIB_PATH, a)["library"] == "liblmgpu.so"
    assert _child("parity", native.CHECK_LIB_PATH, b)["library"] == "liblmgpu_check.so"
    want, got = np.load(a), np.load(b)
    for layout in ("bvh", "qbvh"):
        np.testing.assert_array_equal(got[f"{layout}_tri_id"], want[f"{layout}_tri_id"])
        np.testing.assert_array_equal(got[f"{layout}_t"], want[f"{layout}_t"])
        assert (want[f"{layout}_tri_id"] >= 0).mean() > 0.1
    # Same samples and paths; FP64 films differ only in the order of the
    # film's atomic additions.
    for k in ["film"] + [f"batch_{i}" for i in range(3)]:
        assert want[k].max() > 0
        np.testing.assert_allclose(got[k], want[k], rtol=1e-9, atol=1e-12, err_msg=k)


def test_tree_reference_check_fires_and_recovers(cuda, tmp_path):
    r = _child("node_limit", native.CHECK_LIB_PATH, str(tmp_path / "x"), {"LMGPU_CHECK_NODE_LIMIT": "1"})
    assert r["limited"] == native.ERR_BOUNDS, r
    assert "bounds check" in r["message"]
    assert r["after"] == native.OK and r["after_film_max"] > 0


def test_queue_capacity_check_fires_and_recovers(cuda, tmp_path):
    r = _child("queue_limit", native.CHECK_LIB_PATH, str(tmp_path / "x"), {"LMGPU_CHECK_QUEUE_LIMIT": "1000"})
    assert r["render"] == native.ERR_QUEUE_OVERFLOW, r
    assert "queue" in r["render_message"]
    assert r["batch"] == native.ERR_QUEUE_OVERFLOW, r
    assert r["after"] == native.OK and r["after_film_max"] > 0


def test_product_library_ignores_check_limits(cuda, tmp_path):
    # The unchecked build never reads the limits.
    r = _child("queue_limit_product", native.LIB_PATH, str(tmp_path / "x"), {"LMGPU_CHECK_QUEUE_LIMIT": "1000"})
    assert r["render"] == native.OK and r["batch"] == native.OK, r


def child_queue_limit_product(out_path):
    from lightmetrica_b200 import scenes
    sc = _build(scenes.cornell_box(64, 64))
    res = {"render": _render_device(sc, _renderer(), 64 * 64 * SPP)[0]}
    items = _batch_items()
    built = [_build(p) for p, _, _ in items]
    try:
        _batch_films(items, built)
        res["batch"] = 0
    except native.LmgpuError as e:
        res["batch"] = e.code
    print(json.dumps(res))


if __name__ == "__main__":
    case, out = sys.argv[1], sys.argv[2]
    {"parity": child_parity, "node_limit": child_node_limit, "queue_limit": child_queue_limit,
     "queue_limit_product": child_queue_limit_product}[case](out)
