"""The product's host BVH builder (liblmgpu.so, no GPU needed) against the
oracle: same leaf triangle order (bvhTriIndices), node/leaf counts, depth
and bounds as the restatement of scene.bvh.cpp:270-388."""
import ctypes

import numpy as np
import pytest

import oracle
from lightmetrica_b200 import native
from lightmetrica_b200.scene import Scene, soup_primitives
from lightmetrica_b200.workloads import random_soup


def host_build(pos, faces, layout="bvh", threads=0):
    sc = Scene(layout)
    sc.load(soup_primitives(pos, faces))
    sc.configure({"build_threads": threads})
    desc, keep = sc._describe()
    info = native.SceneInfo()
    n = faces.shape[0]
    order = np.zeros(max(1, n), np.int32)
    native.check(native.lib().lmgpu_scene_build_host(ctypes.byref(desc), ctypes.byref(info), order.ctypes.data, n))
    return info, order[:n]


@pytest.mark.parametrize("ntris,sigma,seed,threads", [(20000, 0.01, 1, 0), (20000, 0.01, 1, 1), (3000, 0.3, 2, 3),
                                                     (1, 0.1, 3, 0), (2, 0.1, 4, 0)])
def test_builder_matches_oracle(ntris, sigma, seed, threads):
    pos, faces = random_soup(ntris, seed=seed, sigma=sigma)
    info, order = host_build(pos, faces, threads=threads)
    o = oracle.OracleScene(pos, faces, "bvh")
    st = o.stats()
    np.testing.assert_array_equal(order, o.tri_order())
    assert info.num_nodes == st["nodes"]
    assert info.num_leaves == st["leaves"]
    assert info.max_depth == st["max_depth"]
    np.testing.assert_array_equal(np.array(info.bounds_min), pos.min(axis=0))
    np.testing.assert_array_equal(np.array(info.bounds_max), pos.max(axis=0))


def test_builder_duplicates_order(golden_dir):
    d = np.load(f"{golden_dir}/soup_duplicates.npz")
    _, order = host_build(d["positions"], d["faces"])
    np.testing.assert_array_equal(order, oracle.OracleScene(d["positions"], d["faces"]).tri_order())


def test_degenerate_centroids_make_one_big_leaf():
    tri = np.array([[0, 0, 0], [1, 0, 0], [0, 1, 0]], np.float32)
    pos = np.tile(tri, (300, 1))
    faces = np.arange(900, dtype=np.uint32).reshape(-1, 3)
    info, order = host_build(pos, faces)
    assert info.num_leaves == 1 and info.num_nodes == 1
    np.testing.assert_array_equal(order, np.arange(300))


def test_empty_scene_builds():
    info, order = host_build(np.zeros((0, 3), np.float32), np.zeros((0, 3), np.uint32))
    assert info.num_triangles == 0 and info.num_nodes == 0


def test_face_index_out_of_range_is_invalid():
    pos = np.zeros((3, 3), np.float32)
    faces = np.array([[0, 1, 7]], np.uint32)
    with pytest.raises(native.LmgpuError) as e:
        host_build(pos, faces)
    assert e.value.code == native.ERR_INVALID


@pytest.mark.parametrize("ntris,sigma,seed", [(20000, 0.01, 1), (5000, 0.2, 5), (1, 0.1, 3), (2, 0.1, 4)])
def test_render_tree_shape(ntris, sigma, seed):
    """The render tree (binned SAH over three axes, leaves of at most 8
    triangles) is a full binary tree over every triangle; the reference tree
    of the same build is unchanged by it."""
    pos, faces = random_soup(ntris, seed=seed, sigma=sigma)
    info, order = host_build(pos, faces)
    assert info.render_tree == native.RENDER_TREE_SAH
    assert info.render_num_nodes == 2 * info.render_num_leaves - 1
    assert info.render_num_leaves >= -(-ntris // 8)
    assert info.render_max_depth <= max(1, ntris)
    np.testing.assert_array_equal(order, oracle.OracleScene(pos, faces, "bvh").tri_order())


def test_render_tree_degenerate_centroids_and_reference_option():
    tri = np.array([[0, 0, 0], [1, 0, 0], [0, 1, 0]], np.float32)
    pos = np.tile(tri, (300, 1))
    faces = np.arange(900, dtype=np.uint32).reshape(-1, 3)
    info, _ = host_build(pos, faces)
    assert info.render_num_leaves == 1 and info.render_num_nodes == 1     # no axis can separate them
    sc = Scene("bvh")
    sc.load(soup_primitives(*random_soup(1000, seed=9, sigma=0.1)))
    sc.configure({"render_tree": "reference"})
    desc, keep = sc._describe()
    inf = native.SceneInfo()
    native.check(native.lib().lmgpu_scene_build_host(ctypes.byref(desc), ctypes.byref(inf), None, 0))
    assert inf.render_tree == native.RENDER_TREE_REFERENCE and inf.render_num_nodes == inf.num_nodes
    with pytest.raises(ValueError):
        sc.configure({"render_tree": "quantised"})
