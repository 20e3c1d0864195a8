"""The oracle (C restatement) against golden vectors produced by the
reference's own code (tests/golden/gen_golden.py)."""
import os

import numpy as np
import pytest

import oracle


def _load(golden_dir, name):
    return np.load(os.path.join(golden_dir, name))


@pytest.mark.parametrize("name", ["intersect_simple.npz", "intersect_simple2.npz", "consistency_random.npz",
                                  "soup_duplicates.npz"])
@pytest.mark.parametrize("kind", ["bvh", "naive"])
def test_oracle_ids_and_t_match_reference(golden_dir, name, kind):
    d = _load(golden_dir, name)
    s = oracle.OracleScene(d["positions"], d["faces"], kind)
    r = s.intersect(d["rays"])
    np.testing.assert_array_equal(r["tri_id"], d[f"{kind}_tri_id"])
    hit = r["tri_id"] >= 0
    np.testing.assert_array_equal(r["t"][hit], d[f"{kind}_t"][hit])


def test_oracle_soup_small_bit_exact(golden_dir):
    d = _load(golden_dir, "soup_small.npz")
    s = oracle.OracleScene(d["positions"], d["faces"], "bvh")
    r = s.intersect(d["rays"])
    np.testing.assert_array_equal(r["tri_id"], d["bvh_tri_id"])
    hit = r["tri_id"] >= 0
    assert hit.sum() > 1000
    for k in ("t", "u", "v"):
        np.testing.assert_array_equal(r[k][hit], d[f"bvh_{k}"][hit])


def test_oracle_simple_known_answers(golden_dir):
    """Intersect_Simple's geometric known answers (test.scene.intersection.cpp:117-151):
    every ray from (0,0,1) towards (x,y,0) hits the z=0 plane at t = |(x,y,-1)|."""
    d = _load(golden_dir, "intersect_simple.npz")
    s = oracle.OracleScene(d["positions"], d["faces"], "bvh")
    r = s.intersect(d["rays"])
    assert (r["tri_id"] >= 0).all() and (r["tri_id"] <= 1).all()
    rays = d["rays"].astype(np.float64)
    p = rays[:, 0:3] + rays[:, 3:6] * r["t"][:, None]
    np.testing.assert_allclose(p[:, 2], 0.0, atol=1e-3)


def test_oracle_counts_root_test_on_miss():
    pos = np.array([[0, 0, 0], [1, 0, 0], [0, 1, 0]], np.float32)
    s = oracle.OracleScene(pos, np.array([[0, 1, 2]], np.uint32), "bvh")
    rays = np.array([[5, 5, 5, 1, 0, 0, 0, 3e38]], np.float32)
    r = s.intersect(rays)
    assert r["tri_id"][0] == -1 and r["node_tests"][0] == 1 and r["tri_tests"][0] == 0
