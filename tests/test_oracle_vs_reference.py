"""The oracle restatement against the reference's own BVHScene on fresh
seeded inputs (needs oracle/_ref, built from the reference sources)."""
import numpy as np
import pytest

import oracle
from lightmetrica_b200.workloads import random_rays, random_soup

pytestmark = pytest.mark.skipif(not oracle.ref_available("f"), reason="oracle/_ref not built here")


@pytest.mark.parametrize("ntris,sigma,seed", [(20000, 0.01, 1), (5000, 0.2, 7), (300, 0.5, 3)])
def test_oracle_matches_reference_bvh(ntris, sigma, seed):
    pos, faces = random_soup(ntris, seed=seed, sigma=sigma)
    rays = random_rays(20000, seed=seed + 100)
    o = oracle.OracleScene(pos, faces, "bvh").intersect(rays)
    r = oracle.RefScene(pos, faces, "bvh").intersect(rays, threads=4)
    np.testing.assert_array_equal(o["tri_id"], r["tri_id"])
    hit = o["tri_id"] >= 0
    np.testing.assert_array_equal(o["t"][hit], r["t"][hit])


def test_reference_qbvh_agrees_on_hit_or_miss():
    pos, faces = random_soup(5000, seed=5, sigma=0.2)
    rays = random_rays(5000, seed=6)
    a = oracle.RefScene(pos, faces, "bvh").intersect(rays)
    b = oracle.RefScene(pos, faces, "qbvh").intersect(rays)
    np.testing.assert_array_equal(a["tri_id"] >= 0, b["tri_id"] >= 0)
