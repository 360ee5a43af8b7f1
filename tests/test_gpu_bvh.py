"""GPU binned-SAH builder: structure of the binary tree and its SAH cost
against the reference builder (leaf size 1 in both)."""
import numpy as np
import pytest

import oracle
from nectarrender_b200 import capi, scenes

pytestmark = pytest.mark.gpu


def check_tree(nodes, order, n_prims):
    left = nodes[:, 6].view(np.int32)
    right = nodes[:, 7].view(np.int32)
    lo, hi = nodes[:, 0:3], nodes[:, 3:6]
    leaves = right <= 0
    inner = ~leaves
    assert leaves.sum() == n_prims and inner.sum() == n_prims - 1
    assert np.all(-right[leaves] == 1)                   # one primitive per leaf
    starts = left[leaves]
    assert sorted(starts.tolist()) == list(range(n_prims))
    assert sorted(order.tolist()) == list(range(n_prims))
    for c in (left[inner], right[inner]):
        assert np.all(lo[c] >= lo[inner]) and np.all(hi[c] <= hi[inner])


@pytest.mark.parametrize("levels", [1, 4, 6])
def test_binary_tree_and_sah(levels):
    spec = scenes.mesh_stress(levels=levels, res_h=8, res_w=8, spp=1, n_spheres=4,
                              hdri_size=(16, 8), scene_seed=4)
    sc = capi.Scene(spec)
    nodes, order = sc.binary_bvh(0)
    n = 20 * 4 ** levels
    check_tree(nodes, order[:n], n)
    ref_sah, ref_nodes = oracle.Oracle().mesh_sah(spec)
    assert ref_nodes == 2 * n - 1
    assert sc.stats()["sah_cost_binary"] <= 1.02 * ref_sah


def test_full_size_mesh_sah():
    spec = scenes.mesh_stress()
    sc = capi.Scene(spec)
    st = sc.stats()
    assert st["n_triangles"] == 1310720
    ref_sah, _ = oracle.Oracle().mesh_sah(spec)
    assert st["sah_cost_binary"] <= 1.02 * ref_sah
