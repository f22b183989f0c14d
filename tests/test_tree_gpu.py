"""GPU tests of the device CompressedDTree construction: bit-exact against
the reference's own dumps (golden fixtures) and the C oracle."""
import os

import numpy as np
import pytest

import oracle_lib as orc
from symprop_b200 import synth

GOLD = os.path.join(os.path.dirname(__file__), "golden")
pytestmark = pytest.mark.gpu


def check_equal(tr, ref, order):
    for l in range(order - 1):
        np.testing.assert_array_equal(tr["level_idx"][l], ref["level_idx"][l])
        np.testing.assert_array_equal(tr["level_ptr"][l], ref["level_ptr"][l])
        if l >= 1:
            np.testing.assert_array_equal(tr["dep_list"][l], ref["dep_list"][l])
    np.testing.assert_array_equal(tr["rem"], ref["rem"])
    np.testing.assert_array_equal(tr["val"], ref["val"])


def test_tree_matches_reference_dumps(gpu):
    g = np.load(os.path.join(GOLD, "trees.npz"))
    ncase = len([k for k in g.files if k.endswith("_meta")])
    for ci in range(ncase):
        order, n, nnz, seed = (int(x) for x in g[f"c{ci}_meta"])
        X = gpu.SpSymtensor(n, order, g[f"c{ci}_inds"], g[f"c{ci}_vals"])
        tr = X.tree()
        ref = {"level_idx": [g[f"c{ci}_idx{l}"] for l in range(order - 1)],
               "level_ptr": [g[f"c{ci}_ptr{l}"] for l in range(order - 1)],
               "dep_list": [g[f"c{ci}_dep{l}"] for l in range(order - 1)],
               "rem": g[f"c{ci}_rem"], "val": g[f"c{ci}_val"]}
        check_equal(tr, ref, order)
        assert X.norm() == pytest.approx(float(g[f"c{ci}_norm"][0]), rel=1e-14)


@pytest.mark.parametrize("order,n,nnz,s", [(3, 2000, 50000, 1.1), (4, 100000, 200000, 1.1),
                                           (5, 300, 20000, 1.2), (6, 70000, 30000, 1.0),
                                           (8, 1000, 2000, 1.1)])
def test_tree_matches_oracle_multiword_keys(gpu, order, n, nnz, s):
    # n = 100000 needs 17-bit ids: order-4 leaves use 51-bit keys, order-6 and
    # order-8 keys span two 64-bit words
    t = synth.zipf_tuples(order, n, nnz, s, 40 + order)
    v = synth.uniform_values(nnz, 3)
    X = gpu.SpSymtensor(n, order, t, v)
    check_equal(X.tree(), orc.tree(order, n, t, v), order)
