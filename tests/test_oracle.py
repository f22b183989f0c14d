"""CPU tests: the C oracle is pinned against the reference's own outputs
(golden fixtures made by tests/golden/make_golden.py from oracle/_ref) and
against the known-answer values of the reference's unit tests."""
import os

import numpy as np
import pytest

import oracle_lib as orc
from symprop_b200 import synth

GOLD = os.path.join(os.path.dirname(__file__), "golden")


def test_packed_sizes_known_answers():
    # reference tests/test_symtensor.cpp:9-24
    L = orc.olib()
    assert L.orc_symtens_size(3, 2) == 6
    assert L.orc_symtens_size(4, 2) == 10
    assert L.orc_symtens_size(3, 3) == 10
    assert L.orc_symtens_size(5, 5) == 126
    # configs: m = C(r+N-2, N-1)
    assert L.orc_symtens_size(8, 4) == 330
    assert L.orc_symtens_size(16, 3) == 816
    assert L.orc_symtens_size(10, 5) == 2002
    assert L.orc_symtens_size(16, 4) == 3876


def test_outer_product_known_answers():
    # reference tests/test_symtensor.cpp:26-58: order-2/3 outer products are
    # products of vector entries in lexicographic packed order
    L = orc.olib()
    v1 = np.array([1.0, 2, 3]); v2 = np.array([4.0, 5, 6]); v3 = np.array([7.0, 8, 9])
    s2 = np.zeros(6)
    L.orc_sym_outer_prod(orc.p(s2), orc.p(v1), orc.p(v2), 3, 2)
    s3 = np.zeros(10)
    L.orc_sym_outer_prod(orc.p(s3), orc.p(s2), orc.p(v3), 3, 3)
    idx3 = orc.packed_indices(3, 3)
    cnt = 0
    for i in range(3):
        for j in range(i, 3):
            for k in range(j, 3):
                assert s3[cnt] == v1[i] * v2[j] * v3[k]
                assert tuple(idx3[cnt]) == (i, j, k)
                q = np.array([i, j, k], np.uint32)
                assert L.orc_packed_offset(orc.p(q), 3, 3) == cnt
                cnt += 1


def test_coefficients_are_permutation_counts():
    c = orc.symtens_coeff(3, 3)
    idx = orc.packed_indices(3, 3)
    from math import factorial
    for q, cq in zip(idx, c):
        _, counts = np.unique(q, return_counts=True)
        assert cq == factorial(3) // np.prod([factorial(x) for x in counts])
    assert c.sum() == 3 ** 3


def test_tree_matches_reference_dumps():
    g = np.load(os.path.join(GOLD, "trees.npz"))
    ncase = len([k for k in g.files if k.endswith("_meta")])
    assert ncase >= 6
    for ci in range(ncase):
        order, n, nnz, seed = g[f"c{ci}_meta"]
        tr = orc.tree(int(order), int(n), g[f"c{ci}_inds"], g[f"c{ci}_vals"])
        for l in range(int(order) - 1):
            np.testing.assert_array_equal(tr["level_idx"][l], g[f"c{ci}_idx{l}"])
            np.testing.assert_array_equal(tr["level_ptr"][l], g[f"c{ci}_ptr{l}"])
            if l >= 1:
                np.testing.assert_array_equal(tr["dep_list"][l], g[f"c{ci}_dep{l}"])
        np.testing.assert_array_equal(tr["rem"], g[f"c{ci}_rem"])
        np.testing.assert_array_equal(tr["val"], g[f"c{ci}_val"])
        assert orc.norm(int(order), g[f"c{ci}_inds"], g[f"c{ci}_vals"]) == pytest.approx(
            float(g[f"c{ci}_norm"][0]), rel=1e-14)


def test_s3ttmc_matches_reference_outputs():
    g = np.load(os.path.join(GOLD, "s3ttmc.npz"))
    ncase = len([k for k in g.files if k.endswith("_meta")])
    for ci in range(ncase):
        order, n, nnz, seed, R = (int(x) for x in g[f"c{ci}_meta"])
        for packed, key in ((True, "Yp"), (False, "Yu")):
            Y = orc.s3ttmc(order, n, g[f"c{ci}_inds"], g[f"c{ci}_vals"], g[f"c{ci}_U"], R, packed)
            ref = g[f"c{ci}_{key}"]
            err = np.linalg.norm(Y - ref) / np.linalg.norm(ref)
            assert err < 1e-13, (ci, key, err)


def test_generator_is_deterministic():
    a = synth.zipf_tuples(4, 100, 500, 1.1, 3)
    b = synth.zipf_tuples(4, 100, 500, 1.1, 3)
    np.testing.assert_array_equal(a, b)
    assert np.all(np.diff(a.astype(np.int64), axis=1) >= 0)
    assert len(np.unique(a, axis=0)) == 500
    assert a.min() >= 1 and a.max() <= 100


def test_golden_vectors_reproducible_from_generator():
    g = np.load(os.path.join(GOLD, "s3ttmc.npz"))
    order, n, nnz, seed, R = (int(x) for x in g["c0_meta"])
    np.testing.assert_array_equal(synth.zipf_tuples(order, n, nnz, 1.2, seed), g["c0_inds"])
