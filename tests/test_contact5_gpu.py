"""The reference's shipped input, examples/contact-5.tns (order 5, dim 245,
12,704 nonzeros; tests/golden/contact5.npz holds it as the reference's
SymtensLoader reads it), through the three Tucker drivers with the
reference CLI's settings (-r 8 -i 20 -d 0.1 -s 0).  Every iteration's error
must equal the reference's own run (tests/golden/tucker.json, "contact5")
within 1e-8, and the mixed-precision HOOI (n = 245 <= m = 330: the
tensor-core row Gram) must end within 1e-6 of the reference's objective."""
import json
import os

import numpy as np
import pytest

GOLD = os.path.join(os.path.dirname(__file__), "golden")
pytestmark = pytest.mark.gpu


def contact5(sp):
    d = np.load(os.path.join(GOLD, "contact5.npz"))
    return sp.SpSymtensor(int(d["dim"]), int(d["order"]), d["inds"].astype(np.uint32), d["vals"])


@pytest.mark.parametrize("alg", ["HOOI", "HOQRI", "AltHOOI"])
def test_contact5_matches_reference_per_iteration(gpu, alg):
    case = json.load(open(os.path.join(GOLD, "tucker.json")))["contact5"]
    X = contact5(gpu)
    fn = {"HOOI": X.TuckerHOOI, "HOQRI": X.TuckerHOQRI, "AltHOOI": X.TuckerAltHOOI}[alg]
    d = fn(rank=case["rank"], max_iter=case["iters"], delta=case["delta"], seed=0)
    ref = np.array(case["runs"][alg]["error"])
    assert d.iterations == len(ref)
    np.testing.assert_allclose(d.error_trace, ref, atol=1e-8, rtol=0)


def test_contact5_mixed_precision_objective(gpu):
    case = json.load(open(os.path.join(GOLD, "tucker.json")))["contact5"]
    X = contact5(gpu)
    d = X.TuckerHOOI(rank=case["rank"], max_iter=case["iters"], delta=case["delta"], seed=0,
                     precision=gpu.PREC_MIXED)
    ref = case["runs"]["HOOI"]["error"][-1]
    assert abs(d.error - ref) <= 1e-6 * ref, (d.error, ref)
