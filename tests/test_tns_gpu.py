"""GPU: the device .tns parser (symprop_tensor_load_tns) against the loader
oracle (oracle/tns_oracle.py, pinned to the reference's SymtensLoader by
tests/test_tns.py): ids and values bit for bit, the same stopping rules, and
the same tensor as one built from the parsed arrays."""
import os
import sys
import tempfile

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, os.path.join(ROOT, "oracle"))
import tns_oracle  # noqa: E402
from tns_cases import CASES, MALFORMED, random_text  # noqa: E402

pytestmark = pytest.mark.gpu


def load(gpu, data: bytes):
    with tempfile.TemporaryDirectory() as d:
        p = os.path.join(d, "x.tns")
        open(p, "wb").write(data)
        return gpu.SpSymtensor.load_tns(p)


@pytest.mark.parametrize("name", sorted(CASES) + ["random"])
def test_parse_matches_oracle(gpu, name):
    data = random_text(2) if name == "random" else CASES[name]
    order, dim, inds, vals = tns_oracle.load_tns(data)
    X = load(gpu, data)
    assert (X.order(), X.dim(), X.size()) == (order, dim, inds.shape[0])
    gi, gv = X.nonzeros()
    np.testing.assert_array_equal(gi, inds)
    assert gv.tobytes() == vals.tobytes()


def test_same_tensor_as_array_constructor(gpu):
    data = random_text(3, order=4, dim=300, nnz=20_000)
    order, dim, inds, vals = tns_oracle.load_tns(data)
    X = load(gpu, data)
    Y = gpu.SpSymtensor(dim, order, inds, vals)
    assert X.norm() == Y.norm()
    U = np.random.default_rng(0).standard_normal((dim, 6))
    np.testing.assert_array_equal(X.S3TTMc(U, 6, True), Y.S3TTMc(U, 6, True))


@pytest.mark.parametrize("name", sorted(MALFORMED))
def test_malformed_token_fails_loudly(gpu, name):
    with pytest.raises(gpu.SympropError) as e:
        load(gpu, MALFORMED[name])
    assert e.value.status == gpu.ERR_INVALID


def test_missing_file_and_bad_ids(gpu):
    with pytest.raises(gpu.SympropError):
        gpu.SpSymtensor.load_tns("/nonexistent/x.tns")
    with pytest.raises(gpu.SympropError) as e:
        load(gpu, b"3 4\n1 2 9 1.0\n")  # id above dim
    assert e.value.status == gpu.ERR_INVALID
