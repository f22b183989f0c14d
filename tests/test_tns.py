"""CPU: the .tns oracle (oracle/tns_oracle.py) against the reference's own
SymtensLoader (oracle/_ref/ref_probe load, src/utils/loader.cpp:8-36),
bit for bit, on every text case of tests/tns_cases.py."""
import os
import struct
import subprocess
import sys
import tempfile

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, os.path.join(ROOT, "oracle"))
import tns_oracle  # noqa: E402
from tns_cases import CASES, random_text  # noqa: E402

PROBE = os.path.join(ROOT, "oracle", "_ref", "ref_probe")


def ref_load(data: bytes):
    with tempfile.TemporaryDirectory() as d:
        src, dst = os.path.join(d, "x.tns"), os.path.join(d, "x.bin")
        open(src, "wb").write(data)
        subprocess.run([PROBE, "load", src, dst], check=True, capture_output=True)
        raw = open(dst, "rb").read()
    order, dim, nnz = struct.unpack_from("<IIQ", raw, 0)
    inds = np.frombuffer(raw, dtype=np.uint32, count=nnz * order, offset=16).reshape(nnz, order)
    vals = np.frombuffer(raw, dtype=np.float64, count=nnz, offset=16 + 4 * nnz * order)
    return order, dim, inds, vals


@pytest.mark.skipif(not os.path.exists(PROBE), reason="reference build (oracle/_ref) not present")
@pytest.mark.parametrize("name", sorted(CASES) + ["random"])
def test_oracle_matches_reference_loader(name):
    data = random_text(1, nnz=3000) if name == "random" else CASES[name]
    o = tns_oracle.load_tns(data)
    r = ref_load(data)
    assert o[0] == r[0] and o[1] == r[1]
    np.testing.assert_array_equal(o[2], r[2])
    assert o[3].tobytes() == r[3].tobytes()


def test_oracle_edge_rules():
    assert tns_oracle.load_tns(CASES["no_trailing_newline"])[2].shape[0] == 2
    assert tns_oracle.load_tns(CASES["partial_record"])[2].shape[0] == 2
    assert tns_oracle.load_tns(CASES["header_only"])[2].shape[0] == 0
