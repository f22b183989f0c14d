"""GPU tests of the binary SPT1 tuple files (symprop_tensor_load_spt /
save_spt): the bytes a tensor saves are synth.write_spt's for its tuples,
loading them back gives the same tensor (tuples, values, S3TTMc bit for bit)
as the arrays and the .tns text do, and malformed files come back as
status codes.  The CLI and the example drivers take SPT1 files by their
magic."""
import struct
import subprocess

import numpy as np
import pytest

from symprop_b200 import synth

pytestmark = pytest.mark.gpu


def test_spt_round_trip_matches_arrays_and_text(gpu, tmp_path):
    order, n, nnz, R = 4, 300, 5000, 6
    t = synth.zipf_tuples(order, n, nnz, 1.2, 3)
    v = synth.uniform_values(nnz, 3)
    X = gpu.SpSymtensor(n, order, t, v)
    inds, vals = X.nonzeros()
    p, q = tmp_path / "x.spt", tmp_path / "ref.spt"
    X.save_spt(str(p))
    synth.write_spt(str(q), order, n, inds, vals)
    assert p.read_bytes() == q.read_bytes()
    Y = gpu.SpSymtensor.load_spt(str(p))
    assert (Y.order(), Y.dim(), Y.size()) == (order, n, inds.shape[0])
    i2, v2 = Y.nonzeros()
    np.testing.assert_array_equal(i2, inds)
    np.testing.assert_array_equal(v2, vals)
    assert Y.norm() == X.norm()
    tns = tmp_path / "x.tns"
    synth.write_tns(str(tns), order, n, t, v)
    Z = gpu.SpSymtensor.load_tns(str(tns))
    U = np.random.default_rng(4).standard_normal((n, R))
    Yx = X.S3TTMc(U, R, True)
    np.testing.assert_array_equal(Y.S3TTMc(U, R, True), Yx)
    np.testing.assert_array_equal(Z.S3TTMc(U, R, True), Yx)


def test_empty_spt(gpu, tmp_path):
    p = tmp_path / "e.spt"
    synth.write_spt(str(p), 3, 7, np.zeros((0, 3), np.uint32), np.zeros(0))
    X = gpu.SpSymtensor.load_spt(str(p))
    assert X.size() == 0 and X.norm() == 0.0
    assert np.all(X.S3TTMc(np.ones((7, 2)), 2, True) == 0)


def test_malformed_spt_is_a_status(gpu, tmp_path):
    t = np.array([[1, 2, 3], [2, 2, 5]], np.uint32)
    v = np.array([1.0, 2.0])
    good = tmp_path / "g.spt"
    synth.write_spt(str(good), 3, 5, t, v)
    raw = good.read_bytes()
    cases = {
        "magic": (b"SPT2" + raw[4:], gpu.ERR_INVALID),
        "truncated": (raw[:-3], gpu.ERR_INVALID),
        "trailing bytes": (raw + b"\0", gpu.ERR_INVALID),
        "id above dim": (raw[:4] + struct.pack("<I", 3) + struct.pack("<I", 4) + raw[12:], gpu.ERR_INVALID),
        "order 9": (raw[:4] + struct.pack("<I", 9) + raw[8:], gpu.ERR_ORDER),
    }
    for name, (data, status) in cases.items():
        p = tmp_path / f"{name.replace(' ', '_')}.spt"
        p.write_bytes(data)
        with pytest.raises(gpu.SympropError) as e:
            gpu.SpSymtensor.load_spt(str(p))
        assert e.value.status == status, name
    unsorted = tmp_path / "u.spt"
    synth.write_spt(str(unsorted), 3, 5, np.array([[3, 2, 1]], np.uint32), np.array([1.0]))
    with pytest.raises(gpu.SympropError) as e:
        gpu.SpSymtensor.load_spt(str(unsorted))
    assert e.value.status == gpu.ERR_INVALID


def test_cli_and_driver_take_spt(gpu, tmp_path):
    order, n, nnz = 3, 60, 800
    t = synth.zipf_tuples(order, n, nnz, 1.2, 31)
    v = np.ones(nnz)
    tns, spt = tmp_path / "x.tns", tmp_path / "x.spt"
    synth.write_tns(str(tns), order, n, t, v)
    synth.write_spt(str(spt), order, n, t, v)

    def iters(path):
        r = subprocess.run([gpu.CLI_PATH, "-f", str(path), "-r", "4", "-i", "5", "-d", "0.5", "-s", "0", "-a", "0"],
                           capture_output=True, text=True, timeout=300)
        assert r.returncode == 0, r.stderr
        return [l for l in r.stdout.splitlines() if l.startswith("Iteration: ")]

    assert iters(spt) == iters(tns) and len(iters(tns)) > 0
    for f in (tns, spt):
        d = tmp_path / f.suffix[1:]
        d.mkdir()
        r = subprocess.run([gpu.TTMC_PATH, str(f), "3"], capture_output=True, text=True, cwd=d, timeout=300)
        assert r.returncode == 0, r.stderr
    assert (tmp_path / "tns" / "ttmc.out").read_bytes() == (tmp_path / "spt" / "ttmc.out").read_bytes()
