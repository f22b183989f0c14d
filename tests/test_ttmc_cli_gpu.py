"""GPU tests of the drop-in example drivers.  symprop_b200/symtens_ttmc
against the reference's own examples/symtens_ttmc.cpp run on the same .tns
files (tests/golden/ttmc.npz, made by tests/golden/make_golden.py);
symprop_b200/s3ttmctc (examples/s3ttmctc.cpp, which prints timings only)
by its output lines.

ttmc.out holds every packed Y value in fixed notation with 5 decimals.  The
FP64 S3TTMc agrees with the reference to about 1e-15 relative, so a printed
value can differ only where the exact result lies within that distance of a
rounding boundary of the last decimal: such tokens may differ by one unit
in the last place (1e-5); every other token, and the layout, must match byte
for byte."""
import os
import re
import subprocess

import numpy as np
import pytest

GOLD = os.path.join(os.path.dirname(__file__), "golden")

pytestmark = pytest.mark.gpu


def test_symtens_ttmc_output_matches_reference_driver(gpu, tmp_path):
    g = np.load(os.path.join(GOLD, "ttmc.npz"))
    ncase = len([k for k in g.files if k.endswith("_meta")])
    assert ncase >= 5
    for ci in range(ncase):
        order, n, nnz, seed, R = (int(x) for x in g[f"c{ci}_meta"])
        d = tmp_path / f"c{ci}"
        d.mkdir()
        (d / "x.tns").write_bytes(bytes(g[f"c{ci}_tns"]))
        r = subprocess.run([gpu.TTMC_PATH, str(d / "x.tns"), str(R)], capture_output=True, text=True, cwd=d)
        assert r.returncode == 0, r.stderr
        lines = r.stdout.splitlines()
        assert lines[0] == "Finished creating compressed dtree"  # src/sparse/spsymtensor.cpp:26
        assert re.fullmatch(r"Insertion time: \d+ ms", lines[1]) and re.fullmatch(r"S3TTMc Time: \d+ ms", lines[2])
        want = bytes(g[f"c{ci}_out"]).decode()
        got = (d / "ttmc.out").read_text()
        if got == want:
            continue
        wl, gl = want.split("\n"), got.split("\n")
        assert len(wl) == len(gl) == n + 1, ci
        off = 0
        for a, b in zip(wl, gl):
            ta, tb = a.split(", "), b.split(", ")
            assert len(ta) == len(tb), ci
            for x, y in zip(ta, tb):
                if x != y:
                    assert abs(float(x) - float(y)) <= 1.000001e-5, (ci, x, y)
                    off += 1
        assert off <= max(2, n // 50), (ci, off)


def test_s3ttmctc_driver_lines(gpu, tmp_path):
    """examples/s3ttmctc.cpp: the tensor line, "Insertion time", ten
    "S3TTMcTC Time" lines and the FunctionTimer table, whose S3TTMc, gemmtn
    and symgemm rows count the ten rounds."""
    g = np.load(os.path.join(GOLD, "ttmc.npz"))
    (tmp_path / "x.tns").write_bytes(bytes(g["c1_tns"]))
    R = int(g["c1_meta"][4])
    r = subprocess.run([gpu.TTMCTC_PATH, str(tmp_path / "x.tns"), str(R)], capture_output=True, text=True,
                       cwd=tmp_path)
    assert r.returncode == 0, r.stderr
    lines = r.stdout.splitlines()
    assert lines[0] == "Finished creating compressed dtree"
    assert re.fullmatch(r"Insertion time: \d+ ms", lines[1])
    assert all(re.fullmatch(r"S3TTMcTC Time: \d+ ms", l) for l in lines[2:12])
    assert lines[12] == "Accumulated function times:"
    rows = {m.group(3): int(m.group(2)) for m in
            (re.fullmatch(r"\s*([0-9.]+) ms  \|\s+(\d+) calls \| (.+)", l) for l in lines[13:]) if m}
    assert rows.get("S3TTMc") == 10 and rows.get("gemmtn") == 10 and rows.get("symgemm") == 10
    r = subprocess.run([gpu.TTMCTC_PATH], capture_output=True, text=True)
    assert r.returncode == 1 and r.stderr.startswith("Usage: ")
