"""Regenerates the golden fixtures in tests/golden/ by running the reference
SymProp itself (its own sources compiled into oracle/_ref by oracle/Makefile).

    make -C oracle ref && python tests/golden/make_golden.py          # all fixtures
    make -C oracle ref && python tests/golden/make_golden.py ttmc     # ttmc.npz only

Fixtures (all small):
  trees.npz     CompressedDTree arrays (level_idx, level_ptr, dep_list,
                owners) dumped from the reference for seeded tensors with
                repeated ids, orders 2..6
  s3ttmc.npz    the reference's S3TTMc Y (packed and unpacked) for seeded
                tensors and factor matrices, orders 3..6
  tucker.json   the reference's per-iteration error lines of HOOI / HOQRI /
                AltHOOI (symtucker CLI) on seeded tensors, and on the shipped
                examples/contact-5.tns when present
  contact5.npz  the tensor of examples/contact-5.tns as the reference's
                SymtensLoader reads it (ids sorted within each tuple, values),
                so that the contact-5 runs can be repeated without the
                reference tree (python tests/golden/make_golden.py contact5)
  ttmc.npz      the reference's examples/symtens_ttmc driver run on seeded
                .tns files: the input text, the driver's ttmc.out bytes
"""
import json
import os
import re
import subprocess
import sys
import tempfile

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)
from symprop_b200 import synth  # noqa: E402

OUT = os.path.dirname(os.path.abspath(__file__))
PROBE = os.path.join(ROOT, "oracle", "_ref", "ref_probe")
CLI = os.path.join(ROOT, "oracle", "_ref", "symtucker")
TTMC = os.path.join(ROOT, "oracle", "_ref", "symtens_ttmc")
# the reference tree (SYMPROP_REF, as in oracle/Makefile's REF)
REF = os.environ.get("SYMPROP_REF", "/root/reference")
CONTACT5 = os.path.join(REF, "examples", "contact-5.tns")

TREE_CASES = [  # order, n, nnz, seed
    (2, 10, 30, 11), (3, 20, 50, 1), (4, 30, 300, 2), (5, 15, 200, 3), (6, 12, 150, 4), (4, 6, 40, 5),
    (3, 40, 1, 6),
]
Y_CASES = [  # order, n, nnz, seed, R
    (3, 25, 120, 21, 3), (3, 30, 200, 22, 7), (4, 30, 300, 23, 4), (4, 50, 600, 24, 6),
    (5, 20, 250, 25, 3), (5, 40, 500, 26, 5), (6, 15, 150, 27, 3), (4, 8, 60, 28, 16),
]
TTMC_CASES = [  # order, n, nnz, seed, R
    (3, 40, 300, 41, 4), (4, 60, 800, 42, 5), (5, 30, 400, 43, 3), (2, 10, 20, 44, 3), (6, 12, 100, 45, 2),
    (4, 120, 2000, 46, 8),
]
TUCKER_CASES = [  # name, order, n, nnz, seed, R, iters, delta, s
    ("o3_n60", 3, 60, 800, 31, 4, 15, 0.5, 1.2),
    ("o4_n80", 4, 80, 2000, 32, 5, 15, 0.3, 1.2),
    ("o5_n250_zipf", 5, 250, 10000, 0, 8, 20, 0.1, 1.2),
]


def read_dump(path):
    f = open(path, "rb").read()
    o = 0

    def get(fmt, size):
        nonlocal o
        v = np.frombuffer(f, dtype=fmt, count=1, offset=o)[0]
        o += size
        return v

    def getv(dt):
        nonlocal o
        n = int(get(np.uint64, 8))
        a = np.frombuffer(f, dtype=dt, count=n, offset=o).copy()
        o += n * np.dtype(dt).itemsize
        return a

    depth = int(get(np.uint32, 4))
    lv = []
    for _ in range(depth):
        lv.append((getv(np.uint32), getv(np.uint64), getv(np.uint64)))
    rem, val = getv(np.uint64), getv(np.float64)
    norm = float(get(np.float64, 8))
    return depth, lv, rem, val, norm


def parse_iters(text):
    runs = {}
    cur = None
    for line in text.splitlines():
        m = re.match(r"Running (\w+) algorithm", line)
        if m:
            cur = m.group(1)
            runs[cur] = {"error": [], "relres": []}
            continue
        m = re.match(r"Iteration: (\d+) relative residual: (\S+) error (\S+)", line)
        if m and cur:
            runs[cur]["relres"].append(float(m.group(2)))
            runs[cur]["error"].append(float(m.group(3)))
    return runs


def make_ttmc(tmp):
    out = {}
    for ci, (order, n, nnz, seed, R) in enumerate(TTMC_CASES):
        t = synth.zipf_tuples(order, n, nnz, 1.2, seed)
        v = synth.uniform_values(nnz, seed)
        d = os.path.join(tmp, f"ttmc{ci}")
        os.makedirs(d)
        tns = os.path.join(d, "x.tns")
        synth.write_tns(tns, order, n, t, v)
        subprocess.run([TTMC, tns, str(R)], check=True, capture_output=True, cwd=d,
                       env=dict(os.environ, OMP_NUM_THREADS="8"))
        out[f"c{ci}_meta"] = np.array([order, n, nnz, seed, R], np.int64)
        out[f"c{ci}_tns"] = np.frombuffer(open(tns, "rb").read(), np.uint8)
        out[f"c{ci}_out"] = np.frombuffer(open(os.path.join(d, "ttmc.out"), "rb").read(), np.uint8)
    np.savez_compressed(os.path.join(OUT, "ttmc.npz"), **out)


def make_contact5(tmp):
    """contact-5 as the reference loader reads it (ref_probe load)."""
    dump = os.path.join(tmp, "contact5.bin")
    subprocess.run([PROBE, "load", CONTACT5, dump], check=True, capture_output=True)
    raw = open(dump, "rb").read()
    order, dim = np.frombuffer(raw[:8], np.uint32)
    nnz = int(np.frombuffer(raw[8:16], np.uint64)[0])
    inds = np.frombuffer(raw[16:16 + 4 * nnz * order], np.uint32).reshape(nnz, order)
    vals = np.frombuffer(raw[16 + 4 * nnz * order:16 + 4 * nnz * order + 8 * nnz], np.float64)
    np.savez_compressed(os.path.join(OUT, "contact5.npz"), order=np.int64(order), dim=np.int64(dim),
                        inds=inds.astype(np.uint8 if dim < 256 else np.uint32), vals=vals)


def main():
    tmp = tempfile.mkdtemp()
    want = set(sys.argv[1:]) or {"trees", "s3ttmc", "tucker", "ttmc", "contact5"}
    if "ttmc" in want:
        make_ttmc(tmp)
    if "contact5" in want and os.path.exists(CONTACT5):
        make_contact5(tmp)
    if not want & {"trees", "s3ttmc", "tucker"}:
        print("wrote", os.listdir(OUT))
        return
    trees = {}
    for ci, (order, n, nnz, seed) in enumerate(TREE_CASES):
        t = synth.zipf_tuples(order, n, nnz, 1.2, seed)
        v = synth.uniform_values(nnz, seed)
        spt = os.path.join(tmp, f"t{ci}.spt")
        synth.write_spt(spt, order, n, t, v)
        subprocess.run([PROBE, "tree", spt, spt + ".tree"], check=True, capture_output=True)
        depth, lv, rem, val, norm = read_dump(spt + ".tree")
        trees[f"c{ci}_meta"] = np.array([order, n, nnz, seed], np.int64)
        trees[f"c{ci}_inds"] = t
        trees[f"c{ci}_vals"] = v
        trees[f"c{ci}_norm"] = np.array([norm])
        for l in range(depth):
            trees[f"c{ci}_idx{l}"] = lv[l][0]
            trees[f"c{ci}_ptr{l}"] = lv[l][1]
            trees[f"c{ci}_dep{l}"] = lv[l][2]
        trees[f"c{ci}_rem"] = rem
        trees[f"c{ci}_val"] = val
    np.savez_compressed(os.path.join(OUT, "trees.npz"), **trees)

    ys = {}
    for ci, (order, n, nnz, seed, R) in enumerate(Y_CASES):
        t = synth.zipf_tuples(order, n, nnz, 1.2, seed)
        v = synth.uniform_values(nnz, seed)
        U = np.random.default_rng(seed).standard_normal((n, R))
        spt = os.path.join(tmp, f"y{ci}.spt")
        synth.write_spt(spt, order, n, t, v)
        U.tofile(spt + ".u")
        ys[f"c{ci}_meta"] = np.array([order, n, nnz, seed, R], np.int64)
        ys[f"c{ci}_inds"] = t
        ys[f"c{ci}_vals"] = v
        ys[f"c{ci}_U"] = U
        for packed in (1, 0):
            subprocess.run([PROBE, "s3ttmc", spt, str(R), spt + ".u", str(packed), spt + ".y"],
                           check=True, capture_output=True)
            ys[f"c{ci}_Y{'p' if packed else 'u'}"] = np.fromfile(spt + ".y").reshape(n, -1)
    np.savez_compressed(os.path.join(OUT, "s3ttmc.npz"), **ys)

    tucker = {}
    for (name, order, n, nnz, seed, R, iters, delta, s) in TUCKER_CASES:
        t = synth.zipf_tuples(order, n, nnz, s, seed)
        v = np.ones(nnz)
        tns = os.path.join(tmp, name + ".tns")
        synth.write_tns(tns, order, n, t, v)
        args = ["-f", tns, "-r", str(R), "-i", str(iters), "-d", str(delta), "-s", "0", "-a", "-1"]
        out = subprocess.run([CLI] + args, check=True, capture_output=True, text=True,
                             env=dict(os.environ, OMP_NUM_THREADS="8")).stdout
        tucker[name] = {"order": order, "n": n, "nnz": nnz, "seed": seed, "zipf": s, "rank": R,
                        "iters": iters, "delta": delta, "runs": parse_iters(out)}
    if os.path.exists(CONTACT5):
        args = ["-f", CONTACT5, "-r", "8", "-i", "20", "-d", "0.1", "-s", "0", "-a", "-1"]
        out = subprocess.run([CLI] + args, check=True, capture_output=True, text=True,
                             env=dict(os.environ, OMP_NUM_THREADS="8")).stdout
        tucker["contact5"] = {"rank": 8, "iters": 20, "delta": 0.1, "runs": parse_iters(out)}
    with open(os.path.join(OUT, "tucker.json"), "w") as f:
        json.dump(tucker, f, indent=1)
    print("wrote", os.listdir(OUT))


if __name__ == "__main__":
    main()
