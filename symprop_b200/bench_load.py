"""Time .tns ingest: the reference's SymtensLoader (host iostream, timed by
oracle/_ref/ref_probe when that build is present) against
symprop_tensor_load_tns (file read + device tokenise/parse + tensor build)
and against symprop_tensor_load_spt (the same tuples as a binary SPT1 file:
file read + tensor build).

    python -m symprop_b200.bench_load --workload s3ttmc_order4_zipf

Writes the workload's tuples as a text .tns (values with 17 significant
digits, so the parser's host strtod path is exercised too) into a temporary
directory, then prints one JSON line.
"""
import argparse
import json
import os
import subprocess
import tempfile
import time

import numpy as np

from . import SpSymtensor, lib, synth

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--workload", default="s3ttmc_order4_zipf")
    ap.add_argument("--scale", type=float, default=1.0)
    ap.add_argument("--reps", type=int, default=3)
    a = ap.parse_args()
    order, n, t, v = synth.workload(a.workload, scale=a.scale)
    lib()
    with tempfile.TemporaryDirectory() as d:
        path = os.path.join(d, "x.tns")
        synth.write_tns(path, order, n, t, v)
        size = os.path.getsize(path)
        X = SpSymtensor.load_tns(path)  # warm-up (module load, first allocations)
        X.close()
        dev = []
        for _ in range(a.reps):
            t0 = time.perf_counter()
            X = SpSymtensor.load_tns(path)
            dev.append((time.perf_counter() - t0) * 1e3)
            assert X.size() == t.shape[0]
            X.close()
        t0 = time.perf_counter()
        Y = SpSymtensor(n, order, t, v)
        build_ms = (time.perf_counter() - t0) * 1e3
        Y.close()
        spt = os.path.join(d, "x.spt")
        synth.write_spt(spt, order, n, t, v)
        spt_size = os.path.getsize(spt)
        spt_ms = []
        for _ in range(a.reps):
            t0 = time.perf_counter()
            Z = SpSymtensor.load_spt(spt)
            spt_ms.append((time.perf_counter() - t0) * 1e3)
            assert Z.size() == t.shape[0]
            Z.close()
        ref = None
        probe = os.path.join(ROOT, "oracle", "_ref", "ref_probe")
        if os.path.exists(probe):
            out = subprocess.run([probe, "load", path, os.path.join(d, "x.bin")], check=True,
                                 capture_output=True, text=True).stdout
            ref = json.loads(out.strip().splitlines()[-1])["load_ms"]
    print(json.dumps({"workload": a.workload, "scale": a.scale, "nnz": int(t.shape[0]), "order": order,
                      "file_mb": round(size / 1e6, 1), "device_load_ms": round(min(dev), 1),
                      "of_which_tensor_build_ms": round(build_ms, 1),
                      "spt_file_mb": round(spt_size / 1e6, 1), "spt_load_ms": round(min(spt_ms), 1),
                      "reference_loader_ms": ref,
                      "reference_loader_note": "host iostream parse only (tree build not included)"}))


if __name__ == "__main__":
    main()
