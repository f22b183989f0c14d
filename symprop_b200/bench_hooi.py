"""HOOI time to tolerance on one GPU: plain FP64 (random start) against
mixed precision (FP32 S3TTMc + tcgen05 split-BF16 Gram + FP64 solves),
from random and learned starts, and the reference CPU build on the small
order-5 workload.

    python -m symprop_b200.bench_hooi --workload hooi_order5_zipf --rank 8 --tol 1e-6
    python -m symprop_b200.bench_hooi --workload learned_order5_powerlaw --scale 0.1 --rank 16

Prints one JSON line per run and a summary line.  Times are device-timed
solves (symprop_result.time_ms) plus, for the learned start, the wall time
of the prediction (features + MLP + QR); tensor construction is excluded
for every arm, and the reference arm's "Time" line likewise excludes its
tree build.
"""
import argparse
import json
import os
import re
import subprocess
import tempfile
import time

import numpy as np

from . import PREC_FP64, PREC_MIXED, SpSymtensor, synth

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def run_ref(order, n, t, v, rank, iters, tol, delta):
    cli = os.path.join(ROOT, "oracle", "_ref", "symtucker")
    if not os.path.exists(cli):
        return None
    with tempfile.TemporaryDirectory() as d:
        tns = os.path.join(d, "x.tns")
        synth.write_tns(tns, order, n, t, v)
        out = subprocess.run([cli, "-f", tns, "-r", str(rank), "-i", str(iters), "-t", str(tol), "-d", str(delta),
                              "-s", "0", "-a", "0"], capture_output=True, text=True,
                             env=dict(os.environ, OMP_NUM_THREADS=str(os.cpu_count() or 1))).stdout
    errs = [float(x) for x in re.findall(r"error (\S+)", out)]
    ms = re.findall(r"Time: (\d+) ms", out)
    return {"arm": "reference_cpu", "iters": len(errs), "error": errs[-1] if errs else None,
            "ms": float(ms[0]) if ms else None, "cores": os.cpu_count()}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--workload", default="hooi_order5_zipf")
    ap.add_argument("--scale", type=float, default=1.0)
    ap.add_argument("--rank", type=int, default=8)
    ap.add_argument("--iters", type=int, default=200)
    ap.add_argument("--tol", type=float, default=1e-6)
    ap.add_argument("--delta", type=float, default=1.0)
    ap.add_argument("--weights", default=None)
    ap.add_argument("--reference", action="store_true")
    ap.add_argument("--arms", default="fp64_random,mixed_random,mixed_learned,fp64_learned",
                    help="comma list of fp64_random, mixed_random, mixed_learned, fp64_learned")
    ap.add_argument("--no-warmup", action="store_true", help="skip the untimed first solve")
    ap.add_argument("--alg", default="hooi", choices=["hooi", "hoqri"])
    a = ap.parse_args()
    arms = set(a.arms.split(","))
    order, n, t, v = synth.workload(a.workload, scale=a.scale)
    X = SpSymtensor(n, order, t, v)
    rows = []
    ref64_box, solved = [], []

    def solve(name, precision, init="rnd", U0=None, extra_ms=0.0):
        kw = dict(rank=a.rank, max_iter=a.iters, rel_tol=a.tol, delta=a.delta, seed=0, precision=precision)
        if U0 is not None:
            kw.update(init="user", init_factor=U0)
        d = (X.TuckerHOOI if a.alg == "hooi" else X.TuckerHOQRI)(**kw)
        row = {"arm": name, "iters": d.iterations, "error": d.error, "ms": d.time_ms + extra_ms,
               "s3ttmc_ms": d.s3ttmc_ms, "dense_ms": d.dense_ms}
        if extra_ms:
            row["prediction_ms"] = extra_ms
        if ref64_box:  # errors against the FP64 random-start solve (the oracle arm)
            r64 = ref64_box[0]
            sv = np.linalg.svd(r64.factor.T @ d.factor, compute_uv=False)
            row["max_principal_angle_vs_fp64"] = float(np.arccos(np.clip(sv.min(), -1.0, 1.0)))
            row["core_norm_sq_rel_err_vs_fp64"] = abs(d.core_norm ** 2 - r64.core_norm ** 2) / r64.core_norm ** 2
        solved.append(d)
        rows.append(row)
        print(json.dumps(row))
        return d

    if not a.no_warmup:
        solve("warmup", PREC_FP64)  # first-use plans and module loading
        rows.clear()
    ref64 = solve("fp64_random", PREC_FP64) if "fp64_random" in arms else None
    if ref64 is not None:
        ref64_box.append(ref64)
    if "mixed_random" in arms:
        solve("mixed_random", PREC_MIXED)
    wpath = a.weights
    if wpath is None:
        cand = os.path.join(os.path.dirname(os.path.abspath(__file__)), f"warmstart_r{a.rank}.npz")
        wpath = cand if os.path.exists(cand) else None
    if wpath and arms & {"mixed_learned", "fp64_learned"}:
        from .warmstart import WarmStartModel
        model = WarmStartModel.load(wpath)
        t0 = time.perf_counter()
        U0 = model.predict(X, seed=0)
        pred_ms = (time.perf_counter() - t0) * 1e3
        if "mixed_learned" in arms:
            solve("mixed_learned", PREC_MIXED, U0=U0, extra_ms=pred_ms)
        if "fp64_learned" in arms:
            solve("fp64_learned", PREC_FP64, U0=U0, extra_ms=pred_ms)
    if a.reference:
        r = run_ref(order, n, t, v, a.rank, a.iters, a.tol, a.delta)
        if r:
            rows.append(r)
            print(json.dumps(r))
    summ = {"workload": a.workload, "scale": a.scale, "order": order, "n": n, "nnz": int(t.shape[0]),
            "rank": a.rank, "tol": a.tol, "delta": a.delta}
    if ref64 is not None:
        summ["speedup_vs_fp64_random"] = {r["arm"]: round(ref64.time_ms / r["ms"], 3) for r in rows if r["ms"]}
        summ["objective_rel_gap_vs_fp64"] = {r["arm"]: (abs(r["error"] - ref64.error) / ref64.error
                                                        if r["error"] is not None else None) for r in rows}
    print(json.dumps(summ))


if __name__ == "__main__":
    main()
