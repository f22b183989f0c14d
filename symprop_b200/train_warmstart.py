"""Train the learned warm start on the GPU and record what it gains.

    python -m symprop_b200.train_warmstart --count 64 --epochs 20 \
        --out symprop_b200/warmstart_r8.npz --report profiles/warmstart_r8.json

Training tensors are seeded synthetic planted-community tensors (order 3..6,
Zipf(1.2) degrees inside communities); labels are the converged factors of
this package's FP64 GPU HOOI (rank 8); 2-layer per-node MLP (hidden 64),
BF16 weights with an FP32 master copy, Adam.  The report compares
random-start and learned-start HOOI on held-out seeds.
"""
import argparse
import json
import time

import numpy as np

from . import warmstart as ws


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--count", type=int, default=64)
    ap.add_argument("--heldout", type=int, default=12)
    ap.add_argument("--epochs", type=int, default=20)
    ap.add_argument("--lr", type=float, default=1e-3)
    ap.add_argument("--rank", type=int, default=8)
    ap.add_argument("--hidden", type=int, default=64)
    ap.add_argument("--full-size", action="store_true", help="n up to 20k, nnz up to 500k")
    ap.add_argument("--family", default="community", choices=["community", "powerlaw"],
                    help="training tensors: planted-community Zipf (orders 3-6) or order-5 power-law")
    ap.add_argument("--out", default=ws.DEFAULT_WEIGHTS)
    ap.add_argument("--report", default=None)
    a = ap.parse_args()
    t0 = time.time()
    samples = ws.make_samples(range(a.count), R=a.rank, small=not a.full_size, family=a.family)
    t1 = time.time()
    model = ws.WarmStartModel(a.rank, a.hidden, seed=0)
    hist = ws.train(model, samples, epochs=a.epochs, lr=a.lr)
    t2 = time.time()
    model.save(a.out)
    rows = ws.compare(model, range(5000, 5000 + a.heldout), R=a.rank, small=not a.full_size,
                      family=a.family)
    rep = {
        "train_tensors": a.count, "family": a.family, "epochs": a.epochs, "lr": a.lr, "rank": a.rank, "hidden": a.hidden,
        "label_gen_s": round(t1 - t0, 1), "train_s": round(t2 - t1, 1), "loss_history": hist,
        "heldout": rows,
        "mean_random_iters": float(np.mean([r["random_iters"] for r in rows])),
        "mean_learned_iters": float(np.mean([r["learned_iters"] for r in rows])),
        "mean_random_ms": float(np.mean([r["random_ms"] for r in rows])),
        "mean_learned_ms": float(np.mean([r["learned_ms"] for r in rows])),
        "max_error_gap": float(max(r["learned_error"] - r["random_error"] for r in rows)),
    }
    print(json.dumps({k: v for k, v in rep.items() if k not in ("heldout", "loss_history")}))
    if a.report:
        with open(a.report, "w") as f:
            json.dump(rep, f, indent=1)


if __name__ == "__main__":
    main()
