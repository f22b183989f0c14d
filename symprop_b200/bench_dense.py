"""Timing of the mixed-precision dense products on one GPU, through the C ABI.

    python -m symprop_b200.bench_dense --n 200000 --m 3876 --r 16

Times (CUDA events around each call, after warm-up; every call also splits
its operand, allocates its workspace and synchronises):
  * gram   G = (Y D^1/2)^T (Y D^1/2), m x m, tcgen05 split-BF16
           (symprop_gram_device, FP32 input);
  * panel  W = (Y D^1/2)(V D^1/2)^T, n x r (symprop_symgemm_device);
  * rows   G = (Y D^1/2)(Y D^1/2)^T for an n <= m slice (symprop_symsyrk_device);
  * gram64 the same m x m Gram from an FP64 Y on the CUDA cores (symprop_gram_device,
           FP64 input: HOOI's dense step in FP64), against the nominal FP64 rate
           of a B200 (37 TFLOP/s).
Rates count the tensor-core work the split needs: three BF16 products over
the upper-triangular half of a Gram (m (m + 1) / 2 entries, K = n), all
n r entries of the panel.  Peaks from MEASURED_PEAKS.json when present.
"""
import argparse
import json
import os

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def main():
    import torch

    from . import FP32, FP64, gram_device, lib, symgemm_device, symsyrk_device
    ap = argparse.ArgumentParser()
    ap.add_argument("--n", type=int, default=200000)
    ap.add_argument("--m", type=int, default=3876)
    ap.add_argument("--r", type=int, default=16)
    ap.add_argument("--rows", type=int, default=2048, help="rows of the row-Gram case")
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--only", default="gram,panel,rows,gram64")
    a = ap.parse_args()
    lib()
    torch.cuda.set_device(0)
    g = torch.Generator(device="cuda").manual_seed(0)
    Y = torch.randn(a.n, a.m, device="cuda", generator=g)
    sd = torch.rand(a.m, device="cuda", generator=g) + 0.5
    peaks = {}
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        peaks = json.load(open(p))
    bf16_peak = float(peaks.get("bf16_tflops", 1590.0))
    out = {"n": a.n, "m": a.m, "r": a.r, "bf16_peak_tflops": bf16_peak,
           "peak_kind": "measured" if peaks else "fallback"}

    def timed(fn):
        for _ in range(a.warmup):
            fn()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(a.steps):
            fn()
        e1.record()
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) / a.steps

    only = set(a.only.split(","))
    if "gram" in only:
        G = torch.empty(a.m, a.m, dtype=torch.float64, device="cuda")
        ms = timed(lambda: gram_device(Y.data_ptr(), a.n, a.m, sd.data_ptr(), G.data_ptr(), FP32))
        fl = 3 * 2.0 * a.n * a.m * (a.m + 1) / 2
        out["gram"] = {"ms": round(ms, 3), "tflops": round(fl / ms / 1e9, 1),
                       "frac_of_bf16_peak": round(fl / ms / 1e9 / bf16_peak, 3)}
    if "panel" in only:
        V = torch.randn(a.r, a.m, dtype=torch.float64, device="cuda", generator=g)
        sdd = sd.double()
        W = torch.empty(a.n, a.r, dtype=torch.float64, device="cuda")
        ms = timed(lambda: symgemm_device(Y.data_ptr(), V.data_ptr(), sdd.data_ptr(), W.data_ptr(), a.m, a.n, a.r))
        out["panel"] = {"ms": round(ms, 3), "y_gbs": round(a.n * a.m * 4 / ms / 1e6, 1)}
    if "rows" in only:
        k = min(a.rows, a.n)
        C = torch.empty(k, k, dtype=torch.float64, device="cuda")
        ms = timed(lambda: symsyrk_device(Y.data_ptr(), sd.data_ptr(), C.data_ptr(), a.m, k))
        fl = 3 * 2.0 * a.m * k * (k + 1) / 2
        out["rows"] = {"rows": k, "ms": round(ms, 3), "tflops": round(fl / ms / 1e9, 1)}
    if "gram64" in only:
        del Y
        torch.cuda.empty_cache()
        Y64 = torch.randn(a.n, a.m, device="cuda", generator=g, dtype=torch.float64)
        sd64 = sd.double()
        G = torch.empty(a.m, a.m, dtype=torch.float64, device="cuda")
        ms = timed(lambda: gram_device(Y64.data_ptr(), a.n, a.m, sd64.data_ptr(), G.data_ptr(), FP64))
        fl = 2.0 * a.n * a.m * (a.m + 1) / 2
        out["gram64"] = {"ms": round(ms, 3), "tflops": round(fl / ms / 1e9, 2),
                         "frac_of_nominal_fp64": round(fl / ms / 1e9 / 37.0, 3)}
    print(json.dumps(out))


if __name__ == "__main__":
    main()
