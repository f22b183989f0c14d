#!/usr/bin/env python
"""Benchmark: S3TTMc throughput in algorithmic GB/s on one B200 per rank.

Workload (the S3TTMc-alone configuration): order-4 sparse symmetric tensor,
n = 100,000, 5,000,000 unique sorted tuples with ids ~ Zipf(1.1), values
uniform (0,1]; U = QR(Gaussian n x 16); Y is n x C(18,3) = 816 packed
columns.  Synthetic data from a seeded generator (no dataset is shipped).

A step is one S3TTMc call over the whole tensor (U and the owner list
resident in HBM; Y written to HBM).  `value` is algorithmic bytes / device
time, the algorithmic bytes being the reference's level-materialising
schedule written once and read once:
    B = s*(2*sum_{L=2}^{N-2} l_L m_L + n m + n r) + 4 N nnz + s nnz
        + sum_{L=2}^{N-1} l_L (4 + 4L) + omega (4 + s)
with l_L the CompressedDTree level sizes, m_L = C(r+L-1, L), omega = N*nnz.
`e2e` is the same metric through the host-pointer C ABI call
(symprop_s3ttmc: U host->device, kernels, Y device->host each step), with
the pinned host buffers allocated while the process runs on the GPU's NUMA
node (NVML's CPU affinity; `e2e.host_cpus`); `e2e.y_copy_alone_ms` is one
plain copy of Y to the host, the floor the overlapped call approaches.

--impl reference times the reference's own OpenMP CPU S3TTMc (oracle/_ref,
built from the reference sources) on a bounded sample of the same workload.
Multi-GPU (torchrun): every rank runs its own replica of the workload
(independent tensors, no collective on the data path): weak scaling.
"""
from __future__ import annotations

import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import tempfile
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

WORKLOAD = "s3ttmc_order4_zipf"
RANK = 16
# --workload choices: the S3TTMc-alone workload (the default bench line) and
# the S3TTMc of the two HOOI workloads with wide packed rows
WORKLOADS = {
    "s3ttmc_order4_zipf": (16, "order 4, n=100000, 5M tuples, Zipf(1.1), values uniform (0,1]"),
    "learned_order5_powerlaw": (16, "order 5, n=200000, 20M tuples, power-law degrees (exponent 2.1), "
                                    "16 planted communities, values 1.0"),
    "mixed_order6_planted": (10, "order 6, n=50000, 2M tuples, 8 planted communities (80% inside), "
                                 "values 1.0"),
}
METRIC = "S3TTMc algorithmic GB/s"
REF_SAMPLE_NNZ = 250_000   # bounded sample for the CPU reference (~1 s per call on 8 cores)


def binom(n, k):
    return math.comb(n, k) if 0 <= k <= n else 0


def msize(r, L):
    return binom(r + L - 1, L)


def alg_bytes(order, n, nnz, r, levels, s):
    """levels[l] = size of CompressedDTree level l (multisets of size l+1)."""
    N = order
    ell = {l + 1: levels[l] for l in range(len(levels))}
    omega = N * nnz
    b = 0.0
    for L in range(2, N - 1):
        b += 2 * ell[L] * msize(r, L)
    b += n * msize(r, N - 1) + n * r
    b *= s
    b += 4 * N * nnz + s * nnz
    for L in range(2, N):
        b += ell[L] * (4 + 4 * L)
    b += omega * (4 + s)
    return b


def alg_flops(order, nnz, r, levels):
    N = order
    ell = {l + 1: levels[l] for l in range(len(levels))}
    f = 0.0
    for L in range(2, N):
        f += 2 * ell[L] * L * msize(r, L)
    f += 2 * N * nnz * msize(r, N - 1)
    return f


class ClockSampler:
    """nvidia-smi clock/throttle sampling during the timed region."""

    def __init__(self, index: int):
        self.index = index
        self.proc = None
        self.path = None

    def __enter__(self):
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.index}", f"--query-gpu={q}", "--format=csv,noheader,nounits",
                 "-lms", "100"], stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None
        time.sleep(0.3)
        return self

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        if not self.path or not os.path.exists(self.path):
            return None
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in open(self.path):
            f = [x.strip() for x in line.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx.append(float(f[2]))
            except ValueError:
                continue
            for nm, v in zip(names, f[5:9]):
                if v.lower() == "active":
                    reasons.add(nm)
        os.unlink(self.path)
        if not sm:
            return None
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": max(mx), "reasons": sorted(reasons),
                "samples": len(sm)}


def load_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        d = json.load(open(p))
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def load_traffic(precision, workload, scale):
    """DRAM bytes per launch of the dominant kernel from the committed ncu
    summary (profiles/) of this workload at full size, or None."""
    p = os.path.join(ROOT, "profiles", f"{workload}_traffic.json")
    if scale == 1.0 and os.path.exists(p):
        d = json.load(open(p))
        return d.get(precision)
    return None


def max_over_ranks(x: float, device: str = "cuda") -> float:
    """The largest x over the ranks of the default process group (x itself
    when there is none): every timing of a multi-rank run is the slowest
    rank's."""
    import torch
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return float(x)
    t = torch.tensor([float(x)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def bind_near_gpu(device: int):
    """Runs this process on the CPUs NVML names as local to the GPU, so that
    the pinned host buffers of the e2e leg sit on the GPU's NUMA node.
    Returns (note for the JSON line, the previous CPU set to restore)."""
    before = os.sched_getaffinity(0)
    try:
        import pynvml
        import torch
        pynvml.nvmlInit()
        p = torch.cuda.get_device_properties(device)
        bus = f"{p.pci_domain_id:08x}:{p.pci_bus_id:02x}:{p.pci_device_id:02x}.0"
        h = pynvml.nvmlDeviceGetHandleByPciBusId(bus)
        words = pynvml.nvmlDeviceGetCpuAffinity(h, 64)
        cpus = {w * 64 + b for w, mask in enumerate(words) for b in range(64) if (mask >> b) & 1} & before
        if cpus and cpus != before:
            os.sched_setaffinity(0, cpus)
            return f"{len(cpus)} of {len(before)} host CPUs (the GPU's NUMA node)", before
        return f"all {len(before)} host CPUs (all local to the GPU)", before
    except Exception as e:  # no NVML or no PCI id: leave the process where it is
        return f"unchanged ({type(e).__name__})", before


def dist_env():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return ws, rank, local


def run_reference(args):
    ws, rank, _ = dist_env()
    if rank != 0:
        return 0
    from symprop_b200 import synth
    probe = os.path.join(ROOT, "oracle", "_ref", "ref_probe")
    if not os.path.exists(probe):
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref/ref_probe not built"}))
        return 0
    if WORKLOAD != "s3ttmc_order4_zipf":
        print(json.dumps({"impl": "reference", "unavailable": "the reference arm times the order-4 S3TTMc "
                          "workload only (the reference materialises the level N-2 array: OOM at order 5/6)"}))
        return 0
    order, n, t, v = synth.workload(WORKLOAD, scale=REF_SAMPLE_NNZ / 5_000_000)
    nnz = t.shape[0]
    tmp = tempfile.mkdtemp()
    spt = os.path.join(tmp, "x.spt")
    synth.write_spt(spt, order, n, t, v)
    cores = os.cpu_count() or 1
    env = dict(os.environ, OMP_NUM_THREADS=str(cores))
    reps = args.warmup + args.steps
    out = subprocess.run([probe, "time", spt, str(RANK), str(reps), "1"], check=True,
                         capture_output=True, text=True, env=env).stdout
    js = json.loads(out.strip().splitlines()[-1])
    ms = js["s3ttmc_ms"][args.warmup:]
    levels = tree_levels_cpu(order, n, t, v)
    B = alg_bytes(order, n, nnz, RANK, levels, 8)
    ms_step = float(np.mean(ms))
    val = B / (ms_step * 1e-3) / 1e9
    line = {"impl": "reference", "metric": METRIC, "value": round(val, 4), "unit": "GB/s",
            "n_gpus": ws, "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(ms_step, 3),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic (seeded generator)",
            "config": {"workload": f"{WORKLOAD}: {WORKLOADS[WORKLOAD][1]}, R={RANK}, packed Y",
                       "sample_nnz": nnz, "levels": levels},
            "cpu_baseline": {"value": round(val, 4), "unit": "GB/s", "cores": int(js["threads"]),
                             "kind": "reference",
                             "sample": f"{nnz} tuples of the workload's distribution (n={n}), "
                                       f"S3TTMc(packed) per step; build {js['build_ms']:.0f} ms excluded"},
            "e2e": {"value": round(val, 4), "unit": "GB/s", "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0}}
    print(json.dumps(line))
    return 0


def tree_levels_cpu(order, n, t, v):
    """Level sizes = counts of unique sorted sub-multisets (needed for B)."""
    levels = []
    from itertools import combinations
    for L in range(1, order):
        subs = [t[:, list(c)] for c in combinations(range(order), L)]
        allk = np.unique(np.concatenate(subs, axis=0), axis=0)
        levels.append(int(allk.shape[0]))
    return levels


def main():
    global WORKLOAD, RANK
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--precision", default="fp64", choices=["fp64", "fp32"])
    ap.add_argument("--e2e-steps", type=int, default=5)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--workload", default=WORKLOAD, choices=sorted(WORKLOADS))
    ap.add_argument("--scale", type=float, default=1.0,
                    help="fraction of the workload's tuples (small cases for profiling only)")
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    WORKLOAD = args.workload
    RANK = WORKLOADS[WORKLOAD][0]
    if args.impl == "reference":
        return run_reference(args)

    import torch
    import symprop_b200 as sp
    from symprop_b200 import synth

    ws, rank, local = dist_env()
    if ws > 1:
        import torch.distributed as dist
        from datetime import timedelta
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=timedelta(seconds=120))
    else:
        torch.cuda.set_device(0)
    sp.lib().symprop_set_device(torch.cuda.current_device())

    order, n, t, v = synth.workload(WORKLOAD, scale=args.scale, seed=1 + rank)
    nnz = t.shape[0]
    prec = sp.FP64 if args.precision == "fp64" else sp.FP32
    s = 8 if prec == sp.FP64 else 4
    dt = torch.float64 if prec == sp.FP64 else torch.float32
    t0 = time.perf_counter()
    X = sp.SpSymtensor(n, order, t, v)
    torch.cuda.synchronize()
    build_ms = (time.perf_counter() - t0) * 1e3
    # level sizes from the device CompressedDTree build (for the byte formula)
    levels = [int(x) for x in X.tree_level_sizes()]
    B = alg_bytes(order, n, nnz, RANK, levels, s)
    F = alg_flops(order, nnz, RANK, levels)
    m = sp.symtens_size(RANK, order - 1)

    g = torch.Generator(device="cpu").manual_seed(1234 + rank)
    U64, _ = torch.linalg.qr(torch.randn(n, RANK, generator=g, dtype=torch.float64))
    dU = U64.to(dt).cuda().contiguous()
    dY = torch.empty((n, m), dtype=dt, device="cuda")
    stream = torch.cuda.current_stream()
    launches_per_step = X.s3ttmc_launches(RANK, True)

    def step():
        X.s3ttmc_device(dU.data_ptr(), RANK, dY.data_ptr(), True, prec, stream.cuda_stream)

    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()
    if ws > 1:
        torch.distributed.barrier()
    with ClockSampler(torch.cuda.current_device()) as clk:
        torch.cuda.synchronize()
        ev0 = torch.cuda.Event(enable_timing=True)
        ev1 = torch.cuda.Event(enable_timing=True)
        ev0.record(stream)
        for _ in range(args.steps):
            step()
        ev1.record(stream)
        torch.cuda.synchronize()
    elapsed_ms = max_over_ranks(ev0.elapsed_time(ev1))
    ms_step = elapsed_ms / args.steps
    value = ws * B / (ms_step * 1e-3) / 1e9

    # e2e through the host-pointer C ABI (pinned host buffers on the GPU's
    # NUMA node)
    affinity, cpus_before = bind_near_gpu(torch.cuda.current_device())
    hU = torch.empty((n, RANK), dtype=dt).pin_memory()
    hU.copy_(U64.to(dt))
    hY = torch.empty((n, m), dtype=dt).pin_memory()
    import ctypes
    L = sp.lib()

    def e2e_step():
        st = L.symprop_s3ttmc(X.handle, ctypes.c_void_p(hU.data_ptr()), RANK, 1,
                              ctypes.c_void_p(hY.data_ptr()), prec)
        if st != 0:
            raise RuntimeError(L.symprop_last_error().decode())

    e2e_step()
    torch.cuda.synchronize()
    if ws > 1:
        torch.distributed.barrier()
    te = time.perf_counter()
    for _ in range(args.e2e_steps):
        e2e_step()
    e2e_ms = max_over_ranks((time.perf_counter() - te) * 1e3 / args.e2e_steps)
    e2e_val = ws * B / (e2e_ms * 1e-3) / 1e9
    # result check against the device result of the timed loop
    diff = float((hY.cuda() - dY).abs().max().item())
    # the copy of Y alone (the floor the overlapped e2e call approaches)
    torch.cuda.synchronize()
    tc = time.perf_counter()
    hY.copy_(dY)
    copy_ms = (time.perf_counter() - tc) * 1e3

    peak, peak_kind = load_peaks()
    achieved = B / (ms_step * 1e-3) / 1e9
    traffic = load_traffic(args.precision, WORKLOAD, args.scale)
    clocks = clk.summary()
    cpu = None
    if rank == 0 and ws == 1 and not args.no_cpu_baseline and WORKLOAD == "s3ttmc_order4_zipf":
        os.sched_setaffinity(0, cpus_before)  # the CPU baseline gets every host core
        cpu = cpu_baseline()
    if rank == 0:
        line = {
            "metric": METRIC, "value": round(value, 2), "unit": "GB/s", "n_gpus": ws,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(ms_step, 4),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f64" if prec == sp.FP64 else "f32",
            "data": "synthetic (seeded generator of the workload; no dataset is shipped)",
            "config": {"workload": f"{WORKLOAD}: {WORKLOADS[WORKLOAD][1]}, nnz={nnz}, R={RANK}, "
                                   f"Y packed n x {m}", "parallelism": f"replicas x{ws}",
                       "levels": levels, "owners_after_merge": X.owner_count(),
                       "alg_bytes_per_step": B, "alg_flops_per_step": F,
                       "l2": "inputs larger than L2 (owner list %.2f GB, Y %.2f GB); U (%.1f MB) is "
                             "L2-resident within a step by design"
                             % (X.owner_count() * (4 * (-(-(order - 1) // 4) * 4) + s) / 1e9, n * m * s / 1e9,
                                n * RANK * s / 1e6),
                       "build_ms": round(build_ms, 1)},
            "roofline": {"bound": "hbm", "achieved": round(achieved, 2), "peak": peak, "unit": "GB/s",
                         "frac": round(achieved / peak, 4), "traffic": traffic,
                         "peak_kind": peak_kind,
                         "fp_rate_tflops": round(F / (ms_step * 1e-3) / 1e12, 3)},
            "e2e": {"value": round(e2e_val, 2), "unit": "GB/s",
                    "h2d_bytes_per_step": int(n * RANK * s), "d2h_bytes_per_step": int(n * m * s),
                    "ms_per_step": round(e2e_ms, 3), "max_abs_diff_vs_device_path": diff,
                    "y_copy_alone_ms": round(copy_ms, 3), "host_cpus": affinity},
            "gpu_launches": int(launches_per_step * args.steps),
            "clocks": clocks,
        }
        if cpu:
            line["cpu_baseline"] = cpu
        print(json.dumps(line))
    if ws > 1:
        torch.distributed.barrier()
        torch.distributed.destroy_process_group()
    return 0


def cpu_baseline():
    """The reference's own OpenMP S3TTMc on a bounded sample (all host cores)."""
    from symprop_b200 import synth
    probe = os.path.join(ROOT, "oracle", "_ref", "ref_probe")
    if not os.path.exists(probe):
        return None
    order, n, t, v = synth.workload(WORKLOAD, scale=REF_SAMPLE_NNZ / 5_000_000)
    tmp = tempfile.mkdtemp()
    spt = os.path.join(tmp, "x.spt")
    synth.write_spt(spt, order, n, t, v)
    cores = os.cpu_count() or 1
    env = dict(os.environ, OMP_NUM_THREADS=str(cores))
    try:
        out = subprocess.run([probe, "time", spt, str(RANK), "4", "1"], check=True, capture_output=True,
                             text=True, env=env, timeout=600).stdout
    except Exception as e:  # noqa: BLE001
        return {"value": None, "unit": "GB/s", "cores": cores, "kind": "reference",
                "sample": f"failed: {e}"}
    js = json.loads(out.strip().splitlines()[-1])
    ms = float(np.mean(js["s3ttmc_ms"][1:]))
    levels = tree_levels_cpu(order, n, t, v)
    B = alg_bytes(order, n, t.shape[0], RANK, levels, 8)
    return {"value": round(B / (ms * 1e-3) / 1e9, 4), "unit": "GB/s", "cores": int(js["threads"]),
            "kind": "reference",
            "sample": f"{t.shape[0]} tuples drawn like the workload (order 4, n=100000, Zipf(1.1)), "
                      f"R=16 packed S3TTMc, mean of 3 calls = {ms:.1f} ms"}


if __name__ == "__main__":
    sys.exit(main())
