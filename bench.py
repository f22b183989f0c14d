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

`hooi` (N = 1 only) is the HOOI headline on the learned-start workload
(order 5, n = 200,000, 20M power-law tuples, r = 16): plain FP64 HOOI from
the random start against mixed precision from the learned and the random
start, each timed to |delta error| < 1e-6 from the host tuple arrays (tensor
build included, file I/O excluded; the median of three runs per arm), with
each arm's objective gap, largest
principal angle and ||C||^2 error against the FP64 arm, the FP32 S3TTMc's
relative Frobenius error of Y, and that tensor's FP32 / FP64 S3TTMc rates.

--impl reference times the reference's own OpenMP CPU S3TTMc (oracle/_ref,
built from the reference sources) on the same workload and `config`: the
whole workload when the host has the memory for the reference's level
arrays, else a bounded sample of it (said in `cpu_baseline.sample`).
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
REF_SAMPLE_NNZ = 1_000_000  # reference arm sample when the host cannot hold the whole workload
CPU_SAMPLE_NNZ = 1_000_000  # cpu_baseline sample (reference tree build ~13 s, ~2 s per call)


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


def workload_config(order, n, nnz, levels, ws, s=8):
    """The `config` object of both arms' lines (the same workload, the same
    algorithmic units; s = bytes per scalar)."""
    m = msize(RANK, order - 1)
    return {"workload": f"{WORKLOAD}: {WORKLOADS[WORKLOAD][1]}, nnz={nnz}, R={RANK}, Y packed n x {m}",
            "parallelism": f"replicas x{ws}", "levels": levels,
            "alg_bytes_per_step": alg_bytes(order, n, nnz, RANK, levels, s),
            "alg_flops_per_step": alg_flops(order, nnz, RANK, levels),
            "l2": f"inputs larger than L2 (126 MB): Y is {n * m * s / 1e9:.2f} GB per step"}


def reference_footprint_bytes(order, n, levels):
    """Host memory the reference's S3TTMc allocates on a tensor with these
    tree levels (src/compressed_dtree.cpp:421-518): its level arrays of
    sizes 2..N-1 (FP64, the last one allocated though unused), the packed Y
    and about 1 KB per level-2 node for the tree itself."""
    arrays = sum(levels[L - 1] * msize(RANK, L) for L in range(2, order))
    return 8.0 * (arrays + n * msize(RANK, order - 1)) + 1024.0 * sum(levels)


def run_ref_probe(order, n, t, v, reps):
    """The reference's own OpenMP S3TTMc (oracle/_ref/ref_probe, built from its
    sources) on every host core: (per-call ms list, build ms, threads)."""
    from symprop_b200 import synth
    probe = os.path.join(ROOT, "oracle", "_ref", "ref_probe")
    with tempfile.TemporaryDirectory() as tmp:
        spt = os.path.join(tmp, "x.spt")
        synth.write_spt(spt, order, n, t, v)
        env = dict(os.environ, OMP_NUM_THREADS=str(os.cpu_count() or 1))
        out = subprocess.run([probe, "time", spt, str(RANK), str(reps), "1"], check=True,
                             capture_output=True, text=True, env=env).stdout
    js = json.loads(out.strip().splitlines()[-1])
    return js["s3ttmc_ms"], js["build_ms"], int(js["threads"])


def run_reference(args):
    """Reference arm: the reference's own CPU S3TTMc on this arm's workload.
    The whole workload runs when the host can hold the reference's level
    arrays (about 100 GB on the order-4 workload, where the unused last level
    alone is 87 GB); otherwise each step is a bounded sample of the same
    distribution, said in `cpu_baseline.sample`."""
    ws, rank, _ = dist_env()
    if rank != 0:
        return 0
    from symprop_b200 import synth
    if not os.path.exists(os.path.join(ROOT, "oracle", "_ref", "ref_probe")):
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref/ref_probe not built"}))
        return 0
    if WORKLOAD != "s3ttmc_order4_zipf":
        print(json.dumps({"impl": "reference", "unavailable": "the reference arm times the order-4 S3TTMc "
                          "workload only (the reference materialises the level N-2 array: OOM at order 5/6)"}))
        return 0
    order, n, t, v = synth.workload(WORKLOAD)
    nnz_full = t.shape[0]
    levels_full = tree_levels_cpu(order, n, t, v)
    config = workload_config(order, n, nnz_full, levels_full, ws)
    need = reference_footprint_bytes(order, n, levels_full)
    avail = host_mem_gb("MemAvailable") * 1e9
    full = need * 1.25 < avail
    if full:
        sample = (f"the whole workload ({nnz_full} tuples) each step: the host has {avail / 1e9:.0f} GB "
                  f"available against the reference's {need / 1e9:.0f} GB")
        levels = levels_full
    else:
        keep = REF_SAMPLE_NNZ
        t, v = t[:keep], v[:keep]
        levels = tree_levels_cpu(order, n, t, v)
        sample = (f"the first {keep} of the workload's {nnz_full} tuples each step: the whole workload "
                  f"needs {need / 1e9:.0f} GB of host memory for the reference's level arrays, "
                  f"{avail / 1e9:.0f} GB are available")
    ms, build_ms, threads = run_ref_probe(order, n, t, v, args.warmup + args.steps)
    B = alg_bytes(order, n, t.shape[0], RANK, levels, 8)
    ms_step = float(np.mean(ms[args.warmup:]))
    val = B / (ms_step * 1e-3) / 1e9
    line = {"impl": "reference", "metric": METRIC, "value": round(val, 4), "unit": "GB/s",
            "n_gpus": ws, "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(ms_step, 3),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic (seeded generator of the workload; no dataset is shipped)",
            "config": config,
            "cpu_baseline": {"value": round(val, 4), "unit": "GB/s", "cores": threads, "kind": "reference",
                             "sample": f"{sample}; S3TTMc (packed Y) per step, the tree build "
                                       f"({build_ms:.0f} ms) excluded as in the GPU arm"},
            "e2e": {"value": round(val, 4), "unit": "GB/s", "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0}}
    print(json.dumps(line))
    return 0


def tree_levels_cpu(order, n, t, v):
    """CompressedDTree level sizes: the number of unique sorted sub-multisets
    of each size 1..N-1 of the tuples."""
    from itertools import combinations
    from symprop_b200 import synth
    levels = []
    for L in range(1, order):
        subs = np.concatenate([t[:, list(c)] for c in combinations(range(order), L)], axis=0)
        levels.append(int(synth._unique_rows(np.ascontiguousarray(subs)).shape[0]))
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
    ap.add_argument("--no-hooi", action="store_true", help="skip the HOOI time-to-tolerance leg")
    ap.add_argument("--hooi-scale", type=float, default=1.0,
                    help="fraction of the HOOI workload's tuples (small cases for testing only)")
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
    owners = X.owner_count()
    owner_gb = owners * (4 * (-(-(order - 1) // 4) * 4) + s) / 1e9
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
    os.sched_setaffinity(0, cpus_before)
    if rank == 0 and ws == 1 and not args.no_cpu_baseline and WORKLOAD == "s3ttmc_order4_zipf":
        cpu = cpu_baseline()  # every host core
    hooi = None
    if rank == 0 and ws == 1 and not args.no_hooi:
        # one GPU: the HOOI headline is a single-device time to tolerance
        X.close()
        del dY, dU, hY, hU
        torch.cuda.empty_cache()
        hooi = hooi_leg(args.hooi_scale)
    if rank == 0:
        line = {
            "metric": METRIC, "value": round(value, 2), "unit": "GB/s", "n_gpus": ws,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(ms_step, 4),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f64" if prec == sp.FP64 else "f32",
            "data": "synthetic (seeded generator of the workload; no dataset is shipped)",
            "config": workload_config(order, n, nnz, levels, ws, s),
            "layout": {"owners_after_merge": owners, "owner_list_gb": round(owner_gb, 3),
                       "u_mb": round(n * RANK * s / 1e6, 1), "build_ms": round(build_ms, 1),
                       "note": "U is L2-resident within a step by design"},
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
        if hooi:
            line["hooi"] = hooi
        print(json.dumps(line))
    if ws > 1:
        torch.distributed.barrier()
        torch.distributed.destroy_process_group()
    return 0


HOOI_WORKLOAD = "learned_order5_powerlaw"
HOOI_RANK, HOOI_TOL, HOOI_DELTA, HOOI_MAX_ITER = 16, 1e-6, 1.0, 100
HOOI_REPEATS = 3  # runs per arm; the median is reported (host stalls on a shared box move single runs)


def _rel_frobenius(A, B, rows_per_chunk=8192):
    """||A - B||_F / ||B||_F over two device matrices, in FP64, by row chunks."""
    import torch
    num = den = 0.0
    for r0 in range(0, B.shape[0], rows_per_chunk):
        a = A[r0:r0 + rows_per_chunk].double()
        b = B[r0:r0 + rows_per_chunk].double()
        num += float(((a - b) ** 2).sum())
        den += float((b ** 2).sum())
    return math.sqrt(num / den) if den > 0 else 0.0


def hooi_leg(scale: float = 1.0):
    """HOOI time to |delta error| < 1e-6 on the learned-start workload (order 5,
    n = 200,000, 20M power-law tuples with 16 planted communities, r = 16,
    Y n x 3876): plain FP64 from the random start (the drop-in) against mixed
    precision (FP32 S3TTMc, tcgen05 split-BF16 dense products, FP64 solves)
    from the learned start and from the random start.

    Each arm is timed from the host tuple arrays to the returned
    decomposition: tensor build (copy + device build), the learned start's
    prediction where it has one, and the solve, with the device synchronised
    on both sides.  The arms' errors are stated against the FP64 arm: the
    objective gap, the largest principal angle between the factors and the
    relative error of ||C||^2; the FP32 S3TTMc's relative Frobenius error of
    Y is measured against the FP64 S3TTMc on the FP64 arm's final factor.
    The same tensor's FP32 and FP64 S3TTMc are timed with CUDA events (the
    order-5 bar of 0.6 of the HBM roofline is stated on the FP32 one)."""
    import torch
    import symprop_b200 as sp
    from symprop_b200 import synth
    from symprop_b200.warmstart import WarmStartModel

    t_gen = time.perf_counter()
    order, n, t, v = synth.workload(HOOI_WORKLOAD, scale=scale)
    gen_s = time.perf_counter() - t_gen
    nnz = t.shape[0]
    R = HOOI_RANK
    m = sp.symtens_size(R, order - 1)
    model = WarmStartModel.load(os.path.join(ROOT, "symprop_b200", f"warmstart_r{R}.npz"))
    kw = dict(rank=R, max_iter=HOOI_MAX_ITER, rel_tol=HOOI_TOL, delta=HOOI_DELTA, seed=0)

    # warm-up (untimed): module loading, the library's scratch pools and the
    # prediction path, one iteration per precision
    X = sp.SpSymtensor(n, order, t, v)
    X.TuckerHOOI(**dict(kw, max_iter=1))
    X.TuckerHOOI(**dict(kw, max_iter=1, precision=sp.PREC_MIXED))
    model.predict(X, seed=0)
    X.close()
    del X
    torch.cuda.synchronize()

    def run_arm(precision, learned):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        Xa = sp.SpSymtensor(n, order, t, v)
        torch.cuda.synchronize()
        t1 = time.perf_counter()
        extra = {}
        if learned:
            U0 = model.predict(Xa, seed=0)
            t2 = time.perf_counter()
            extra["prediction_ms"] = round((t2 - t1) * 1e3, 1)
            d = Xa.TuckerHOOI(**dict(kw, precision=precision, init="user", init_factor=U0))
        else:
            d = Xa.TuckerHOOI(**dict(kw, precision=precision))
        torch.cuda.synchronize()
        wall = (time.perf_counter() - t0) * 1e3
        row = {"ms": round(wall, 1), "build_ms": round((t1 - t0) * 1e3, 1),
               "solve_device_ms": round(d.time_ms, 1), "s3ttmc_ms": round(d.s3ttmc_ms, 1),
               "dense_ms": round(d.dense_ms, 1), "iterations": int(d.iterations), "error": d.error}
        row.update(extra)
        return Xa, d, row

    def run_median(precision, learned):
        """HOOI_REPEATS runs of an arm (each from the host tuples: build,
        prediction, solve); the run of median wall time is reported, with
        every run's wall time in repeats_ms.  Returns the last run's tensor
        (all runs build the same one)."""
        runs = []
        for k in range(HOOI_REPEATS):
            Xa, d, row = run_arm(precision, learned)
            runs.append((row["ms"], d, row))
            if k + 1 < HOOI_REPEATS:
                Xa.close()
        med = sorted(runs, key=lambda x: x[0])[len(runs) // 2]
        row = dict(med[2], repeats_ms=[r[0] for r in runs])
        return Xa, med[1], row

    out = {"workload": f"{HOOI_WORKLOAD}: order {order}, n={n}, {nnz} tuples, power-law degrees "
                       f"(exponent 2.1), 16 planted communities (80% inside), values 1.0; rank {R} "
                       f"(Y n x {m}); stop at |delta error| < {HOOI_TOL:g}; delta {HOOI_DELTA:g}; seed 0",
           "timing": "wall clock per arm with the device synchronised on both sides, from host tuple "
                     "arrays: tensor build (copy + device build) + prediction (learned arm) + solve; "
                     f"the median of {HOOI_REPEATS} runs per arm (repeats_ms lists all); "
                     "file I/O and the seeded generator excluded",
           "generator_s": round(gen_s, 1)}
    with ClockSampler(torch.cuda.current_device()) as clk:
        X64, d64, r64 = run_median(sp.PREC_FP64, False)
        U64 = d64.factor.copy()
        X64.close()
        del X64
        arms = {"fp64_random": r64}
        for name, prec, learned in (("mixed_learned", sp.PREC_MIXED, True),
                                    ("mixed_random", sp.PREC_MIXED, False)):
            Xa, d, row = run_median(prec, learned)
            sv = np.linalg.svd(U64.T @ d.factor, compute_uv=False)
            row["objective_rel_gap_vs_fp64"] = (d.error - d64.error) / d64.error
            row["max_principal_angle_vs_fp64"] = float(np.arccos(np.clip(sv.min(), -1.0, 1.0)))
            row["core_norm_sq_rel_err_vs_fp64"] = abs(d.core_norm ** 2 - d64.core_norm ** 2) / d64.core_norm ** 2
            row["speedup_vs_fp64_random"] = round(r64["ms"] / row["ms"], 3)
            arms[name] = row
            if name == "mixed_random":
                X = Xa
            else:
                Xa.close()
        out["arms"] = arms

        # S3TTMc of this tensor: FP32 (the mixed path's) and FP64, device-timed
        levels = [int(x) for x in X.tree_level_sizes()]
        stream = torch.cuda.current_stream()
        dU64 = torch.from_numpy(U64).cuda().contiguous()
        dU32 = dU64.float().contiguous()
        res = {}
        Ys = {}
        for prec, name, dU, dt, s in ((sp.FP32, "s3ttmc_fp32", dU32, torch.float32, 4),
                                      (sp.FP64, "s3ttmc_fp64", dU64, torch.float64, 8)):
            dY = torch.empty((n, m), dtype=dt, device="cuda")
            for _ in range(3):
                X.s3ttmc_device(dU.data_ptr(), R, dY.data_ptr(), True, prec, stream.cuda_stream)
            steps = 5
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            torch.cuda.synchronize()
            e0.record(stream)
            for _ in range(steps):
                X.s3ttmc_device(dU.data_ptr(), R, dY.data_ptr(), True, prec, stream.cuda_stream)
            e1.record(stream)
            torch.cuda.synchronize()
            ms = e0.elapsed_time(e1) / steps
            B = alg_bytes(order, n, nnz, R, levels, s)
            peak, peak_kind = load_peaks()
            res[name] = {"ms": round(ms, 3), "alg_gbs": round(B / (ms * 1e-3) / 1e9, 1),
                         "frac": round(B / (ms * 1e-3) / 1e9 / peak, 4), "peak_gbs": peak,
                         "peak_kind": peak_kind, "alg_bytes": B}
            Ys[name] = dY
        out.update(res)
        out["y_fp32_rel_frobenius_vs_fp64"] = _rel_frobenius(Ys["s3ttmc_fp32"], Ys["s3ttmc_fp64"])
        out["levels"] = levels
        del Ys
        X.close()
    out["clocks"] = clk.summary()
    lm, ll = arms["mixed_learned"], arms["mixed_random"]
    out["summary"] = {
        "fp64_random_ms": r64["ms"], "mixed_learned_ms": lm["ms"], "mixed_random_ms": ll["ms"],
        "speedup_mixed_learned_vs_fp64": lm["speedup_vs_fp64_random"],
        "speedup_mixed_random_vs_fp64": ll["speedup_vs_fp64_random"],
        "mixed_learned_reaches_fp64_objective": bool(lm["error"] <= d64.error * (1 + HOOI_TOL)),
    }
    # the reference's own HOOI on this workload: what its schedule holds in
    # host memory at least (the unpacked Y, and the two consecutive tree
    # levels alive at once in its S3TTMc level loop, FP64)
    pair = max(levels[L - 2] * msize(R, L - 1) + levels[L - 1] * msize(R, L) for L in range(2, order))
    need = 8.0 * (n * R ** (order - 1) + pair)
    svd_flops = 4.0 * n * float(R ** (order - 1)) ** 2  # dgesvd of the unpacked n x R^(N-1) Y
    total = host_mem_gb()
    why = (f"OOM: the reference's HOOI holds at least {need / 1e9:.0f} GB in FP64 (the unpacked Y and two "
           f"materialised tree levels), host memory {total:.0f} GB" if not need < total * 1e9 else
           f"its leftsvd is a dgesvd of the unpacked {n} x {R ** (order - 1)} Y (about {svd_flops:.1e} "
           f"flops per iteration) on {need / 1e9:.0f} GB")
    out["reference_cpu"] = {"unavailable": f"infeasible on host: {why}", "cores": os.cpu_count()}
    return out


def host_mem_gb(field="MemTotal"):
    try:
        for line in open("/proc/meminfo"):
            if line.startswith(field + ":"):
                return int(line.split()[1]) / 1e6
    except OSError:
        pass
    return float("nan")


def cpu_baseline():
    """The reference's own OpenMP S3TTMc on every host core, on a bounded sample
    of the workload (its first CPU_SAMPLE_NNZ tuples, about 10-30 s of CPU
    work with the reference's tree build)."""
    from symprop_b200 import synth
    if not os.path.exists(os.path.join(ROOT, "oracle", "_ref", "ref_probe")):
        return None
    order, n, t, v = synth.workload(WORKLOAD)
    t, v = t[:CPU_SAMPLE_NNZ], v[:CPU_SAMPLE_NNZ]
    try:
        ms, build_ms, threads = run_ref_probe(order, n, t, v, 4)
    except Exception as e:  # noqa: BLE001
        return {"value": None, "unit": "GB/s", "cores": os.cpu_count(), "kind": "reference",
                "sample": f"failed: {e}"}
    step = float(np.mean(ms[1:]))
    B = alg_bytes(order, n, t.shape[0], RANK, tree_levels_cpu(order, n, t, v), 8)
    return {"value": round(B / (step * 1e-3) / 1e9, 4), "unit": "GB/s", "cores": threads, "kind": "reference",
            "sample": f"the first {t.shape[0]} tuples of the workload (order 4, n={n}, Zipf(1.1)), R={RANK} "
                      f"packed S3TTMc, mean of 3 calls after one warm-up = {step:.1f} ms; tree build "
                      f"{build_ms:.0f} ms excluded"}


if __name__ == "__main__":
    sys.exit(main())
