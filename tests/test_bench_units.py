"""CPU checks of bench.py's algorithmic units against the worked values of
the roofline definition: bytes B = s*(2*sum_{L=2}^{N-2} l_L m_L + n m + n r)
+ 4 N nnz + s nnz + sum_{L=2}^{N-1} l_L (4 + 4L) + omega (4 + s) and flops
F = 2*sum_{L=2}^{N-1} l_L L m_L + 2 omega m, evaluated at the level sizes
measured for the three S3TTMc configurations (order 5 / n 250 / 10k
tuples / r 8; order 4 / n 100k / 5M tuples / r 16; order 6 / n 50k / 2M
tuples / r 10).  These are the units `value` and `roofline.achieved` use."""
import os
import sys

import pytest

sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
import bench  # noqa: E402


def test_order4_units():
    lv = [100_000, 7_788_501, 13_448_292]
    assert bench.alg_bytes(4, 100_000, 5_000_000, 16, lv, 4) / 1e9 == pytest.approx(9.4, abs=0.05)
    assert bench.alg_bytes(4, 100_000, 5_000_000, 16, lv, 8) / 1e9 == pytest.approx(18.3, abs=0.05)
    assert bench.alg_flops(4, 5_000_000, 16, lv) / 1e9 == pytest.approx(103, abs=0.5)


def test_order5_small_units():
    lv = [250, 9_869, 31_777, 31_182]
    assert bench.alg_bytes(5, 250, 10_000, 8, lv, 8) / 1e9 == pytest.approx(0.07, abs=0.005)
    assert bench.alg_flops(5, 10_000, 8, lv) / 1e9 == pytest.approx(0.14, abs=0.005)


def test_order6_units():
    lv = [50_000, 28.1e6, 40.0e6, 30.0e6, 12.0e6]  # level sizes known to three digits
    assert bench.alg_bytes(6, 50_000, 2_000_000, 10, lv, 4) / 1e9 == pytest.approx(255, rel=0.01)
    assert bench.alg_flops(6, 2_000_000, 10, lv) / 1e9 == pytest.approx(519, rel=0.005)


def test_packed_sizes():
    assert [bench.msize(r, L) for r, L in [(16, 3), (16, 4), (10, 5), (8, 4)]] == [816, 3876, 2002, 330]


def test_numa_binding_leaves_the_process_alone_without_a_gpu():
    """bench.bind_near_gpu moves the process to the GPU's NUMA node through
    NVML; with no GPU (or no NVML) it changes nothing and says so."""
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is visible: the binding would apply")
    before = os.sched_getaffinity(0)
    note, prev = bench.bind_near_gpu(0)
    assert note.startswith("unchanged") and prev == before
    assert os.sched_getaffinity(0) == before
