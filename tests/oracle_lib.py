"""ctypes bindings of the C oracle (oracle/s3ttmc_oracle.c) for the tests.

The oracle is the checker: tests compare the CUDA path with it; nothing in
the product imports this module."""
import ctypes
import os

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
ORACLE_SO = os.path.join(ROOT, "oracle", "liboracle.so")
REF_PROBE = os.path.join(ROOT, "oracle", "_ref", "ref_probe")
REF_CLI = os.path.join(ROOT, "oracle", "_ref", "symtucker")

_P = ctypes.c_void_p
_lib = None


def olib():
    global _lib
    if _lib is None:
        if not os.path.exists(ORACLE_SO):
            import subprocess
            subprocess.run(["make", "-C", os.path.join(ROOT, "oracle"), "oracle"], check=True,
                           capture_output=True)
        L = ctypes.CDLL(ORACLE_SO)
        L.orc_tree_build.restype = _P
        L.orc_tree_build.argtypes = [ctypes.c_uint32, ctypes.c_uint32, ctypes.c_uint64, _P, _P]
        L.orc_tree_level_size.restype = ctypes.c_uint64
        L.orc_tree_level_size.argtypes = [_P, ctypes.c_int]
        L.orc_tree_nowners.restype = ctypes.c_uint64
        L.orc_tree_nowners.argtypes = [_P]
        L.orc_tree_copy_level.argtypes = [_P, ctypes.c_int, _P, _P, _P, _P]
        L.orc_tree_copy_owners.argtypes = [_P, _P, _P]
        L.orc_tree_free.argtypes = [_P]
        L.orc_symtens_size.restype = ctypes.c_uint64
        L.orc_symtens_size.argtypes = [ctypes.c_uint64, ctypes.c_uint64]
        L.orc_binomial.restype = ctypes.c_uint64
        L.orc_binomial.argtypes = [ctypes.c_uint64, ctypes.c_uint64]
        L.orc_norm.restype = ctypes.c_double
        L.orc_norm.argtypes = [ctypes.c_uint32, ctypes.c_uint64, _P, _P]
        L.orc_s3ttmc.restype = ctypes.c_int
        L.orc_s3ttmc.argtypes = [ctypes.c_uint32, ctypes.c_uint32, ctypes.c_uint64, _P, _P,
                                 ctypes.c_uint32, _P, ctypes.c_int, _P]
        L.orc_packed_offset.restype = ctypes.c_uint64
        L.orc_packed_offset.argtypes = [_P, ctypes.c_int, ctypes.c_uint32]
        L.orc_packed_indices.argtypes = [ctypes.c_uint32, ctypes.c_int, _P]
        L.orc_symtens_coeff.argtypes = [ctypes.c_uint32, ctypes.c_int, _P]
        L.orc_sym_outer_prod.argtypes = [_P, _P, _P, ctypes.c_uint32, ctypes.c_int]
        L.orc_unpack.argtypes = [_P, ctypes.c_uint32, ctypes.c_int, _P]
        L.orc_s3ttmc_rows.restype = ctypes.c_int
        L.orc_s3ttmc_rows.argtypes = [ctypes.c_uint32, ctypes.c_uint32, ctypes.c_uint64, _P, _P,
                                      ctypes.c_uint32, _P, ctypes.c_uint64, _P, _P]
        L.orc_multinomial_sorted.restype = ctypes.c_uint64
        L.orc_multinomial_sorted.argtypes = [_P, ctypes.c_int]
        _lib = L
    return _lib


def p(a):
    return ctypes.c_void_p(a.ctypes.data)


def s3ttmc(order, dim, inds, vals, U, R, packed=True):
    L = olib()
    inds = np.ascontiguousarray(inds, np.uint32)
    vals = np.ascontiguousarray(vals, np.float64)
    U = np.ascontiguousarray(U, np.float64)
    cols = L.orc_symtens_size(R, order - 1) if packed else R ** (order - 1)
    Y = np.zeros((dim, cols))
    st = L.orc_s3ttmc(order, dim, vals.shape[0], p(inds), p(vals), R, p(U), int(packed), p(Y))
    assert st == 0
    return Y


def s3ttmc_rows(order, dim, inds, vals, U, R, rows):
    """Packed Y of the oracle on the listed rows only (0-based, distinct):
    len(rows) x C(R+N-2, N-1)."""
    L = olib()
    inds = np.ascontiguousarray(inds, np.uint32)
    vals = np.ascontiguousarray(vals, np.float64)
    U = np.ascontiguousarray(U, np.float64)
    rows = np.ascontiguousarray(rows, np.uint32)
    Y = np.zeros((rows.shape[0], L.orc_symtens_size(R, order - 1)))
    st = L.orc_s3ttmc_rows(order, dim, vals.shape[0], p(inds), p(vals), R, p(U), rows.shape[0], p(rows), p(Y))
    assert st == 0, st
    return Y


def tree(order, dim, inds, vals):
    L = olib()
    inds = np.ascontiguousarray(inds, np.uint32)
    vals = np.ascontiguousarray(vals, np.float64)
    T = L.orc_tree_build(order, dim, vals.shape[0], p(inds), p(vals))
    out = {"level_idx": [], "level_ptr": [], "dep_list": [], "keys": []}
    for l in range(order - 1):
        n = L.orc_tree_level_size(T, l)
        idx = np.zeros(n, np.uint32)
        ptr = np.zeros(n + 1, np.uint64)
        dep = np.zeros(max(n * (l + 1), 1), np.uint64)
        keys = np.zeros(max(n * (l + 1), 1), np.uint32)
        L.orc_tree_copy_level(T, l, p(idx), p(ptr), p(dep), p(keys))
        out["level_idx"].append(idx)
        out["level_ptr"].append(ptr)
        out["dep_list"].append(dep[: n * (l + 1)] if l >= 1 else np.zeros(0, np.uint64))
        out["keys"].append(keys[: n * (l + 1)].reshape(n, l + 1))
    no = L.orc_tree_nowners(T)
    rem = np.zeros(no, np.uint64)
    val = np.zeros(no)
    L.orc_tree_copy_owners(T, p(rem), p(val))
    out["rem"], out["val"] = rem, val
    L.orc_tree_free(T)
    return out


def norm(order, inds, vals):
    inds = np.ascontiguousarray(inds, np.uint32)
    vals = np.ascontiguousarray(vals, np.float64)
    return olib().orc_norm(order, vals.shape[0], p(inds), p(vals))


def packed_indices(dim, order):
    m = olib().orc_symtens_size(dim, order)
    out = np.zeros(m * order, np.uint32)
    olib().orc_packed_indices(dim, order, p(out))
    return out.reshape(m, order)


def symtens_coeff(dim, order):
    c = np.zeros(olib().orc_symtens_size(dim, order))
    olib().orc_symtens_coeff(dim, order, p(c))
    return c
