"""symprop_b200 — B200-native SymProp S3TTMc / Tucker path.

Python mirror of the reference's C++ interface (SpSymtensor, Config,
SymTuckerDecomp; include/detail/sparse/spsymtensor.hpp:24-65,
include/detail/tucker.hpp:14-45) over the C ABI in include/symprop.h
(libsymprop_b200.so, built in-tree by symprop_b200/Makefile).  Every compute
call runs on the GPU; there is no CPU fallback: if the library or a CUDA
device is missing the calls raise.
"""
from __future__ import annotations

import ctypes
import os
import subprocess
from dataclasses import dataclass, field

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
# SYMPROP_B200_LIB selects another build of the library, e.g. the
# bounds-checked libsymprop_b200_checked.so (make -C symprop_b200 checked)
LIB_PATH = os.environ.get("SYMPROP_B200_LIB") or os.path.join(HERE, "libsymprop_b200.so")
CLI_PATH = os.path.join(HERE, "symtucker")
TTMC_PATH = os.path.join(HERE, "symtens_ttmc")
TTMCTC_PATH = os.path.join(HERE, "s3ttmctc")

SYMPROP_OK = 0
ERR_INVALID, ERR_ORDER, ERR_OOM, ERR_CUDA, ERR_NOCONV, ERR_TIMEOUT, ERR_SIZE, ERR_NODEVICE = range(1, 9)
FP64, FP32 = 0, 1
HOOI, HOQRI, ALTHOOI = 0, 1, 2
INIT = {"rnd": 0, "hoevd": 1, "hosvd": 2, "user": 3}
PREC_FP64, PREC_MIXED = 0, 1

_P = ctypes.c_void_p
_U32, _U64, _I, _D = ctypes.c_uint32, ctypes.c_uint64, ctypes.c_int, ctypes.c_double


class SympropError(RuntimeError):
    def __init__(self, status: int, msg: str):
        super().__init__(f"[{status}] {msg}")
        self.status = status


class Config(ctypes.Structure):  # symprop_config
    _fields_ = [("rank", _U32), ("max_iter", _U64), ("rel_tol", _D), ("delta", _D),
                ("seed", _U64), ("init", _I), ("precision", _I), ("verbose", _I)]


class _Result(ctypes.Structure):  # symprop_result
    _fields_ = [("core", _P), ("factor", _P), ("error_trace", _P), ("relres_trace", _P),
                ("trace_cap", _U64), ("init_factor", _P), ("iterations", _U64), ("error", _D),
                ("core_norm", _D), ("time_ms", _D), ("s3ttmc_ms", _D), ("dense_ms", _D)]


_lib = None


def build(force: bool = False) -> None:
    """Compile libsymprop_b200.so, the symtucker CLI and the symtens_ttmc / s3ttmctc drivers (make; sm_100a)."""
    cmd = ["make", "-C", HERE, "-j8"]
    if force:
        subprocess.run(["make", "-C", HERE, "clean"], check=True)
    subprocess.run(cmd, check=True)


def lib():
    """The loaded C-ABI library; raises if it has not been built."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise ImportError(f"{LIB_PATH} is missing: run symprop_b200.build() (make -C symprop_b200)")
    L = ctypes.CDLL(LIB_PATH)
    sig = {
        "symprop_status_string": (ctypes.c_char_p, [_I]),
        "symprop_last_error": (ctypes.c_char_p, []),
        "symprop_device_count": (_I, [ctypes.POINTER(_I)]),
        "symprop_set_device": (_I, [_I]),
        "symprop_trim_memory": (_I, []),
        "symprop_tensor_create": (_I, [_U32, _U32, _P, _P, _U64, ctypes.POINTER(_P)]),
        "symprop_tensor_destroy": (_I, [_P]),
        "symprop_tensor_order": (_I, [_P, ctypes.POINTER(_U32)]),
        "symprop_tensor_dim": (_I, [_P, ctypes.POINTER(_U32)]),
        "symprop_tensor_nnz": (_I, [_P, ctypes.POINTER(_U64)]),
        "symprop_tensor_norm": (_I, [_P, ctypes.POINTER(_D)]),
        "symprop_tensor_owner_count": (_I, [_P, ctypes.POINTER(_U64)]),
        "symprop_tree_build": (_I, [_P]),
        "symprop_tree_level_size": (_I, [_P, _U32, ctypes.POINTER(_U64)]),
        "symprop_tree_owner_count": (_I, [_P, ctypes.POINTER(_U64)]),
        "symprop_tree_copy_level": (_I, [_P, _U32, _P, _P, _P]),
        "symprop_tree_copy_owners": (_I, [_P, _P, _P]),
        "symprop_s3ttmc": (_I, [_P, _P, _U32, _I, _P, _I]),
        "symprop_s3ttmc_device": (_I, [_P, _P, _U32, _I, _P, _I, _P]),
        "symprop_s3ttmc_launches": (_I, [_P, _U32, _I, ctypes.POINTER(_U32)]),
        "symprop_symtens_size": (_U64, [_U32, _U32]),
        "symprop_symtens_coeff": (_I, [_U32, _U32, _P]),
        "symprop_unpack_rows_device": (_I, [_P, _U64, _U32, _U32, _P, _P]),
        "symprop_tucker": (_I, [_P, ctypes.POINTER(Config), _I, ctypes.POINTER(_Result)]),
        "symprop_write_decomp": (_I, [ctypes.c_char_p, _P, _P, _U32, _U32, _U32, _I]),
        "symprop_gram_device": (_I, [_P, _U64, _U32, _P, _P, _I, _P]),
        "symprop_s3ttmc_schedule": (_I, [_I]),
        "symprop_gram_device_noalloc": (_I, [_P, _U64, _U32, _P, _P, _P]),
        "symprop_symsyrk_device": (_I, [_P, _P, _P, _U64, _U64, _P]),
        "symprop_symgemm_device": (_I, [_P, _P, _P, _P, _U64, _U64, _U64, _P]),
        "symprop_debug_set_tc_wait_ns": (_I, [_U64]),
        "symprop_tensor_load_tns": (_I, [ctypes.c_char_p, ctypes.POINTER(_P)]),
        "symprop_tensor_copy_nonzeros": (_I, [_P, _P, _P]),
        "symprop_tensor_load_spt": (_I, [ctypes.c_char_p, ctypes.POINTER(_P)]),
        "symprop_tensor_save_spt": (_I, [_P, ctypes.c_char_p]),
        "symprop_gemmtn": (_I, [_P, _P, _P, _U64, _U64, _U64]),
        "symprop_symgemm": (_I, [_P, _P, _P, _P, _U64, _U64, _U64]),
        "symprop_symsyrk": (_I, [_P, _P, _P, _U64, _U64]),
        "symprop_qr": (_I, [_P, _U64, _U64]),
        "symprop_syevd": (_I, [_P, _P, _U64, _U64]),
        "symprop_leftsvd": (_I, [_P, _P, _U64, _U64, _U64]),
    }
    for name, (res, args) in sig.items():
        f = getattr(L, name)
        f.restype = res
        f.argtypes = args
    _lib = L
    return L


def exported_symbols() -> list[str]:
    return [
        "symprop_status_string", "symprop_last_error", "symprop_device_count", "symprop_set_device",
        "symprop_trim_memory",
        "symprop_tensor_create", "symprop_tensor_destroy", "symprop_tensor_order", "symprop_tensor_dim",
        "symprop_tensor_nnz", "symprop_tensor_norm", "symprop_tensor_owner_count", "symprop_tree_build",
        "symprop_tree_level_size", "symprop_tree_owner_count", "symprop_tree_copy_level",
        "symprop_tree_copy_owners", "symprop_s3ttmc", "symprop_s3ttmc_device", "symprop_s3ttmc_launches",
        "symprop_symtens_size", "symprop_symtens_coeff", "symprop_unpack_rows_device", "symprop_tucker",
        "symprop_write_decomp", "symprop_gram_device", "symprop_s3ttmc_schedule",
        "symprop_tensor_load_tns", "symprop_tensor_copy_nonzeros", "symprop_tensor_load_spt",
        "symprop_tensor_save_spt",
        "symprop_gemmtn", "symprop_symgemm", "symprop_symsyrk", "symprop_qr", "symprop_syevd", "symprop_leftsvd",
        "symprop_symsyrk_device", "symprop_symgemm_device", "symprop_debug_set_tc_wait_ns",
    ]


def _check(st: int) -> None:
    if st != SYMPROP_OK:
        L = lib()
        raise SympropError(st, f"{L.symprop_status_string(st).decode()}: {L.symprop_last_error().decode()}")


def _ptr(a: np.ndarray):
    return ctypes.c_void_p(a.ctypes.data)


def device_count() -> int:
    n = _I(0)
    _check(lib().symprop_device_count(ctypes.byref(n)))
    return n.value


def trim_memory() -> None:
    """Return the unused memory of the library's device pool (the dense
    steps' scratch, kept between calls) to the current device."""
    _check(lib().symprop_trim_memory())


def gram_device(dY_ptr: int, n: int, m: int, dscale_ptr: int, dG_ptr: int, precision: int = FP64,
                stream: int = 0) -> None:
    """G = (Y diag(scale))^T (Y diag(scale)) on the device (FP64 CUDA cores or
    FP32 input on tcgen05 tensor cores with split-BF16 operands)."""
    _check(lib().symprop_gram_device(_P(dY_ptr), n, m, _P(dscale_ptr), _P(dG_ptr), precision, _P(stream)))


def symsyrk_device(dA_ptr: int, dscale_ptr: int, dC_ptr: int, ncoeff: int, I1: int, stream: int = 0) -> None:
    """C (I1 x I1, FP64) = (A diag(scale)) (A diag(scale))^T for an FP32 device
    A (I1 x ncoeff) and FP32 scale, on the tensor cores (split-BF16)."""
    _check(lib().symprop_symsyrk_device(_P(dA_ptr), _P(dscale_ptr), _P(dC_ptr), ncoeff, I1, _P(stream)))


def symgemm_device(dA_ptr: int, dB_ptr: int, dscale_ptr: int, dC_ptr: int, ncoeff: int, I1: int, I2: int,
                   stream: int = 0) -> None:
    """C (I1 x I2, FP64) = (A diag(scale)) (B diag(scale))^T for an FP32 device
    A (I1 x ncoeff), FP64 B (I2 x ncoeff) and FP64 scale, on the tensor cores."""
    _check(lib().symprop_symgemm_device(_P(dA_ptr), _P(dB_ptr), _P(dscale_ptr), _P(dC_ptr), ncoeff, I1, I2,
                                        _P(stream)))


class matrix:
    """The reference's symprop::matrix operations (src/dense/matrixops.cpp:18-146)
    on FP64 row-major arrays, computed on the GPU.  Functions return new arrays
    instead of writing into the caller's; symsyrk fills the upper triangle of
    the C it is given (the rest is kept) as cblas_dsyrk does."""

    @staticmethod
    def _f64(a, shape):
        return np.ascontiguousarray(a, dtype=np.float64).reshape(shape)

    @staticmethod
    def gemmtn(A, B, arow: int, acol: int, bcol: int) -> np.ndarray:
        A, B = matrix._f64(A, (arow, acol)), matrix._f64(B, (arow, bcol))
        C = np.zeros((acol, bcol))
        _check(lib().symprop_gemmtn(_ptr(C), _ptr(A), _ptr(B), arow, acol, bcol))
        return C

    @staticmethod
    def symgemm(A, B, row_coeff, I1: int, I2: int) -> np.ndarray:
        c = np.ascontiguousarray(row_coeff, dtype=np.float64).reshape(-1)
        A, B = matrix._f64(A, (I1, c.size)), matrix._f64(B, (I2, c.size))
        C = np.zeros((I1, I2))
        _check(lib().symprop_symgemm(_ptr(C), _ptr(A), _ptr(B), _ptr(c), c.size, I1, I2))
        return C

    @staticmethod
    def symsyrk(C, A, row_coeff, I1: int) -> np.ndarray:
        c = np.ascontiguousarray(row_coeff, dtype=np.float64).reshape(-1)
        A = matrix._f64(A, (I1, c.size))
        C = matrix._f64(C, (I1, I1)).copy()
        _check(lib().symprop_symsyrk(_ptr(C), _ptr(A), _ptr(c), c.size, I1))
        return C

    @staticmethod
    def qr(A, nr: int, nc: int) -> np.ndarray:
        A = matrix._f64(A, (nr, nc)).copy()
        _check(lib().symprop_qr(_ptr(A), nr, nc))
        return A

    @staticmethod
    def syevd(A, dim: int, rank: int) -> np.ndarray:
        A = matrix._f64(A, (dim, dim))
        U = np.zeros((dim, rank))
        _check(lib().symprop_syevd(_ptr(A), _ptr(U), dim, rank))
        return U

    @staticmethod
    def leftsvd(A, nr: int, nc: int, rank: int) -> np.ndarray:
        A = matrix._f64(A, (nr, nc))
        U = np.zeros((nr, rank))
        _check(lib().symprop_leftsvd(_ptr(A), _ptr(U), nr, nc, rank))
        return U


def symtens_size(dim: int, order: int) -> int:
    return int(lib().symprop_symtens_size(dim, order))


def symtens_coeff(dim: int, order: int) -> np.ndarray:
    c = np.zeros(symtens_size(dim, order))
    _check(lib().symprop_symtens_coeff(dim, order, _ptr(c)))
    return c


@dataclass
class SymTuckerDecomp:
    """Result of a Tucker solve (include/detail/tucker.hpp:25-45)."""
    core: np.ndarray
    factor: np.ndarray
    iterations: int
    error: float
    core_norm: float
    error_trace: np.ndarray
    relres_trace: np.ndarray
    time_ms: float
    s3ttmc_ms: float
    dense_ms: float
    rank: int = 0
    dim: int = 0
    order: int = 0

    def print(self, path: str, append: bool = False) -> None:
        """SymTuckerDecomp::print (src/tucker.cpp:47-61) to a file/stdout/stderr."""
        _check(lib().symprop_write_decomp(path.encode(), _ptr(self.core), _ptr(self.factor),
                                          self.dim, self.rank, self.order, int(append)))


class SpSymtensor:
    """Device-resident sparse symmetric tensor (SpSymtensor,
    include/detail/sparse/spsymtensor.hpp:24-65).  inds: nnz x order 1-based
    ids sorted within each row; vals: nnz values."""

    def __init__(self, dim: int, order: int, inds, vals):
        inds = np.ascontiguousarray(inds, dtype=np.uint32).reshape(-1, order)
        vals = np.ascontiguousarray(vals, dtype=np.float64).reshape(-1)
        if inds.shape[0] != vals.shape[0]:
            raise ValueError("inds and vals disagree on nnz")
        self._dim, self._order, self._nnz = int(dim), int(order), int(vals.shape[0])
        h = _P()
        _check(lib().symprop_tensor_create(order, dim, _ptr(inds), _ptr(vals), self._nnz, ctypes.byref(h)))
        self._h = h
        n = _D(0)
        _check(lib().symprop_tensor_norm(self._h, ctypes.byref(n)))
        self._norm = n.value

    @classmethod
    def load_tns(cls, path: str) -> "SpSymtensor":
        """SymtensLoader + SpSymtensor with the .tns text parsed on the device
        (symprop_tensor_load_tns)."""
        return cls._from_file(lib().symprop_tensor_load_tns, path)

    @classmethod
    def load_spt(cls, path: str) -> "SpSymtensor":
        """A binary SPT1 tuple file (symprop_tensor_load_spt; layout in
        include/symprop.h and synth.write_spt)."""
        return cls._from_file(lib().symprop_tensor_load_spt, path)

    def save_spt(self, path: str) -> None:
        _check(lib().symprop_tensor_save_spt(self._h, os.fsencode(path)))

    @classmethod
    def _from_file(cls, loader, path: str) -> "SpSymtensor":
        self = cls.__new__(cls)
        h = _P()
        _check(loader(os.fsencode(path), ctypes.byref(h)))
        self._h = h
        o, d, z, n = _U32(0), _U32(0), _U64(0), _D(0)
        _check(lib().symprop_tensor_order(h, ctypes.byref(o)))
        _check(lib().symprop_tensor_dim(h, ctypes.byref(d)))
        _check(lib().symprop_tensor_nnz(h, ctypes.byref(z)))
        _check(lib().symprop_tensor_norm(h, ctypes.byref(n)))
        self._order, self._dim, self._nnz, self._norm = o.value, d.value, z.value, n.value
        return self

    def nonzeros(self):
        """(inds nnz x order uint32, vals nnz float64) as held on the device
        (SpSymtensor::unnz_inds / unnzs)."""
        inds = np.empty((self._nnz, self._order), dtype=np.uint32)
        vals = np.empty(self._nnz, dtype=np.float64)
        _check(lib().symprop_tensor_copy_nonzeros(self._h, _ptr(inds), _ptr(vals)))
        return inds, vals

    def close(self):
        if getattr(self, "_h", None):
            lib().symprop_tensor_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def order(self) -> int: return self._order
    def dim(self) -> int: return self._dim
    def size(self) -> int: return self._nnz
    def norm(self) -> float: return self._norm

    @property
    def handle(self):
        return self._h

    def owner_count(self) -> int:
        v = _U64(0)
        _check(lib().symprop_tensor_owner_count(self._h, ctypes.byref(v)))
        return v.value

    def ncols(self, R: int, packed: bool) -> int:
        return symtens_size(R, self._order - 1) if packed else R ** (self._order - 1)

    # ---- S3TTMc (src/sparse/spsymtensor.cpp:30-110)
    def S3TTMc(self, U: np.ndarray, R: int, partial_sym_res: bool = False,
               precision: int = FP64) -> np.ndarray:
        dt = np.float64 if precision == FP64 else np.float32
        U = np.ascontiguousarray(U, dtype=dt).reshape(self._dim, R)
        Y = np.empty((self._dim, self.ncols(R, partial_sym_res)), dtype=dt)
        _check(lib().symprop_s3ttmc(self._h, _ptr(U), R, int(partial_sym_res), _ptr(Y), precision))
        return Y

    def s3ttmc_device(self, dU_ptr: int, R: int, dY_ptr: int, packed: bool = True,
                      precision: int = FP64, stream: int = 0) -> None:
        _check(lib().symprop_s3ttmc_device(self._h, _P(dU_ptr), R, int(packed), _P(dY_ptr),
                                           precision, _P(stream)))

    def s3ttmc_launches(self, R: int, packed: bool = True) -> int:
        v = _U32(0)
        _check(lib().symprop_s3ttmc_launches(self._h, R, int(packed), ctypes.byref(v)))
        return v.value

    # ---- CompressedDTree export (src/compressed_dtree.cpp:13-131)
    def tree_level_sizes(self) -> list:
        L = lib()
        _check(L.symprop_tree_build(self._h))
        out = []
        for l in range(self._order - 1):
            sz = _U64(0)
            _check(L.symprop_tree_level_size(self._h, l, ctypes.byref(sz)))
            out.append(sz.value)
        return out

    def tree(self) -> dict:
        L = lib()
        _check(L.symprop_tree_build(self._h))
        depth = self._order - 1
        out = {"level_idx": [], "level_ptr": [], "dep_list": []}
        for l in range(depth):
            sz = _U64(0)
            _check(L.symprop_tree_level_size(self._h, l, ctypes.byref(sz)))
            n = sz.value
            idx = np.zeros(n, np.uint32)
            ptr = np.zeros(n + 1, np.uint64)
            dep = np.zeros(max(n * (l + 1), 1), np.uint64)
            _check(L.symprop_tree_copy_level(self._h, l, _ptr(idx), _ptr(ptr), _ptr(dep)))
            out["level_idx"].append(idx)
            out["level_ptr"].append(ptr)
            out["dep_list"].append(dep[: n * (l + 1)] if l >= 1 else np.zeros(0, np.uint64))
        no = _U64(0)
        _check(L.symprop_tree_owner_count(self._h, ctypes.byref(no)))
        rem = np.zeros(no.value, np.uint64)
        val = np.zeros(no.value)
        _check(L.symprop_tree_copy_owners(self._h, _ptr(rem), _ptr(val)))
        out["rem"], out["val"] = rem, val
        return out

    # ---- Tucker (src/sparse/spsymtensor.cpp:201-337)
    def _tucker(self, alg: int, rank: int, max_iter: int = 10, rel_tol: float = 1e-6,
                delta: float = 0.5, seed: int = 0, init: str = "rnd", precision: int = PREC_FP64,
                verbose: bool = False, init_factor: np.ndarray | None = None) -> SymTuckerDecomp:
        cfg = Config(rank, max_iter, rel_tol, delta, seed, INIT[init], precision, int(verbose))
        core = np.zeros(rank ** self._order)
        factor = np.zeros((self._dim, rank))
        et = np.zeros(max(max_iter, 1))
        rt = np.zeros(max(max_iter, 1))
        r = _Result()
        r.core, r.factor = _ptr(core), _ptr(factor)
        r.error_trace, r.relres_trace = _ptr(et), _ptr(rt)
        r.trace_cap = max_iter
        keep = None
        if init == "user":
            keep = np.ascontiguousarray(init_factor, dtype=np.float64).reshape(self._dim, rank)
            r.init_factor = _ptr(keep)
        _check(lib().symprop_tucker(self._h, ctypes.byref(cfg), alg, ctypes.byref(r)))
        it = int(r.iterations)
        return SymTuckerDecomp(core, factor, it, r.error, r.core_norm, et[:it].copy(), rt[:it].copy(),
                               r.time_ms, r.s3ttmc_ms, r.dense_ms, rank, self._dim, self._order)

    def TuckerHOOI(self, **kw) -> SymTuckerDecomp: return self._tucker(HOOI, **kw)
    def TuckerHOQRI(self, **kw) -> SymTuckerDecomp: return self._tucker(HOQRI, **kw)
    def TuckerAltHOOI(self, **kw) -> SymTuckerDecomp: return self._tucker(ALTHOOI, **kw)
