/*
 * symprop.h — C ABI of the B200-native SymProp S3TTMc / Tucker path.
 *
 * Every entry point takes plain pointers and sizes and returns an int status
 * (SYMPROP_OK == 0).  Host-pointer entry points copy inputs to the GPU and
 * results back; *_device entry points take device pointers and a CUDA
 * stream (cudaStream_t passed as void*, NULL = legacy default stream).
 *
 * The reference interface each entry point replaces is cited as
 * <file>:<line> of the reference SymProp sources.
 *
 * Conventions carried over from the reference:
 *   - index tuples are 1-based, sorted ascending inside each tuple
 *     (src/utils/loader.cpp:29-31); ids must lie in [1, dim];
 *   - U is row-major dim x R; Y is row-major dim x ldy, fully overwritten;
 *   - packed Y has ldy = C(R+N-2, N-1) columns in lexicographic order of
 *     sorted column indices (include/detail/dense/symtensor.hpp:58-62,
 *     129-142); unpacked Y has ldy = R^(N-1) (src/sparse/spsymtensor.cpp:34-35).
 */
#ifndef SYMPROP_B200_H
#define SYMPROP_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ------------------------------------------------------------- status */
enum {
  SYMPROP_OK = 0,
  SYMPROP_ERR_INVALID = 1,   /* bad argument (null, out-of-range id, unsorted tuple, R = 0) */
  SYMPROP_ERR_ORDER = 2,     /* unsupported order (the reference dispatcher throws
                                std::out_of_range, include/utils/dispatcher.hpp:48-54) */
  SYMPROP_ERR_OOM = 3,       /* device or pinned-host allocation failed */
  SYMPROP_ERR_CUDA = 4,      /* a CUDA runtime call failed */
  SYMPROP_ERR_NOCONV = 5,    /* an iterative FP64 solve did not converge
                                (reference prints "... failed to converge",
                                src/dense/matrixops.cpp:31-33,69-72,86-89) */
  SYMPROP_ERR_TIMEOUT = 6,   /* a bounded device wait expired */
  SYMPROP_ERR_SIZE = 7,      /* sizes beyond what this build supports */
  SYMPROP_ERR_NODEVICE = 8   /* no CUDA device / the CUDA path is unavailable */
};

enum {
  SYMPROP_FP64 = 0,          /* U, Y in double: the drop-in precision */
  SYMPROP_FP32 = 1           /* U, Y in float, compensated FP32 accumulation */
};

enum { SYMPROP_HOOI = 0, SYMPROP_HOQRI = 1, SYMPROP_ALTHOOI = 2 };
enum { SYMPROP_INIT_RND = 0, SYMPROP_INIT_HOEVD = 1, SYMPROP_INIT_HOSVD = 2,
       SYMPROP_INIT_USER = 3 };
enum { SYMPROP_PREC_FP64 = 0,   /* plain FP64 drop-in path */
       SYMPROP_PREC_MIXED = 1   /* FP32 S3TTMc + 3xBF16 tcgen05 Gram + FP64 solves */ };

/* Human-readable text for a status code and the last error of this thread. */
const char *symprop_status_string(int status);
const char *symprop_last_error(void);

/* ------------------------------------------------------------- tensor */
typedef struct symprop_tensor symprop_tensor;

/* Builds the device-resident tensor: uploads the tuples, computes ||X|| and
 * the row-segmented owner list used by S3TTMc (a device radix sort of the
 * N owners of every nonzero by their remaining index).
 * Replaces SpSymtensor::SpSymtensor (include/detail/sparse/spsymtensor.hpp:26-27,
 * src/sparse/spsymtensor.cpp:16-28).  inds: nnz*order uint32, vals: nnz. */
int symprop_tensor_create(uint32_t order, uint32_t dim, const uint32_t *inds,
                          const double *vals, uint64_t nnz,
                          symprop_tensor **out);
int symprop_tensor_destroy(symprop_tensor *t);

/* Reads a .tns file and builds the tensor, parsing the text on the device.
 * Replaces SymtensLoader::SymtensLoader (src/utils/loader.cpp:8-36) followed
 * by SpSymtensor::SpSymtensor.  Same records as the loader: tuples sorted
 * ascending; reading stops where the loader's stream stops (a trailing
 * partial record, and a last value that ends the file with no whitespace
 * after it, are dropped).  A malformed token (one the loader's stream would
 * stop on or read only in part) gives SYMPROP_ERR_INVALID with its byte
 * offset instead of a silently shortened tensor.  Orders 2..8. */
int symprop_tensor_load_tns(const char *path, symprop_tensor **out);

/* Binary tuple files (SPT1; this library's companion to .tns, which the
 * reference reads as text only).  Layout, little endian: "SPT1", u32 order,
 * u32 dim, u32 0, u64 nnz, then nnz*order u32 ids (1-based, each tuple
 * ascending) and nnz f64 values.  load_spt builds the same tensor as
 * SpSymtensor(dim, order, ids, values) with no text to parse; a file whose
 * size disagrees with its header, or an id outside [1, dim] or an unsorted
 * tuple, is SYMPROP_ERR_INVALID; orders 2..8 (SYMPROP_ERR_ORDER otherwise).
 * save_spt writes a tensor's tuples and values in that layout. */
int symprop_tensor_load_spt(const char *path, symprop_tensor **out);
int symprop_tensor_save_spt(const symprop_tensor *t, const char *path);

/* Copies the tensor's sorted tuples (nnz*order uint32, 1-based) and values
 * (nnz) to host arrays; either pointer may be NULL.
 * SpSymtensor::unnz_inds / unnzs (include/detail/sparse/spsymtensor.hpp:35-37). */
int symprop_tensor_copy_nonzeros(const symprop_tensor *t, uint32_t *inds, double *vals);

/* order/dim/size/norm accessors: include/detail/sparse/spsymtensor.hpp:29-34,43 */
int symprop_tensor_order(const symprop_tensor *t, uint32_t *order);
int symprop_tensor_dim(const symprop_tensor *t, uint32_t *dim);
int symprop_tensor_nnz(const symprop_tensor *t, uint64_t *nnz);
int symprop_tensor_norm(const symprop_tensor *t, double *norm);   /* SpSymtensor::norm, spsymtensor.cpp:112 */
/* number of (row, leaf) owner records after merging repeated indices */
int symprop_tensor_owner_count(const symprop_tensor *t, uint64_t *owners);

/* ------------------------------------------------ CompressedDTree export */
/* Builds, on the device (radix sort + unique + segmentation), the
 * reference's CompressedDTree arrays for this tensor and keeps them until
 * the tensor is destroyed.  Replaces DTree::banerjee_insert
 * (src/dtree.cpp:56-80) + CompressedDTree::CompressedDTree
 * (src/compressed_dtree.cpp:13-90) + init_dep_list (:92-131).
 * depth = order - 1 levels; level l holds the sorted (l+1)-sub-multisets. */
int symprop_tree_build(symprop_tensor *t);
int symprop_tree_level_size(const symprop_tensor *t, uint32_t level, uint64_t *size);
int symprop_tree_owner_count(const symprop_tensor *t, uint64_t *owners);
/* Copies level_idx[level] (size), level_ptr[level] (size+1; for the last
 * level the owner CSR) and dep_list[level] (size*(level+1); level >= 1) into
 * host buffers.  Any pointer may be NULL. (compressed_dtree.hpp:52-57) */
int symprop_tree_copy_level(const symprop_tensor *t, uint32_t level,
                            uint32_t *level_idx, uint64_t *level_ptr,
                            uint64_t *dep_list);
/* Copies the owner list `nonzero` (compressed_dtree.hpp:59): remaining
 * index (1-based) and value, in the reference's order. */
int symprop_tree_copy_owners(const symprop_tensor *t, uint64_t *rem, double *val);

/* ------------------------------------------------------------- S3TTMc */
/* Y = X_(1) (U (x) ... (x) U), packed or unpacked, host buffers.
 * Replaces SpSymtensor::S3TTMc (include/detail/sparse/spsymtensor.hpp:38-39,
 * src/sparse/spsymtensor.cpp:30-110).  precision SYMPROP_FP64: U, Y are
 * double*; SYMPROP_FP32: float*. */
int symprop_s3ttmc(const symprop_tensor *t, const void *U, uint32_t R,
                   int packed, void *Y, int precision);
/* Same with device pointers on `stream`; Y is written asynchronously. */
int symprop_s3ttmc_device(const symprop_tensor *t, const void *dU, uint32_t R,
                          int packed, void *dY, int precision, void *stream);
/* Selects the S3TTMc schedule for the whole process: 0 automatic (default:
 * the pivot chain where it applies, else warp-per-owner where the packed
 * output fits one warp's registers, else CTA register-tiled, else the
 * per-owner rows kernel), 1 rows kernel, 2 CTA register-tiled only,
 * 3 warp-per-owner only, 4 pivot chain only (2, 3 and 4 return
 * SYMPROP_ERR_SIZE on shapes they do not cover).  All compute the same Y
 * up to rounding; tests use this to check each schedule against the oracle. */
int symprop_s3ttmc_schedule(int schedule);
/* Number of kernel launches one symprop_s3ttmc_device call issues for
 * (R, packed); lets callers count their launches. */
int symprop_s3ttmc_launches(const symprop_tensor *t, uint32_t R, int packed,
                            uint32_t *launches);

/* ------------------------------------------------------ packed helpers */
/* symtens_size (include/detail/dense/symtensor_base.hpp:28-30) */
uint64_t symprop_symtens_size(uint32_t dim, uint32_t order);
/* symtens_coeff (src/dense/symtensor.cpp:53-59): coeff[symtens_size] */
int symprop_symtens_coeff(uint32_t dim, uint32_t order, double *coeff);
/* unpack_symtens (src/dense/symtensor.cpp:40-45) on the device for
 * `rows` rows: packed rows x C(dim+order-1,order) -> rows x dim^order. */
int symprop_unpack_rows_device(const double *dpacked, uint64_t rows,
                               uint32_t dim, uint32_t order, double *dfull,
                               void *stream);

/* ---------------------------------------------------------- dense step */
/* Packed Gram matrix G = (Y diag(scale))^T (Y diag(scale)) (m x m, FP64,
 * full symmetric) of a device n x m row-major Y, the dense step HOOI uses
 * in place of leftsvd(Y) (src/sparse/spsymtensor.cpp:225,
 * src/dense/matrixops.cpp:18-43; symsyrk :126-146 is its n x n twin).
 * precision SYMPROP_FP64: dY, dscale are double*, FP64 CUDA-core GEMM;
 * SYMPROP_FP32: dY, dscale are float*, tcgen05 tensor cores with split-BF16
 * operands and FP32 accumulation. */
int symprop_gram_device(const void *dY, uint64_t n, uint32_t m, const void *dscale,
                        double *dG, int precision, void *stream);

/* The tensor-core (FP32-input) form of symprop_gram_device for callers that
 * cannot allocate device memory at call time: services that reserve all
 * device memory for their own pool allocator at start-up (a later cudaMalloc
 * fails or fragments the pool), and code that must not take the implicit
 * device synchronisation of cudaMalloc/cudaFree.  It allocates nothing: its
 * workspace is one fixed 32 MiB device array inside this library, held by
 * every GPU that loads the library until the process exits.  Inputs whose
 * workspace (about 4*m*n + 4*m*m bytes) exceeds it are rejected with
 * SYMPROP_ERR_SIZE.  The first call on each device looks the array up with
 * that device current and keeps its address; make that first call before
 * any stream capture, and do not use this entry point across a device reset.
 * Every call reads its error flag back and synchronises `stream` before it
 * returns.  Every call reuses the same array, so calls that overlap on the
 * GPU (other streams, other host threads) race and must be serialised by
 * the caller.  The result equals symprop_gram_device's (FP32) bit for bit.
 * This entry point has no counterpart in the reference. */
int symprop_gram_device_noalloc(const float *dY, uint64_t n, uint32_t m, const float *dscale,
                                double *dG, void *stream);

/* Device forms of matrix::symsyrk and matrix::symgemm (src/dense/
 * matrixops.cpp:126-146, :102-124) on the tcgen05 tensor cores, the dense
 * products of mixed-precision HOOI and HOQRI.  A is an FP32 row-major
 * I1 x ncoeff device matrix and scale a device vector of ncoeff column
 * scales (the square roots of the reference's row_coeff); A diag(scale) is
 * split into BF16 hi/lo parts and every product keeps three of the four
 * hi/lo terms, with FP32 accumulation.  Both synchronise `stream`.
 * symsyrk_device: C (I1 x I1, FP64, full symmetric) = (A diag(scale))
 *   (A diag(scale))^T; dscale is float*.
 * symgemm_device: C (I1 x I2, FP64, row-major) = (A diag(scale))
 *   (B diag(scale))^T for an FP64 I2 x ncoeff B; dscale is double*. */
int symprop_symsyrk_device(const float *dA, const float *dscale, double *dC, uint64_t ncoeff,
                           uint64_t I1, void *stream);
int symprop_symgemm_device(const float *dA, const double *dB, const double *dscale, double *dC,
                           uint64_t ncoeff, uint64_t I1, uint64_t I2, void *stream);

/* Failure injection for tests: bounds the tensor-core kernels' main-loop
 * waits (TMA copies, MMA completion) at ns nanoseconds instead of 2 s; 0
 * restores the default.  A wait that expires ends the call with
 * SYMPROP_ERR_TIMEOUT after the kernel has drained what it issued. */
int symprop_debug_set_tc_wait_ns(uint64_t ns);

/* ------------------------------------------- matrix:: operations (host) */
/* FP64 row-major matrices in host memory, computed on the current device:
 * the operations of the reference's symprop::matrix namespace
 * (include/detail/dense/matrixops.hpp:12-45, src/dense/matrixops.cpp).
 * Each copies its operands to the device and its result back. */

/* C (acol x bcol) = A^T B; A is arow x acol, B is arow x bcol
 * (matrix::gemmtn, src/dense/matrixops.cpp:45-56). */
int symprop_gemmtn(double *C, const double *A, const double *B, uint64_t arow, uint64_t acol,
                   uint64_t bcol);

/* C (I1 x I2) = A diag(row_coeff) B^T; A is I1 x ncoeff, B is I2 x ncoeff
 * (matrix::symgemm, :102-124). */
int symprop_symgemm(double *C, const double *A, const double *B, const double *row_coeff,
                    uint64_t ncoeff, uint64_t I1, uint64_t I2);

/* Upper triangle (j >= i) of C (I1 x I1) = A diag(row_coeff) A^T; A is
 * I1 x ncoeff; the strict lower triangle of C is left as it was, as
 * cblas_dsyrk(CblasUpper) leaves it (matrix::symsyrk, :126-146). */
int symprop_symsyrk(double *C, const double *A, const double *row_coeff, uint64_t ncoeff,
                    uint64_t I1);

/* A (nr x nc, nr >= nc) replaced in place by the explicit Q of its
 * Householder QR, with LAPACK's dgeqrf/dorgqr reflector convention
 * (matrix::qr, :58-75). */
int symprop_qr(double *A, uint64_t nr, uint64_t nc);

/* U (dim x rank) = eigenvectors of the rank largest eigenvalues of the
 * symmetric dim x dim matrix A, in ascending eigenvalue order as dsyevd
 * returns them (matrix::syevd, :77-100).  A is not modified (the reference
 * leaves dsyevd's eigenvectors in it).  rank <= 48 when dim > 96. */
int symprop_syevd(const double *A, double *U, uint64_t dim, uint64_t rank);

/* U (nr x rank) = the rank leading left singular vectors of A (nr x nc),
 * in descending singular-value order, from the eigenvectors of the smaller
 * Gram matrix (matrix::leftsvd, :18-43).  A is not modified (the reference
 * leaves dgesvd's left vectors in it).  rank <= min(nr, nc). */
int symprop_leftsvd(const double *A, double *U, uint64_t nr, uint64_t nc, uint64_t rank);

/* ------------------------------------------------------------- Tucker */
typedef struct {
  uint32_t rank;      /* Config::rank     (include/detail/tucker.hpp:15) */
  uint64_t max_iter;  /* Config::max_iter (tucker.hpp:16) */
  double rel_tol;     /* Config::rel_tol  (tucker.hpp:17) */
  double delta;       /* Config::delta    (tucker.hpp:18) */
  uint64_t seed;      /* Config::seed     (tucker.hpp:19) */
  int init;           /* Config::init: SYMPROP_INIT_* (tucker.hpp:20) */
  int precision;      /* SYMPROP_PREC_FP64 (drop-in) or SYMPROP_PREC_MIXED */
  int verbose;        /* print the reference's per-iteration lines to stdout */
} symprop_config;

typedef struct {
  /* caller-owned outputs (may be NULL) */
  double *core;        /* rank^order doubles: SymTuckerDecomp::_core (tucker.hpp:43) */
  double *factor;      /* dim*rank doubles:  SymTuckerDecomp::_factor (tucker.hpp:44) */
  double *error_trace; /* trace_cap doubles: error per iteration */
  double *relres_trace;/* trace_cap doubles: relative residual per iteration */
  uint64_t trace_cap;
  const double *init_factor; /* dim*rank doubles when init == SYMPROP_INIT_USER */
  /* filled in */
  uint64_t iterations;
  double error;        /* final sqrt(||X||^2-||C||^2)/||X|| (src/tucker.cpp:40-45) */
  double core_norm;    /* ||C|| */
  double time_ms;      /* device-timed duration of the whole solve */
  double s3ttmc_ms;    /* device time spent in S3TTMc */
  double dense_ms;     /* device time spent in the dense steps */
} symprop_result;

/* Runs HOOI / HOQRI / AltHOOI.  Replaces SpSymtensor::TuckerHOOI /
 * TuckerHOQRI / TuckerAltHOOI (src/sparse/spsymtensor.cpp:201-252,
 * 254-299, 301-337) including hosvd_init (:339-383) and the random
 * SymTuckerDecomp factor (src/tucker.cpp:25-36). */
int symprop_tucker(const symprop_tensor *t, const symprop_config *cfg, int alg,
                   symprop_result *res);

/* Writes the decomposition in the reference's text format
 * (SymTuckerDecomp::print, src/tucker.cpp:47-61) to `path`
 * ("stdout"/"stderr"/file; "" writes nothing). */
int symprop_write_decomp(const char *path, const double *core,
                         const double *factor, uint32_t dim, uint32_t rank,
                         uint32_t order, int append);

/* --------------------------------------------------- learned warm start */
/* No counterpart in the reference, which starts from random factors
 * (src/tucker.cpp:25-36) or hoevd/hosvd (src/sparse/spsymtensor.cpp:339-383).
 * A per-node MLP (F = R+2 inputs -> H hidden (ReLU) -> R outputs) maps node
 * features to an initial factor; weights are one flat array
 * [W1 (H x F), b1 (H), W2 (R x H), b2 (R)] of P = H*F + H + R*H + R values.
 * All pointers below are device pointers except where marked host. */

/* dX (dim x (R+2), FP32): standardised [log1p(degree), log1p(weighted
 * degree), R-column sketch Y D^1/2 Omega of one S3TTMc pass with a Gaussian
 * factor]; `seed` fixes the Gaussian draws. */
int symprop_ws_features(const symprop_tensor *t, uint32_t R, uint64_t seed, float *dX, void *stream);
/* forward: dZ1 (n x H) pre-activations, dOut (n x O); weights in BF16 */
int symprop_mlp_forward(const float *dX, uint32_t n, uint32_t F, uint32_t H, uint32_t O,
                        const void *dW_bf16, float *dZ1, float *dOut, void *stream);
/* backward: dgrad (P, FP32) = dL/dW for dL/dOut = dgOut (n x O) */
int symprop_mlp_backward(const float *dX, uint32_t n, uint32_t F, uint32_t H, uint32_t O,
                         const void *dW_bf16, const float *dZ1, const float *dgOut, float *dgrad,
                         void *stream);
/* rotation-invariant projector loss L = r - tr(P_label P_out) with
 * P_out = X (X^T X)^-1 X^T, X = dOut (n x r); dUlabel n x r orthonormal
 * (FP64); writes dL/dX to dgOut and L to *loss (host). */
int symprop_projector_loss(const float *dOut, const double *dUlabel, uint32_t n, uint32_t r,
                           float *dgOut, double *loss, void *stream);
/* Adam on the FP32 master weights; refreshes the BF16 shadow dw_bf16. */
int symprop_adam_step(float *dw, float *dm, float *dv, const float *dg, uint32_t P, float lr,
                      float beta1, float beta2, float eps, uint32_t step, void *dw_bf16,
                      void *stream);
/* Initial factor for a tensor: features -> MLP (host FP32 weights hW, H
 * hidden) -> orthonormal basis; writes dim x R doubles to host hU. */
int symprop_ws_predict(const symprop_tensor *t, uint32_t R, uint64_t seed, uint32_t H,
                       const float *hW, double *hU);

/* ------------------------------------------------------------- devices */
int symprop_device_count(int *count);
int symprop_set_device(int device);
/* The library keeps the scratch of its dense steps (eigensolver blocks,
 * GEMM and Gram partial sums) in a per-device pool between calls, so that a
 * repeated solve allocates no new scratch.  This waits for the current
 * device and returns the pool's unused memory to it (memory in use is not
 * touched); call it before handing the GPU to other work.  (No reference
 * counterpart: the reference allocates host memory per call.) */
int symprop_trim_memory(void);

#ifdef __cplusplus
}
#endif
#endif /* SYMPROP_B200_H */
