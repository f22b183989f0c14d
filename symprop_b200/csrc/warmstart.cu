// Learned warm start for HOOI / HOQRI (no counterpart in the reference,
// whose factor starts from std::normal_distribution draws,
// src/tucker.cpp:25-36, or from hoevd/hosvd, src/sparse/spsymtensor.cpp:339-383).
//
// Per node i the features are
//   x_i = [ log(1+deg_i), log(1+wdeg_i), sketch_i (R values) ]   (standardised)
// with deg the number of tuples containing i, wdeg the value-weighted
// degree, and sketch = Y D^1/2 Omega from one S3TTMc pass with a Gaussian U
// (Y n x m packed, Omega m x R Gaussian).  A 2-layer per-node MLP
//   out_i = W2 relu(W1 x_i + b1) + b2          (F -> H -> R)
// is applied to every node with the same weights (permutation-equivariant
// over nodes); U0 = orth(out).  Training minimises the rotation-invariant
// projector loss  L = R - tr(P_label P_out),  P_out = X (X^T X)^-1 X^T.
//
// Weights are kept as an FP32 master copy with a BF16 shadow used by the
// forward kernel; Adam updates the master and refreshes the shadow.
#include <cuda_bf16.h>

#include <cmath>
#include <random>
#include <vector>

#include "dense.cuh"
#include "tensor.cuh"

namespace spb {
namespace ws {
namespace {

inline unsigned cdiv(uint64_t a, uint64_t b) { return (unsigned)((a + b - 1) / b); }

__global__ void degree_kernel(const uint32_t *inds0, const double *vals, uint64_t nnz, uint32_t order,
                              double *deg, double *wdeg) {
  uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= nnz) return;
  const uint32_t *t = inds0 + i * order;
  for (uint32_t j = 0; j < order; ++j) {
    if (j == 0 || t[j] != t[j - 1]) atomicAdd(&deg[t[j]], 1.0);
    atomicAdd(&wdeg[t[j]], vals[i]);
  }
}

__global__ void gaussian_kernel(float *A, size_t n, uint64_t seed) {
  size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  auto mix = [](uint64_t z) {
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
  };
  uint64_t a = mix(seed + 0x9E3779B97F4A7C15ull * (2 * i + 1));
  uint64_t b = mix(seed + 0x9E3779B97F4A7C15ull * (2 * i + 2));
  double u1 = ((double)(a >> 11) + 0.5) * (1.0 / 9007199254740992.0);
  double u2 = (double)(b >> 11) * (1.0 / 9007199254740992.0);
  A[i] = (float)(sqrt(-2.0 * log(u1)) * cos(6.283185307179586 * u2));  // Box-Muller
}

// column standardisation of an n x F feature matrix (F <= 64), one block
__global__ void standardize_kernel(float *X, int n, int F) {
  __shared__ double s1[64], s2[64];
  if (threadIdx.x < 64) { s1[threadIdx.x] = 0; s2[threadIdx.x] = 0; }
  __syncthreads();
  for (int f = 0; f < F; ++f) {
    double a = 0, b = 0;
    for (int i = threadIdx.x; i < n; i += blockDim.x) {
      double v = X[(size_t)i * F + f];
      a += v;
      b += v * v;
    }
    for (int o = 16; o > 0; o >>= 1) {
      a += __shfl_down_sync(0xffffffffu, a, o);
      b += __shfl_down_sync(0xffffffffu, b, o);
    }
    __shared__ double wa[32], wb[32];
    if ((threadIdx.x & 31) == 0) { wa[threadIdx.x >> 5] = a; wb[threadIdx.x >> 5] = b; }
    __syncthreads();
    if (threadIdx.x == 0) {
      double ta = 0, tb = 0;
      for (int w = 0; w < (int)(blockDim.x >> 5); ++w) { ta += wa[w]; tb += wb[w]; }
      s1[f] = ta / n;
      s2[f] = sqrt(fmax(tb / n - (ta / n) * (ta / n), 0.0)) + 1e-6;
    }
    __syncthreads();
  }
  for (size_t idx = threadIdx.x; idx < (size_t)n * F; idx += blockDim.x) {
    int f = (int)(idx % F);
    X[idx] = (float)((X[idx] - s1[f]) / s2[f]);
  }
}

__global__ void assemble_kernel(const double *deg, const double *wdeg, const double *sk, int n, int R,
                                float *X) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const int F = R + 2;
  X[(size_t)i * F + 0] = (float)log1p(deg[i]);
  X[(size_t)i * F + 1] = (float)log1p(fabs(wdeg[i]));
  for (int c = 0; c < R; ++c) X[(size_t)i * F + 2 + c] = (float)sk[(size_t)i * R + c];
}

// ------------------------------------------------------------------ MLP

struct Shapes {
  int F, H, O;
  __host__ __device__ int oW1() const { return 0; }
  __host__ __device__ int ob1() const { return H * F; }
  __host__ __device__ int oW2() const { return H * F + H; }
  __host__ __device__ int ob2() const { return H * F + H + O * H; }
  __host__ __device__ int total() const { return H * F + H + O * H + O; }
};

// one thread per node; BF16 weights staged in shared memory as FP32
__global__ void mlp_forward_kernel(const float *X, int n, Shapes s, const __nv_bfloat16 *Wb,
                                   float *Z1, float *Out) {
  extern __shared__ float sw[];
  for (int p = threadIdx.x; p < s.total(); p += blockDim.x) sw[p] = __bfloat162float(Wb[p]);
  __syncthreads();
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  float x[64], h[128];
  for (int f = 0; f < s.F; ++f) x[f] = X[(size_t)i * s.F + f];
  for (int k = 0; k < s.H; ++k) {
    float z = sw[s.ob1() + k];
    for (int f = 0; f < s.F; ++f) z += sw[s.oW1() + k * s.F + f] * x[f];
    Z1[(size_t)i * s.H + k] = z;
    h[k] = z > 0.f ? z : 0.f;
  }
  for (int o = 0; o < s.O; ++o) {
    float y = sw[s.ob2() + o];
    for (int k = 0; k < s.H; ++k) y += sw[s.oW2() + o * s.H + k] * h[k];
    Out[(size_t)i * s.O + o] = y;
  }
}

// per block of 128 nodes: per-parameter gradient partial sums (deterministic)
constexpr int kBwdNodes = 128;
__global__ void mlp_backward_kernel(const float *X, int n, Shapes s, const __nv_bfloat16 *Wb,
                                    const float *Z1, const float *gOut, float *part) {
  extern __shared__ float sm[];
  float *sW = sm;                              // total
  float *sX = sW + s.total();                  // kBwdNodes x F
  float *sH = sX + kBwdNodes * s.F;            // kBwdNodes x H (relu(z1))
  float *sD = sH + kBwdNodes * s.H;            // kBwdNodes x H (dz1)
  float *sG = sD + kBwdNodes * s.H;            // kBwdNodes x O (gOut)
  for (int p = threadIdx.x; p < s.total(); p += blockDim.x) sW[p] = __bfloat162float(Wb[p]);
  const int base = blockIdx.x * kBwdNodes;
  __syncthreads();
  for (int a = threadIdx.x; a < kBwdNodes; a += blockDim.x) {
    int i = base + a;
    bool ok = i < n;
    for (int f = 0; f < s.F; ++f) sX[a * s.F + f] = ok ? X[(size_t)i * s.F + f] : 0.f;
    for (int o = 0; o < s.O; ++o) sG[a * s.O + o] = ok ? gOut[(size_t)i * s.O + o] : 0.f;
    for (int k = 0; k < s.H; ++k) {
      float z = ok ? Z1[(size_t)i * s.H + k] : 0.f;
      sH[a * s.H + k] = z > 0.f ? z : 0.f;
      float dh = 0.f;
      for (int o = 0; o < s.O; ++o) dh += sW[s.oW2() + o * s.H + k] * sG[a * s.O + o];
      sD[a * s.H + k] = z > 0.f ? dh : 0.f;
    }
  }
  __syncthreads();
  float *out = part + (size_t)blockIdx.x * s.total();
  for (int p = threadIdx.x; p < s.total(); p += blockDim.x) {
    float g = 0.f;
    if (p < s.ob1()) {  // W1[k][f] += dz1[k] x[f]
      int k = p / s.F, f = p % s.F;
      for (int a = 0; a < kBwdNodes; ++a) g += sD[a * s.H + k] * sX[a * s.F + f];
    } else if (p < s.oW2()) {
      int k = p - s.ob1();
      for (int a = 0; a < kBwdNodes; ++a) g += sD[a * s.H + k];
    } else if (p < s.ob2()) {  // W2[o][k] += gOut[o] h[k]
      int q = p - s.oW2(), o = q / s.H, k = q % s.H;
      for (int a = 0; a < kBwdNodes; ++a) g += sG[a * s.O + o] * sH[a * s.H + k];
    } else {
      int o = p - s.ob2();
      for (int a = 0; a < kBwdNodes; ++a) g += sG[a * s.O + o];
    }
    out[p] = g;
  }
}

__global__ void sum_parts_kernel(const float *part, int nparts, int P, float *g) {
  int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= P) return;
  float a = 0.f;
  for (int b = 0; b < nparts; ++b) a += part[(size_t)b * P + p];
  g[p] = a;
}

__global__ void adam_kernel(float *w, float *m, float *v, const float *g, int P, float lr, float b1,
                            float b2, float eps, float c1, float c2, __nv_bfloat16 *wb) {
  int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= P) return;
  float gi = g[p];
  float mi = b1 * m[p] + (1.f - b1) * gi;
  float vi = b2 * v[p] + (1.f - b2) * gi * gi;
  m[p] = mi;
  v[p] = vi;
  float wi = w[p] - lr * (mi / c1) / (sqrtf(vi / c2) + eps);
  w[p] = wi;
  wb[p] = __float2bfloat16_rn(wi);
}

__global__ void f2d_kernel(const float *a, double *b, size_t n) {
  size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) b[i] = a[i];
}
__global__ void d2f_kernel(const double *a, float *b, size_t n) {
  size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) b[i] = (float)a[i];
}

// small r x r helpers in one thread block (r <= 32): Ginv (SPD inverse),
// M1 = A Ginv, M2 = Ginv A^T A Ginv, f = tr(Ginv A^T A)
__global__ void proj_small_kernel(const double *A, const double *G, int r, double *M1, double *M2,
                                  double *f_out) {
  __shared__ double sG[32 * 32], sI[32 * 32], sA[32 * 32], sT[32 * 32];
  const int tid = threadIdx.x;
  for (int i = tid; i < r * r; i += blockDim.x) {
    sG[i] = G[i];
    sA[i] = A[i];
    sI[i] = (i / r == i % r) ? 1.0 : 0.0;
  }
  __syncthreads();
  // Gauss-Jordan on the SPD matrix (pivots stay positive)
  for (int k = 0; k < r; ++k) {
    __syncthreads();
    double piv = sG[k * r + k];
    if (!(piv > 0)) piv = 1e-300;
    __syncthreads();
    for (int j = tid; j < r; j += blockDim.x) {
      sG[k * r + j] /= piv;
      sI[k * r + j] /= piv;
    }
    __syncthreads();
    for (int idx = tid; idx < r * r; idx += blockDim.x) {
      int i = idx / r, j = idx % r;
      if (i == k) continue;
      double fct = sG[i * r + k];
      sI[i * r + j] -= fct * sI[k * r + j];
      if (j != k) sG[i * r + j] -= fct * sG[k * r + j];
    }
    __syncthreads();
    for (int i = tid; i < r; i += blockDim.x)
      if (i != k) sG[i * r + k] = 0.0;
  }
  __syncthreads();
  // M1 = A Ginv; T = A^T A
  for (int idx = tid; idx < r * r; idx += blockDim.x) {
    int i = idx / r, j = idx % r;
    double a = 0, t = 0;
    for (int k = 0; k < r; ++k) {
      a += sA[i * r + k] * sI[k * r + j];
      t += sA[k * r + i] * sA[k * r + j];
    }
    M1[idx] = a;
    sT[idx] = t;
  }
  __syncthreads();
  // sG <- T Ginv (reuse), then M2 = Ginv (T Ginv)
  for (int idx = tid; idx < r * r; idx += blockDim.x) {
    int i = idx / r, j = idx % r;
    double a = 0;
    for (int k = 0; k < r; ++k) a += sT[i * r + k] * sI[k * r + j];
    sG[idx] = a;
  }
  __syncthreads();
  for (int idx = tid; idx < r * r; idx += blockDim.x) {
    int i = idx / r, j = idx % r;
    double a = 0;
    for (int k = 0; k < r; ++k) a += sI[i * r + k] * sG[k * r + j];
    M2[idx] = a;
  }
  if (tid == 0) {
    double f = 0;
    for (int i = 0; i < r; ++i)
      for (int k = 0; k < r; ++k) f += sI[i * r + k] * sT[k * r + i];
    f_out[0] = f;
  }
}

}  // namespace

// features (n x (R+2), FP32) of tensor t for rank R
void features(TensorState &t, uint32_t R, uint64_t seed, float *dX, cudaStream_t st) {
  const int n = (int)t.dim;
  const uint32_t L = t.order - 1;
  const int m = (int)symsize(R, L);
  const int F = (int)R + 2;
  DBuf<double> deg(n), wdeg(n);
  SPB_CUDA(cudaMemsetAsync(deg.p, 0, sizeof(double) * n, st));
  SPB_CUDA(cudaMemsetAsync(wdeg.p, 0, sizeof(double) * n, st));
  if (t.nnz) {
    degree_kernel<<<cdiv(t.nnz, 256), 256, 0, st>>>(t.inds.p, t.vals.p, t.nnz, t.order, deg.p, wdeg.p);
    SPB_LAUNCH_CHECK();
  }
  DBuf<float> Ug((size_t)n * R), Y((size_t)n * m), Om((size_t)m * R);
  gaussian_kernel<<<cdiv((size_t)n * R, 256), 256, 0, st>>>(Ug.p, (size_t)n * R, seed);
  gaussian_kernel<<<cdiv((size_t)m * R, 256), 256, 0, st>>>(Om.p, (size_t)m * R, seed ^ 0xABCDEFull);
  SPB_LAUNCH_CHECK();
  s3ttmc_run(t, Ug.p, R, true, Y.p, SYMPROP_FP32, st);
  // sketch = Y D^1/2 Omega
  std::vector<float> hsd(m);
  for_each_sorted(R, (int)L, [&](const std::vector<uint32_t> &q, uint64_t lin) {
    uint64_t denom = 1, run = 1;
    for (size_t j = 1; j <= q.size(); ++j) {
      if (j < q.size() && q[j] == q[j - 1]) ++run;
      else { denom *= factorial_u64((int)run); run = 1; }
    }
    hsd[lin] = (float)std::sqrt((double)(factorial_u64((int)L) / denom));
  });
  DBuf<float> sd(m), SK((size_t)n * R);
  SPB_CUDA(cudaMemcpyAsync(sd.p, hsd.data(), sizeof(float) * m, cudaMemcpyHostToDevice, st));
  dense::gemm<float>(st, n, (int)R, m, 1.f, Y.p, m, false, Om.p, (int)R, false, 0.f, SK.p, (int)R, sd.p);
  DBuf<double> SKd((size_t)n * R);
  f2d_kernel<<<cdiv((size_t)n * R, 256), 256, 0, st>>>(SK.p, SKd.p, (size_t)n * R);
  assemble_kernel<<<cdiv(n, 256), 256, 0, st>>>(deg.p, wdeg.p, SKd.p, n, (int)R, dX);
  standardize_kernel<<<1, 1024, 0, st>>>(dX, n, F);
  SPB_LAUNCH_CHECK();
  SPB_CUDA(cudaStreamSynchronize(st));
}

void mlp_forward(const float *dX, int n, int F, int H, int O, const void *Wb, float *dZ1, float *dOut,
                 cudaStream_t st) {
  if (F > 64 || H > 128) fail(SYMPROP_ERR_SIZE, "MLP sizes F<=64, H<=128");
  Shapes s{F, H, O};
  size_t smem = sizeof(float) * s.total();
  mlp_forward_kernel<<<cdiv(n, 128), 128, smem, st>>>(dX, n, s, (const __nv_bfloat16 *)Wb, dZ1, dOut);
  SPB_LAUNCH_CHECK();
}

void mlp_backward(const float *dX, int n, int F, int H, int O, const void *Wb, const float *dZ1,
                  const float *dgOut, float *dgrad, cudaStream_t st) {
  Shapes s{F, H, O};
  const int nb = (int)cdiv(n, kBwdNodes);
  DBuf<float> part((size_t)nb * s.total());
  size_t smem = sizeof(float) * (s.total() + kBwdNodes * (F + 2 * H + O));
  if (smem > 48 * 1024)
    SPB_CUDA(cudaFuncSetAttribute(mlp_backward_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  mlp_backward_kernel<<<nb, 128, smem, st>>>(dX, n, s, (const __nv_bfloat16 *)Wb, dZ1, dgOut, part.p);
  SPB_LAUNCH_CHECK();
  sum_parts_kernel<<<cdiv(s.total(), 256), 256, 0, st>>>(part.p, nb, s.total(), dgrad);
  SPB_LAUNCH_CHECK();
  SPB_CUDA(cudaStreamSynchronize(st));
}

// L = r - tr(P_label P_X); gX = dL/dX (n x r, FP32).  Ut: n x r orthonormal (FP64)
double projector_loss(const float *dXo, const double *dUt, int n, int r, float *dgX, cudaStream_t st) {
  if (r > 32) fail(SYMPROP_ERR_SIZE, "projector loss supports r <= 32");
  DBuf<double> X((size_t)n * r), A(r * r), G(r * r), M1(r * r), M2(r * r), f(1), gx((size_t)n * r);
  f2d_kernel<<<cdiv((size_t)n * r, 256), 256, 0, st>>>(dXo, X.p, (size_t)n * r);
  SPB_LAUNCH_CHECK();
  dense::gemm<double>(st, r, r, n, 1.0, dUt, r, true, X.p, r, false, 0.0, A.p, r);   // A = Ut^T X
  dense::gemm<double>(st, r, r, n, 1.0, X.p, r, true, X.p, r, false, 0.0, G.p, r);   // G = X^T X
  proj_small_kernel<<<1, 256, 0, st>>>(A.p, G.p, r, M1.p, M2.p, f.p);
  SPB_LAUNCH_CHECK();
  // gX = -2 (Ut M1 - X M2)
  dense::gemm<double>(st, n, r, r, -2.0, dUt, r, false, M1.p, r, false, 0.0, gx.p, r);
  dense::gemm<double>(st, n, r, r, 2.0, X.p, r, false, M2.p, r, false, 1.0, gx.p, r);
  d2f_kernel<<<cdiv((size_t)n * r, 256), 256, 0, st>>>(gx.p, dgX, (size_t)n * r);
  SPB_LAUNCH_CHECK();
  double hf = 0;
  SPB_CUDA(cudaMemcpyAsync(&hf, f.p, sizeof(double), cudaMemcpyDeviceToHost, st));
  SPB_CUDA(cudaStreamSynchronize(st));
  return (double)r - hf;
}

void adam(float *w, float *m, float *v, const float *g, int P, float lr, float b1, float b2, float eps,
          int step, void *wb, cudaStream_t st) {
  float c1 = 1.f - std::pow(b1, (float)step), c2 = 1.f - std::pow(b2, (float)step);
  adam_kernel<<<cdiv(P, 256), 256, 0, st>>>(w, m, v, g, P, lr, b1, b2, eps, c1, c2, (__nv_bfloat16 *)wb);
  SPB_LAUNCH_CHECK();
}

}  // namespace ws
}  // namespace spb

// ------------------------------------------------------------------ C ABI
using namespace spb;

namespace {
inline uint32_t nparams(uint32_t F, uint32_t H, uint32_t O) { return H * F + H + O * H + O; }
__global__ void f2bf_kernel(const float *a, __nv_bfloat16 *b, uint32_t n) {
  uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) b[i] = __float2bfloat16_rn(a[i]);
}
}  // namespace

extern "C" {

int symprop_ws_features(const symprop_tensor *t, uint32_t R, uint64_t seed, float *dX, void *stream) {
  return guard([&] {
    if (!t || !dX || R == 0 || R > 62) fail(SYMPROP_ERR_INVALID, "bad arguments");
    SPB_CUDA(cudaSetDevice(t->s.device));
    ws::features(const_cast<TensorState &>(t->s), R, seed, dX, (cudaStream_t)stream);
  });
}

int symprop_mlp_forward(const float *dX, uint32_t n, uint32_t F, uint32_t H, uint32_t O,
                        const void *dW_bf16, float *dZ1, float *dOut, void *stream) {
  return guard([&] {
    if (!dX || !dW_bf16 || !dZ1 || !dOut) fail(SYMPROP_ERR_INVALID, "null argument");
    ws::mlp_forward(dX, (int)n, (int)F, (int)H, (int)O, dW_bf16, dZ1, dOut, (cudaStream_t)stream);
  });
}

int symprop_mlp_backward(const float *dX, uint32_t n, uint32_t F, uint32_t H, uint32_t O,
                         const void *dW_bf16, const float *dZ1, const float *dgOut, float *dgrad,
                         void *stream) {
  return guard([&] {
    if (!dX || !dW_bf16 || !dZ1 || !dgOut || !dgrad) fail(SYMPROP_ERR_INVALID, "null argument");
    ws::mlp_backward(dX, (int)n, (int)F, (int)H, (int)O, dW_bf16, dZ1, dgOut, dgrad,
                     (cudaStream_t)stream);
  });
}

int symprop_projector_loss(const float *dOut, const double *dUlabel, uint32_t n, uint32_t r,
                           float *dgOut, double *loss, void *stream) {
  return guard([&] {
    if (!dOut || !dUlabel || !dgOut || !loss) fail(SYMPROP_ERR_INVALID, "null argument");
    *loss = ws::projector_loss(dOut, dUlabel, (int)n, (int)r, dgOut, (cudaStream_t)stream);
  });
}

int symprop_adam_step(float *dw, float *dm, float *dv, const float *dg, uint32_t P, float lr,
                      float beta1, float beta2, float eps, uint32_t step, void *dw_bf16,
                      void *stream) {
  return guard([&] {
    if (!dw || !dm || !dv || !dg || !dw_bf16 || step == 0) fail(SYMPROP_ERR_INVALID, "bad arguments");
    ws::adam(dw, dm, dv, dg, (int)P, lr, beta1, beta2, eps, (int)step, dw_bf16, (cudaStream_t)stream);
  });
}

int symprop_ws_predict(const symprop_tensor *t, uint32_t R, uint64_t seed, uint32_t H,
                       const float *hW, double *hU) {
  return guard([&] {
    if (!t || !hW || !hU || R == 0 || R > 62) fail(SYMPROP_ERR_INVALID, "bad arguments");
    TensorState &s = const_cast<TensorState &>(t->s);
    SPB_CUDA(cudaSetDevice(s.device));
    const uint32_t n = s.dim, F = R + 2, P = nparams(F, H, R);
    cudaStream_t st = 0;
    DBuf<float> X((size_t)n * F), Z1((size_t)n * H), Out((size_t)n * R), W(P);
    DBuf<__nv_bfloat16> Wb(P);
    DBuf<double> U((size_t)n * R);
    SPB_CUDA(cudaMemcpy(W.p, hW, sizeof(float) * P, cudaMemcpyHostToDevice));
    f2bf_kernel<<<(P + 255) / 256, 256, 0, st>>>(W.p, Wb.p, P);
    SPB_LAUNCH_CHECK();
    ws::features(s, R, seed, X.p, st);
    ws::mlp_forward(X.p, (int)n, (int)F, (int)H, (int)R, Wb.p, Z1.p, Out.p, st);
    dense::convert<float, double>(st, Out.p, U.p, (size_t)n * R);
    dense::orthonormalize(st, U.p, (int)n, (int)R);
    SPB_CUDA(cudaMemcpy(hU, U.p, sizeof(double) * n * R, cudaMemcpyDeviceToHost));
  });
}

}  // extern "C"
