// Kernels of the learned initial guess (no counterpart in the reference): a
// small MLP trained and evaluated on the GPU.  Matrix products run on the
// tensor cores in BF16 with FP32 accumulation (WMMA 16x16x16 fragments, one
// 32x32 tile per warp, 64x64 per block); bias, activation, loss and the Adam
// step are FP32.  Every dimension handed to the GEMM is a multiple of 64 (the
// caller pads), and every matrix is row-major with its row length as stride.

#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <mma.h>

#include <cmath>
#include <cstdint>
#include <string>
#include <type_traits>

#include "pfe_common.cuh"

namespace pfe {

using namespace nvcuda;

// C[M,N] (+)= op(A)[M,K] op(B)[K,N]; A is M x K (TA = false) or K x M (TA = true),
// B is K x N (TB = false) or N x K (TB = true); all BF16 row-major, C FP32.
template <bool TA, bool TB>
__global__ void __launch_bounds__(128) k_gemm_bf16(const __nv_bfloat16* __restrict__ A,
                                                   const __nv_bfloat16* __restrict__ B, float* __restrict__ C, int M,
                                                   int N, int K, int accumulate) {
  using LA = typename std::conditional<TA, wmma::col_major, wmma::row_major>::type;
  using LB = typename std::conditional<TB, wmma::col_major, wmma::row_major>::type;
  const int warp = threadIdx.x >> 5;
  const int m0 = blockIdx.y * 64 + (warp >> 1) * 32;
  const int n0 = blockIdx.x * 64 + (warp & 1) * 32;
  wmma::fragment<wmma::accumulator, 16, 16, 16, float> acc[2][2];
#pragma unroll
  for (int i = 0; i < 2; ++i)
#pragma unroll
    for (int j = 0; j < 2; ++j) {
      if (accumulate) wmma::load_matrix_sync(acc[i][j], C + (size_t)(m0 + 16 * i) * N + n0 + 16 * j, N, wmma::mem_row_major);
      else wmma::fill_fragment(acc[i][j], 0.0f);
    }
  const int lda = TA ? M : K, ldb = TB ? K : N;
  for (int k = 0; k < K; k += 16) {
    wmma::fragment<wmma::matrix_a, 16, 16, 16, __nv_bfloat16, LA> a[2];
    wmma::fragment<wmma::matrix_b, 16, 16, 16, __nv_bfloat16, LB> b[2];
#pragma unroll
    for (int i = 0; i < 2; ++i) {
      const int r = m0 + 16 * i;
      const __nv_bfloat16* pa = TA ? A + (size_t)k * lda + r : A + (size_t)r * lda + k;
      wmma::load_matrix_sync(a[i], pa, lda);
    }
#pragma unroll
    for (int j = 0; j < 2; ++j) {
      const int c = n0 + 16 * j;
      const __nv_bfloat16* pb = TB ? B + (size_t)c * ldb + k : B + (size_t)k * ldb + c;
      wmma::load_matrix_sync(b[j], pb, ldb);
    }
#pragma unroll
    for (int i = 0; i < 2; ++i)
#pragma unroll
      for (int j = 0; j < 2; ++j) wmma::mma_sync(acc[i][j], a[i], b[j], acc[i][j]);
  }
#pragma unroll
  for (int i = 0; i < 2; ++i)
#pragma unroll
    for (int j = 0; j < 2; ++j)
      wmma::store_matrix_sync(C + (size_t)(m0 + 16 * i) * N + n0 + 16 * j, acc[i][j], N, wmma::mem_row_major);
}

__device__ __forceinline__ float silu(float z) { return z / (1.0f + __expf(-z)); }
__device__ __forceinline__ float silu_grad(float z) {
  const float s = 1.0f / (1.0f + __expf(-z));
  return s * (1.0f + z * (1.0f - s));
}

// H = act(Z + b) (FP32 and a BF16 copy); Z keeps the pre-activation for backward.
__global__ void k_bias_act(float* __restrict__ Z, const float* __restrict__ bias, float* __restrict__ H,
                           __nv_bfloat16* __restrict__ Hb, int M, int N, int act) {
  const long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (t >= (long long)M * N) return;
  const float z = Z[t] + bias[t % N];
  Z[t] = z;
  const float h = act ? silu(z) : z;
  H[t] = h;
  if (Hb) Hb[t] = __float2bfloat16(h);
}

// dZ = dH * act'(Z) (FP32 and BF16 copy)
__global__ void k_act_grad(const float* __restrict__ dH, const float* __restrict__ Z, float* __restrict__ dZ,
                           __nv_bfloat16* __restrict__ dZb, long long n, int act) {
  const long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (t >= n) return;
  const float g = act ? dH[t] * silu_grad(Z[t]) : dH[t];
  dZ[t] = g;
  dZb[t] = __float2bfloat16(g);
}

// db[j] = sum_i dZ[i, j] (one thread per column; M is a few thousand at most)
__global__ void k_colsum(const float* __restrict__ dZ, float* __restrict__ db, int M, int N) {
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= N) return;
  float s = 0.0f;
  for (int i = 0; i < M; ++i) s += dZ[(size_t)i * N + j];
  db[j] = s;
}

// masked mean-square error: loss = sum w (Y - T)^2 / sum w; dY = 2 w (Y - T) / sum w
__global__ void k_mse(const float* __restrict__ Y, const float* __restrict__ T, const float* __restrict__ W,
                      float inv_wsum, float* __restrict__ dY, float* __restrict__ loss, long long n) {
  const long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  float l = 0.0f;
  if (t < n) {
    const float d = Y[t] - T[t];
    dY[t] = 2.0f * W[t] * d * inv_wsum;
    l = W[t] * d * d * inv_wsum;
  }
  for (int o = 16; o > 0; o >>= 1) l += __shfl_xor_sync(0xffffffffu, l, o);
  if ((threadIdx.x & 31) == 0 && l != 0.0f) atomicAdd(loss, l);
}

// Adam on FP32 master weights; the BF16 copy used by the GEMMs is refreshed.
__global__ void k_adam(float* __restrict__ w, __nv_bfloat16* __restrict__ wb, const float* __restrict__ g,
                       float* __restrict__ m, float* __restrict__ v, long long n, float lr, float b1, float b2, float eps,
                       float c1, float c2, float decay) {
  const long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (t >= n) return;
  const float gt = g[t] + decay * w[t];
  const float mt = b1 * m[t] + (1.0f - b1) * gt;
  const float vt = b2 * v[t] + (1.0f - b2) * gt * gt;
  m[t] = mt;
  v[t] = vt;
  const float wt = w[t] - lr * (mt / c1) / (sqrtf(vt / c2) + eps);
  w[t] = wt;
  if (wb) wb[t] = __float2bfloat16(wt);
}

__global__ void k_to_bf16(const float* __restrict__ x, __nv_bfloat16* __restrict__ y, long long n) {
  const long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (t < n) y[t] = __float2bfloat16(x[t]);
}

static int bad_dims(int M, int N, int K) {
  if (M <= 0 || N <= 0 || K <= 0 || (M % 64) || (N % 64) || (K % 64)) {
    set_error("pfe_mlp_gemm: M, N and K must be positive multiples of 64");
    return 1;
  }
  return 0;
}

static unsigned blocks_for(long long n) { return (unsigned)((n + 255) / 256); }

}  // namespace pfe

extern "C" {

int32_t pfe_mlp_gemm(const void* a, const void* b, float* c, int32_t m, int32_t n, int32_t k, int32_t trans_a,
                     int32_t trans_b, int32_t accumulate, void* stream) {
  if (!a || !b || !c) { pfe::set_error("pfe_mlp_gemm: null pointer"); return PFE_EINVAL; }
  if (pfe::bad_dims(m, n, k)) return PFE_EINVAL;
  const dim3 grid(n / 64, m / 64);
  cudaStream_t s = (cudaStream_t)stream;
  const auto* A = static_cast<const __nv_bfloat16*>(a);
  const auto* B = static_cast<const __nv_bfloat16*>(b);
  if (!trans_a && !trans_b) pfe::k_gemm_bf16<false, false><<<grid, 128, 0, s>>>(A, B, c, m, n, k, accumulate);
  else if (!trans_a && trans_b) pfe::k_gemm_bf16<false, true><<<grid, 128, 0, s>>>(A, B, c, m, n, k, accumulate);
  else if (trans_a && !trans_b) pfe::k_gemm_bf16<true, false><<<grid, 128, 0, s>>>(A, B, c, m, n, k, accumulate);
  else pfe::k_gemm_bf16<true, true><<<grid, 128, 0, s>>>(A, B, c, m, n, k, accumulate);
  PFE_CUDA(cudaGetLastError());
  return PFE_OK;
}

int32_t pfe_mlp_bias_act(float* z, const float* bias, float* h, void* h_bf16, int32_t m, int32_t n, int32_t act,
                         void* stream) {
  if (!z || !bias || !h || m <= 0 || n <= 0) { pfe::set_error("pfe_mlp_bias_act: bad argument"); return PFE_EINVAL; }
  pfe::k_bias_act<<<pfe::blocks_for((long long)m * n), 256, 0, (cudaStream_t)stream>>>(
      z, bias, h, static_cast<__nv_bfloat16*>(h_bf16), m, n, act);
  PFE_CUDA(cudaGetLastError());
  return PFE_OK;
}

int32_t pfe_mlp_act_grad(const float* dh, const float* z, float* dz, void* dz_bf16, int64_t n, int32_t act,
                         void* stream) {
  if (!dh || !z || !dz || !dz_bf16 || n <= 0) { pfe::set_error("pfe_mlp_act_grad: bad argument"); return PFE_EINVAL; }
  pfe::k_act_grad<<<pfe::blocks_for(n), 256, 0, (cudaStream_t)stream>>>(dh, z, dz, static_cast<__nv_bfloat16*>(dz_bf16),
                                                                        n, act);
  PFE_CUDA(cudaGetLastError());
  return PFE_OK;
}

int32_t pfe_mlp_colsum(const float* dz, float* db, int32_t m, int32_t n, void* stream) {
  if (!dz || !db || m <= 0 || n <= 0) { pfe::set_error("pfe_mlp_colsum: bad argument"); return PFE_EINVAL; }
  pfe::k_colsum<<<(n + 127) / 128, 128, 0, (cudaStream_t)stream>>>(dz, db, m, n);
  PFE_CUDA(cudaGetLastError());
  return PFE_OK;
}

int32_t pfe_mlp_mse(const float* y, const float* t, const float* w, float inv_wsum, float* dy, float* loss, int64_t n,
                    void* stream) {
  if (!y || !t || !w || !dy || !loss || n <= 0) { pfe::set_error("pfe_mlp_mse: bad argument"); return PFE_EINVAL; }
  pfe::k_mse<<<pfe::blocks_for(n), 256, 0, (cudaStream_t)stream>>>(y, t, w, inv_wsum, dy, loss, n);
  PFE_CUDA(cudaGetLastError());
  return PFE_OK;
}

int32_t pfe_mlp_adam(float* w, void* w_bf16, const float* g, float* m, float* v, int64_t n, float lr, float beta1,
                     float beta2, float eps, int32_t step, float decay, void* stream) {
  if (!w || !g || !m || !v || n <= 0 || step < 1) { pfe::set_error("pfe_mlp_adam: bad argument"); return PFE_EINVAL; }
  const float c1 = 1.0f - powf(beta1, (float)step), c2 = 1.0f - powf(beta2, (float)step);
  pfe::k_adam<<<pfe::blocks_for(n), 256, 0, (cudaStream_t)stream>>>(w, static_cast<__nv_bfloat16*>(w_bf16), g, m, v, n,
                                                                     lr, beta1, beta2, eps, c1, c2, decay);
  PFE_CUDA(cudaGetLastError());
  return PFE_OK;
}

int32_t pfe_mlp_to_bf16(const float* x, void* y, int64_t n, void* stream) {
  if (!x || !y || n <= 0) { pfe::set_error("pfe_mlp_to_bf16: bad argument"); return PFE_EINVAL; }
  pfe::k_to_bf16<<<pfe::blocks_for(n), 256, 0, (cudaStream_t)stream>>>(x, static_cast<__nv_bfloat16*>(y), n);
  PFE_CUDA(cudaGetLastError());
  return PFE_OK;
}

}  // extern "C"
