// libpolymer_fock: B200 direct J/K (Fock) build behind the C ABI of
// include/polymer_fock.h.  Replaces SUBROUTINE FOURINDEX_ERI
// (src/pfourindexdirect.f90:1-814).
//
// This file holds what both build paths share: the error string, the op-table
// registry of the generated recursion, the CC contraction of primitive J'/K'
// on cuBLAS, and the FP64 peak probe.  The molecular path is pfe_mol.cu, the
// lattice / helical path pfe_lattice.cu.

#include <map>
#include <mutex>
#include <cublas_v2.h>

#include <algorithm>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <string>
#include <vector>

#include "pfe_common.cuh"
#include "pfe_context.cuh"
#include "pfe_interp.cuh"
#include "generated/eri_classes.cuh"

namespace pfe {

static thread_local std::string g_err;
void set_error(const std::string& msg) { g_err = msg; }

int upload_constants(int) { return PFE_OK; }  // constants are static-initialised

// out = A + A^T for n x n column-major matrices, batched over cells
__global__ void k_symmetrize_impl(const double* __restrict__ a, double* __restrict__ out, int n, int ncell) {
  const long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  const long long per = (long long)n * n;
  if (t >= per * ncell) return;
  const long long c = t / per, r = t % per;
  const int i = (int)(r % n), j = (int)(r / n);
  out[t] = a[c * per + i + (long long)n * j] + a[c * per + j + (long long)n * i];
}

// list the pairs of one class (any order)
__global__ void k_select_class_impl(const unsigned char* __restrict__ cls, int want, int* __restrict__ list,
                                    int* __restrict__ count, long long n) {
  const long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (t < n && cls[t] == want) list[atomicAdd(count, 1)] = (int)t;
}

void launch_symmetrize(const double* a, double* out, int n, int ncell, cudaStream_t s) {
  const long long t = (long long)n * n * ncell;
  k_symmetrize_impl<<<(unsigned)((t + 255) / 256), 256, 0, s>>>(a, out, n, ncell);
}

void launch_select_class(const unsigned char* cls, int want, int* list, int* count, long long n, cudaStream_t s) {
  k_select_class_impl<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(cls, want, list, count, n);
}

const OpTableHost* host_optable(int cb, int ck) {
  switch (cb * 8 + ck) {
    case 1 * 8 + 0: return &op_1000;
    case 1 * 8 + 1: return &op_1010;
    case 2 * 8 + 0: return &op_1100;
    case 2 * 8 + 1: return &op_1110;
    case 2 * 8 + 2: return &op_1111;
    case 3 * 8 + 0: return &op_2000;
    case 3 * 8 + 1: return &op_2010;
    case 3 * 8 + 2: return &op_2011;
    case 3 * 8 + 3: return &op_2020;
    case 4 * 8 + 0: return &op_2100;
    case 4 * 8 + 1: return &op_2110;
    case 4 * 8 + 2: return &op_2111;
    case 4 * 8 + 3: return &op_2120;
    case 4 * 8 + 4: return &op_2121;
    case 5 * 8 + 0: return &op_2200;
    case 5 * 8 + 1: return &op_2210;
    case 5 * 8 + 2: return &op_2211;
    case 5 * 8 + 3: return &op_2220;
    case 5 * 8 + 4: return &op_2221;
    case 5 * 8 + 5: return &op_2222;
    case 0: return &op_0000;
    default: return nullptr;
  }
}

// The pure-bra variant of a class's table (bra classes with a p or d shell),
// or null.
const OpTableHost* host_optable_pure(int cb, int ck) {
  switch (cb * 8 + ck) {
    case 1 * 8 + 0: return &op_1000_pure;
    case 1 * 8 + 1: return &op_1010_pure;
    case 2 * 8 + 0: return &op_1100_pure;
    case 2 * 8 + 1: return &op_1110_pure;
    case 2 * 8 + 2: return &op_1111_pure;
    case 3 * 8 + 0: return &op_2000_pure;
    case 3 * 8 + 1: return &op_2010_pure;
    case 3 * 8 + 2: return &op_2011_pure;
    case 3 * 8 + 3: return &op_2020_pure;
    case 4 * 8 + 0: return &op_2100_pure;
    case 4 * 8 + 1: return &op_2110_pure;
    case 4 * 8 + 2: return &op_2111_pure;
    case 4 * 8 + 3: return &op_2120_pure;
    case 4 * 8 + 4: return &op_2121_pure;
    case 5 * 8 + 0: return &op_2200_pure;
    case 5 * 8 + 1: return &op_2210_pure;
    case 5 * 8 + 2: return &op_2211_pure;
    case 5 * 8 + 3: return &op_2220_pure;
    case 5 * 8 + 4: return &op_2221_pure;
    case 5 * 8 + 5: return &op_2222_pure;
    case 0: return nullptr;
    default: return nullptr;
  }
}

// The variant with pure bra and pure ket shells, or null (ket classes with no
// p or d shell, and classes where it saves no op over the pure-bra table).
const OpTableHost* host_optable_pure2(int cb, int ck) {
  switch (cb * 8 + ck) {
    case 2 * 8 + 1: return &op_1110_pure2;
    case 2 * 8 + 2: return &op_1111_pure2;
    case 3 * 8 + 2: return &op_2011_pure2;
    case 4 * 8 + 1: return &op_2110_pure2;
    case 4 * 8 + 2: return &op_2111_pure2;
    case 4 * 8 + 3: return &op_2120_pure2;
    case 4 * 8 + 4: return &op_2121_pure2;
    case 5 * 8 + 1: return &op_2210_pure2;
    case 5 * 8 + 2: return &op_2211_pure2;
    case 5 * 8 + 3: return &op_2220_pure2;
    case 5 * 8 + 4: return &op_2221_pure2;
    case 5 * 8 + 5: return &op_2222_pure2;
    default: return nullptr;
  }
}

// The op tables are immutable: each is uploaded once per device and shared by
// every context on it (a batch holds hundreds of contexts).  The copies live as
// long as the process.
static std::mutex g_optable_mu;
static std::map<std::pair<int, const OpTableHost*>, OpTableDev> g_optables;

// The device view of an op table on the context's device (uploaded on first use).
int upload_optable(pfe_context* ctx, const OpTableHost* h, OpTableDev* d) {
  std::lock_guard<std::mutex> lock(g_optable_mu);
  const auto key = std::make_pair(ctx->device, h);
  const auto it = g_optables.find(key);
  if (it != g_optables.end()) {
    *d = it->second;
    return PFE_OK;
  }
  unsigned short *ops = nullptr, *out = nullptr;
  int* lev = nullptr;
  PFE_CUDA(cudaMalloc((void**)&ops, sizeof(unsigned short) * 8 * (h->nops + 1)));
  PFE_CUDA(cudaMalloc((void**)&out, sizeof(unsigned short) * (h->nout ? h->nout : 1)));
  PFE_CUDA(cudaMalloc((void**)&lev, sizeof(int) * (h->nlevels + 1)));
  {  // 16-byte records: the seven generated fields (header, five sources, destination) and a zero pad
    std::vector<unsigned short> rec((size_t)8 * (h->nops + 1), 0);
    for (int o = 0; o < h->nops; ++o)
      for (int k = 0; k < 7; ++k) rec[(size_t)8 * o + k] = h->ops[(size_t)7 * o + k];
    PFE_CUDA(cudaMemcpy(ops, rec.data(), sizeof(unsigned short) * rec.size(), cudaMemcpyHostToDevice));
  }
  PFE_CUDA(cudaMemcpy(out, h->out, sizeof(unsigned short) * h->nout, cudaMemcpyHostToDevice));
  PFE_CUDA(cudaMemcpy(lev, h->levels, sizeof(int) * (h->nlevels + 1), cudaMemcpyHostToDevice));
  d->ops = ops;
  d->out = out;
  d->levels = lev;
  d->nlevels = h->nlevels;
  d->nout = h->nout;
  d->nslots = h->nslots;
  g_optables[key] = *d;
  return PFE_OK;
}

int contract_outputs(pfe_context* ctx, const double* jp, const double* kp, double* d_cc, double* d_xc,
                     bool symmetrize, int ncell, cudaStream_t s) {
  const int np = ctx->npgs, nc = ctx->ncgs;
  const double one = 1.0, zero = 0.0;
  if (!ensure_blas(ctx)) { set_error("cublasCreate failed"); return PFE_ECUDA; }
  cublasSetStream(ctx->blas, s);
  const double* src[2] = {jp, kp};
  double* dst[2] = {d_cc, d_xc};
  for (int o = 0; o < 2; ++o) {
    // W1 = CC . M   (nc x np)(np x np) per cell
    cublasStatus_t st = cublasDgemmStridedBatched(ctx->blas, CUBLAS_OP_N, CUBLAS_OP_N, nc, np, np, &one, ctx->d_cc, nc, 0,
                                                  src[o], np, (long long)np * np, &zero, ctx->d_w1, nc,
                                                  (long long)nc * np, ncell);
    if (st != CUBLAS_STATUS_SUCCESS) { set_error("cublasDgemmStridedBatched (CC.M) failed"); return PFE_ECUDA; }
    double* target = symmetrize ? ctx->d_w2 : dst[o];
    st = cublasDgemmStridedBatched(ctx->blas, CUBLAS_OP_N, CUBLAS_OP_T, nc, nc, np, &one, ctx->d_w1, nc,
                                   (long long)nc * np, ctx->d_cc, nc, 0, &zero, target, nc, (long long)nc * nc, ncell);
    if (st != CUBLAS_STATUS_SUCCESS) { set_error("cublasDgemmStridedBatched (W.CC^T) failed"); return PFE_ECUDA; }
    if (symmetrize) {
      launch_symmetrize(ctx->d_w2, dst[o], nc, ncell, s);
      PFE_CUDA(cudaGetLastError());
    }
  }
  return PFE_OK;
}

const char* last_error_cstr() { return g_err.c_str(); }

// Independent FMA chains: 8 accumulators per thread, no memory traffic.
__global__ void k_dfma_peak(double* out, int iters, double a, double b) {
  double x0 = threadIdx.x, x1 = x0 + 1, x2 = x0 + 2, x3 = x0 + 3, x4 = x0 + 4, x5 = x0 + 5, x6 = x0 + 6, x7 = x0 + 7;
  for (int i = 0; i < iters; ++i) {
#pragma unroll
    for (int k = 0; k < 16; ++k) {
      x0 = fma(x0, a, b); x1 = fma(x1, a, b); x2 = fma(x2, a, b); x3 = fma(x3, a, b);
      x4 = fma(x4, a, b); x5 = fma(x5, a, b); x6 = fma(x6, a, b); x7 = fma(x7, a, b);
    }
  }
  const double r = x0 + x1 + x2 + x3 + x4 + x5 + x6 + x7;
  if (r == 1.2345) out[0] = r;  // keeps the chains live
}

int measure_fp64_peak(int device, double* tflops) {
  PFE_CUDA(cudaSetDevice(device));
  cudaDeviceProp prop;
  PFE_CUDA(cudaGetDeviceProperties(&prop, device));
  double* d = nullptr;
  PFE_CUDA(cudaMalloc(&d, sizeof(double)));
  const int blocks = prop.multiProcessorCount * 8, threads = 256, iters = 4096;
  cudaEvent_t e0, e1;
  PFE_CUDA(cudaEventCreate(&e0));
  PFE_CUDA(cudaEventCreate(&e1));
  k_dfma_peak<<<blocks, threads>>>(d, 64, 0.999999, 1e-7);  // warm-up
  float best = 1e30f;
  for (int r = 0; r < 5; ++r) {
    PFE_CUDA(cudaEventRecord(e0));
    k_dfma_peak<<<blocks, threads>>>(d, iters, 0.999999, 1e-7);
    PFE_CUDA(cudaEventRecord(e1));
    PFE_CUDA(cudaEventSynchronize(e1));
    float ms = 0.f;
    PFE_CUDA(cudaEventElapsedTime(&ms, e0, e1));
    best = std::min(best, ms);
  }
  const double flops = 2.0 * 8.0 * 16.0 * (double)iters * blocks * threads;
  *tflops = flops / (best * 1e-3) / 1e12;
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  cudaFree(d);
  return PFE_OK;
}

}  // namespace pfe
