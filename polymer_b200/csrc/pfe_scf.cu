// The device side of one batched closed-shell SCF iteration around the Fock
// build (include/polymer_scf.h): density bookkeeping, Fock assembly with the
// energy, the DIIS commutator, Pulay extrapolation, the SP2 projector steps and
// the iteration's statistics.  The reference runs these steps on the host
// (FOCK_BUILD src/pfock.f90:185-337, DIIS src/pdensitymatrix.f90:253-339,
// ENERGY_CALC); the dense products between them are the caller's GEMMs.
//
// All of it is HBM-bound elementwise work over batches of n x n matrices:
// transposed reads go through 32 x 32 shared-memory tiles (both tiles of a
// mirrored pair in one block, so each element is read and written once), and
// every reduction is blockwise into per-block partials that one warp per
// molecule sums in a fixed order -- the results do not depend on scheduling.
#include <algorithm>

#include "pfe_common.cuh"
#include "../../include/polymer_scf.h"

namespace pfe {
namespace {

constexpr int TS = 32;        // tile side of the transposing kernels (blocks of 32 x 8 threads)
constexpr int CH = 8192;      // elements per block of the chunked kernels (blocks of 256 threads)
constexpr int MAXD = 16;      // DIIS history slots supported

inline int tiles_of(int n) { const int t = (n + TS - 1) / TS; return t * (t + 1) / 2; }
inline int chunks_of(int n) { return (int)(((long long)n * n + CH - 1) / CH); }

// the u-th tile of the upper triangle (ti <= tj) of T x T tiles, row by row
__device__ inline void tile_of(int u, int T, int& ti, int& tj) {
  int r = 0;
  while (u >= T - r) { u -= T - r; ++r; }
  ti = r;
  tj = r + u;
}

__device__ inline double warp_sum_d(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

__device__ inline double warp_max_d(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
  return v;
}

// Sum (or max) of v over the block, in a fixed order; valid in thread 0.
template <bool MAX>
__device__ double block_reduce(double v, double* sh) {
  const int tid = threadIdx.x + blockDim.x * threadIdx.y, nw = (blockDim.x * blockDim.y) / 32;
  v = MAX ? warp_max_d(v) : warp_sum_d(v);
  __syncthreads();   // sh may still be read by an earlier reduction
  if ((tid & 31) == 0) sh[tid >> 5] = v;
  __syncthreads();
  double r = MAX ? -INFINITY : 0.0;
  if (tid == 0)
    for (int w = 0; w < nw; ++w) r = MAX ? fmax(r, sh[w]) : r + sh[w];
  return r;
}

// out[b] = sum (or max) of part[b][0..np) (+ add[b]): one warp per molecule.
template <bool MAX>
__global__ void k_finish_partials(const double* __restrict__ part, int np, const double* __restrict__ add,
                                  double* __restrict__ out) {
  const int b = blockIdx.x;
  double v = MAX ? -INFINITY : 0.0;
  for (int k = threadIdx.x; k < np; k += 32) v = MAX ? fmax(v, part[(size_t)b * np + k]) : v + part[(size_t)b * np + k];
  v = MAX ? warp_max_d(v) : warp_sum_d(v);
  if (threadIdx.x == 0) out[b] = add ? v + add[b] : v;
}

__global__ void __launch_bounds__(256) k_next_density(int n, int nd, double* __restrict__ p,
                                                      const double* __restrict__ p_new,
                                                      const double* __restrict__ p_nuc, const uint8_t* __restrict__ take,
                                                      const uint8_t* __restrict__ restart,
                                                      const double* __restrict__ incr, const double* __restrict__ live,
                                                      const double* __restrict__ p_ref, double* __restrict__ dp,
                                                      uint8_t* __restrict__ valid) {
  const int b = blockIdx.y;
  const long long m = (long long)n * n;
  const size_t off = (size_t)b * m;
  const bool tk = take[b] != 0, rs = restart != nullptr && restart[b] != 0;
  const double inc = incr[b], lv = live[b];
  const long long x1 = min(m, (long long)(blockIdx.x + 1) * CH);
  for (long long x = (long long)blockIdx.x * CH + threadIdx.x; x < x1; x += blockDim.x) {
    double v = p[off + x];
    if (tk) v = p_new[off + x];
    if (rs) v = p_nuc[off + x];
    p[off + x] = v;
    dp[off + x] = (v - p_ref[off + x] * inc) * lv;
  }
  if (rs && blockIdx.x == 0 && threadIdx.x < nd) valid[(size_t)b * nd + threadIdx.x] = 0;
}

// One mirrored tile pair of every molecule: C, X and the references, G = H + C
// - hfx/2 X staged in shared memory, F = (G + G^T)/2, the energy's partial sum.
__global__ void __launch_bounds__(256) k_fock_assemble(int n, const double* __restrict__ h,
                                                       const double* __restrict__ d_c, const double* __restrict__ d_x,
                                                       double* __restrict__ c_ref, double* __restrict__ x_ref,
                                                       const double* __restrict__ p, double* __restrict__ p_ref,
                                                       const double* __restrict__ incr, const double* __restrict__ hfx,
                                                       double* __restrict__ f, double* __restrict__ part) {
  __shared__ double ga[TS][TS + 1], gb[TS][TS + 1];
  __shared__ double sh[32];
  const int b = blockIdx.y, T = (n + TS - 1) / TS;
  int ti, tj;
  tile_of(blockIdx.x, T, ti, tj);
  const size_t off = (size_t)b * n * n;
  const double inc = incr[b], hf = hfx[b];
  double e = 0.0;
  // g[k][tx] = G(i0 + tx, j0 + k), element (i, j) at j*n + i
  auto visit = [&](int i0, int j0, double (*g)[TS + 1]) {
    for (int k = threadIdx.y; k < TS; k += blockDim.y) {
      const int i = i0 + threadIdx.x, j = j0 + k;
      double v = 0.0;
      if (i < n && j < n) {
        const size_t x = off + (size_t)j * n + i;
        const double c = d_c[x] + inc * c_ref[x], xx = d_x[x] + inc * x_ref[x], hh = h[x], pp = p[x];
        c_ref[x] = c;
        x_ref[x] = xx;
        p_ref[x] = pp;
        v = hh + c - 0.5 * hf * xx;
        e += pp * (hh + 0.5 * c - 0.25 * hf * xx);
      }
      g[k][threadIdx.x] = v;
    }
  };
  visit(ti * TS, tj * TS, ga);
  if (ti != tj) visit(tj * TS, ti * TS, gb);
  __syncthreads();
  auto emit = [&](int i0, int j0, double (*g)[TS + 1], double (*gt)[TS + 1]) {
    for (int k = threadIdx.y; k < TS; k += blockDim.y) {
      const int i = i0 + threadIdx.x, j = j0 + k;
      if (i < n && j < n) f[off + (size_t)j * n + i] = 0.5 * (g[k][threadIdx.x] + gt[threadIdx.x][k]);
    }
  };
  if (ti == tj) {
    emit(ti * TS, tj * TS, ga, ga);
  } else {
    emit(ti * TS, tj * TS, ga, gb);
    emit(tj * TS, ti * TS, gb, ga);
  }
  const double r = block_reduce<false>(e, sh);
  if (threadIdx.x == 0 && threadIdx.y == 0) part[(size_t)b * gridDim.x + blockIdx.x] = r;
}

// E = A - A^T into the history slot, F_o beside it, the largest |E| per tile.
__global__ void __launch_bounds__(256) k_commutator(int n, int nd, const double* __restrict__ a,
                                                    const double* __restrict__ f_o, const int64_t* __restrict__ slot,
                                                    double* __restrict__ hist_e, double* __restrict__ hist_f,
                                                    uint8_t* __restrict__ valid, double* __restrict__ part) {
  __shared__ double ga[TS][TS + 1], gb[TS][TS + 1];
  __shared__ double sh[32];
  const int b = blockIdx.y, T = (n + TS - 1) / TS;
  int ti, tj;
  tile_of(blockIdx.x, T, ti, tj);
  const size_t m = (size_t)n * n, off = (size_t)b * m;
  const int s = (int)*slot;
  const size_t hoff = ((size_t)b * nd + s) * m;
  auto load = [&](int i0, int j0, double (*g)[TS + 1]) {
    for (int k = threadIdx.y; k < TS; k += blockDim.y) {
      const int i = i0 + threadIdx.x, j = j0 + k;
      double v = 0.0;
      if (i < n && j < n) {
        const size_t x = (size_t)j * n + i;
        v = a[off + x];
        hist_f[hoff + x] = f_o[off + x];
      }
      g[k][threadIdx.x] = v;
    }
  };
  load(ti * TS, tj * TS, ga);
  if (ti != tj) load(tj * TS, ti * TS, gb);
  __syncthreads();
  double mx = 0.0;
  auto emit = [&](int i0, int j0, double (*g)[TS + 1], double (*gt)[TS + 1]) {
    for (int k = threadIdx.y; k < TS; k += blockDim.y) {
      const int i = i0 + threadIdx.x, j = j0 + k;
      if (i < n && j < n) {
        const double v = g[k][threadIdx.x] - gt[threadIdx.x][k];
        hist_e[hoff + (size_t)j * n + i] = v;
        mx = fmax(mx, fabs(v));
      }
    }
  };
  if (ti == tj) {
    emit(ti * TS, tj * TS, ga, ga);
  } else {
    emit(ti * TS, tj * TS, ga, gb);
    emit(tj * TS, ti * TS, gb, ga);
  }
  const double r = block_reduce<true>(mx, sh);
  if (threadIdx.x == 0 && threadIdx.y == 0) {
    part[(size_t)b * gridDim.x + blockIdx.x] = r;
    if (blockIdx.x == 0) valid[(size_t)b * nd + s] = 1;
  }
}

// Partial dot products of the newest error vector with every history slot.
__global__ void __launch_bounds__(256) k_diis_row(int n, int nd, const double* __restrict__ hist_e,
                                                  const int64_t* __restrict__ slot, double* __restrict__ part) {
  __shared__ double sh[32];
  const int b = blockIdx.y;
  const long long m = (long long)n * n;
  const int s = (int)*slot;
  const double* es = hist_e + ((size_t)b * nd + s) * m;
  const double* eb = hist_e + (size_t)b * nd * m;
  double acc[MAXD];
#pragma unroll
  for (int d = 0; d < MAXD; ++d) acc[d] = 0.0;
  const long long x1 = min(m, (long long)(blockIdx.x + 1) * CH);
  for (long long x = (long long)blockIdx.x * CH + threadIdx.x; x < x1; x += blockDim.x) {
    const double v = es[x];
#pragma unroll
    for (int d = 0; d < MAXD; ++d)
      if (d < nd) acc[d] = fma(v, eb[(size_t)d * m + x], acc[d]);
  }
#pragma unroll
  for (int d = 0; d < MAXD; ++d) {
    if (d >= nd) break;
    const double r = block_reduce<false>(acc[d], sh);
    if (threadIdx.x == 0) part[((size_t)b * gridDim.x + blockIdx.x) * nd + d] = r;
  }
}

// The Gram row and column of the newest slot, then c = G^-1 1 / 1^T G^-1 1 over
// the valid slots (scaled, regularised; Cholesky), the newest slot alone when the
// solve is not finite.  One warp per molecule; the solve runs in lane 0.
__global__ void k_diis_solve(int nd, int nchunk, const double* __restrict__ part, const uint8_t* __restrict__ valid,
                             const int64_t* __restrict__ slot, double* __restrict__ gram, double* __restrict__ coef) {
  const int b = blockIdx.x, s = (int)*slot;
  double* G = gram + (size_t)b * nd * nd;
  if ((int)threadIdx.x < nd) {
    const int d = threadIdx.x;
    double v = 0.0;
    for (int c = 0; c < nchunk; ++c) v += part[((size_t)b * nchunk + c) * nd + d];
    G[s * nd + d] = v;
    G[d * nd + s] = v;
  }
  __syncwarp();
  if (threadIdx.x != 0) return;
  double vm[MAXD], A[MAXD][MAXD], L[MAXD][MAXD], y[MAXD], c[MAXD];
  double scale = 0.0;
  for (int i = 0; i < nd; ++i) {
    vm[i] = valid[(size_t)b * nd + i] ? 1.0 : 0.0;
    scale = fmax(scale, G[i * nd + i] * vm[i]);
  }
  scale = fmax(scale, 1e-300);
  for (int i = 0; i < nd; ++i)
    for (int j = 0; j < nd; ++j)
      A[i][j] = (G[i * nd + j] / scale) * vm[i] * vm[j] + (i == j ? 1.0 - vm[i] + vm[i] * 1e-12 : 0.0);
  for (int j = 0; j < nd; ++j) {
    double sj = A[j][j];
    for (int k = 0; k < j; ++k) sj -= L[j][k] * L[j][k];
    const double ljj = sqrt(fmax(sj, 1e-300));
    L[j][j] = ljj;
    for (int i = j + 1; i < nd; ++i) {
      double v = A[i][j];
      for (int k = 0; k < j; ++k) v -= L[i][k] * L[j][k];
      L[i][j] = v / ljj;
    }
  }
  for (int j = 0; j < nd; ++j) {
    double v = vm[j];
    for (int k = 0; k < j; ++k) v -= L[j][k] * y[k];
    y[j] = v / L[j][j];
  }
  for (int j = nd - 1; j >= 0; --j) {
    double v = y[j];
    for (int k = j + 1; k < nd; ++k) v -= L[k][j] * c[k];
    c[j] = v / L[j][j];
  }
  double sum = 0.0;
  for (int j = 0; j < nd; ++j) sum += c[j];
  bool ok = true;
  for (int j = 0; j < nd; ++j) {
    c[j] /= sum;
    ok = ok && isfinite(c[j]);
  }
  for (int j = 0; j < nd; ++j) coef[(size_t)b * nd + j] = ok ? c[j] : (j == s ? 1.0 : 0.0);
}

__global__ void __launch_bounds__(256) k_diis_extrapolate(int n, int nd, const double* __restrict__ hist_f,
                                                          const double* __restrict__ coef, double* __restrict__ f_x) {
  const int b = blockIdx.y;
  const long long m = (long long)n * n;
  double c[MAXD];
#pragma unroll
  for (int d = 0; d < MAXD; ++d) c[d] = d < nd ? coef[(size_t)b * nd + d] : 0.0;
  const double* hb = hist_f + (size_t)b * nd * m;
  const long long x1 = min(m, (long long)(blockIdx.x + 1) * CH);
  for (long long x = (long long)blockIdx.x * CH + threadIdx.x; x < x1; x += blockDim.x) {
    double v = 0.0;
#pragma unroll
    for (int d = 0; d < MAXD; ++d)
      if (d < nd) v = fma(c[d], hb[(size_t)d * m + x], v);
    f_x[(size_t)b * m + x] = v;
  }
}

// Gershgorin bounds of one molecule's F (a warp per row), then X0.
__global__ void __launch_bounds__(256) k_sp2_init(int n, const double* __restrict__ f, const uint8_t* __restrict__ pad,
                                                  double* __restrict__ x) {
  __shared__ double sh[32];
  const int b = blockIdx.x, lane = threadIdx.x & 31, w = threadIdx.x >> 5, nw = blockDim.x >> 5;
  const size_t off = (size_t)b * n * n;
  const uint8_t* pb = pad + (size_t)b * n;
  double lo = INFINITY, hi = -INFINITY;
  for (int i = w; i < n; i += nw) {
    double r = 0.0;
    for (int j = lane; j < n; j += 32) r += fabs(f[off + (size_t)i * n + j]);
    r = warp_sum_d(r);
    const double d = f[off + (size_t)i * n + i];
    r -= fabs(d);
    if (!pb[i]) {
      lo = fmin(lo, d - r);
      hi = fmax(hi, d + r);
    }
  }
  __shared__ double bounds[2];
  const double lo_b = -block_reduce<true>(-lo, sh);
  const double hi_b = block_reduce<true>(hi, sh);
  if (threadIdx.x == 0) {
    bounds[0] = lo_b;
    bounds[1] = fmax(hi_b, lo_b + 1e-8);
  }
  __syncthreads();
  const double L = bounds[0], H = bounds[1], span = H - L;
  const long long m = (long long)n * n;
  for (long long k = threadIdx.x; k < m; k += blockDim.x) {
    const int i = (int)(k / n), j = (int)(k % n);
    const double v = ((i == j ? H : 0.0) - f[off + k]) / span;
    x[off + k] = (pb[i] || pb[j]) ? 0.0 : v;
  }
}

__global__ void k_sp2_trace(int n, int nocc, const double* __restrict__ x, const double* __restrict__ x2,
                            double* __restrict__ defect, double* __restrict__ up) {
  const int b = blockIdx.x;
  const size_t off = (size_t)b * n * n;
  double t1 = 0.0, t2 = 0.0;
  for (int i = threadIdx.x; i < n; i += 32) {
    t1 += x[off + (size_t)i * n + i];
    t2 += x2[off + (size_t)i * n + i];
  }
  t1 = warp_sum_d(t1);
  t2 = warp_sum_d(t2);
  if (threadIdx.x == 0) {
    defect[b] = fabs(t1 - t2);
    up[b] = (fabs(t2 - nocc) < fabs(2.0 * t1 - t2 - nocc)) ? 1.0 : 0.0;
  }
}

__global__ void __launch_bounds__(256) k_sp2_update(int n, double* __restrict__ x, const double* __restrict__ x2,
                                                    const double* __restrict__ up) {
  const int b = blockIdx.y;
  const long long m = (long long)n * n;
  const size_t off = (size_t)b * m;
  const bool u = up[b] != 0.0;
  const long long x1 = min(m, (long long)(blockIdx.x + 1) * CH);
  for (long long k = (long long)blockIdx.x * CH + threadIdx.x; k < x1; k += blockDim.x)
    x[off + k] = u ? x2[off + k] : 2.0 * x[off + k] - x2[off + k];
}

__global__ void __launch_bounds__(256) k_finish(int n, double scale, const double* __restrict__ q,
                                                const double* __restrict__ p, double* __restrict__ p_new,
                                                double* __restrict__ part) {
  __shared__ double sh[32];
  const int b = blockIdx.y;
  const long long m = (long long)n * n;
  const size_t off = (size_t)b * m;
  double acc = 0.0;
  const long long x1 = min(m, (long long)(blockIdx.x + 1) * CH);
  for (long long k = (long long)blockIdx.x * CH + threadIdx.x; k < x1; k += blockDim.x) {
    const double v = scale * q[off + k];
    p_new[off + k] = v;
    const double d = v - p[off + k];
    acc = fma(d, d, acc);
  }
  const double r = block_reduce<false>(acc, sh);
  if (threadIdx.x == 0) part[(size_t)b * gridDim.x + blockIdx.x] = r;
}

__global__ void k_finish_stats(int n, int nchunk, const double* __restrict__ part, const double* __restrict__ energy,
                               const double* __restrict__ err_max, const double* __restrict__ defect,
                               double* __restrict__ stats) {
  const int b = blockIdx.x;
  double v = 0.0;
  for (int k = threadIdx.x; k < nchunk; k += 32) v += part[(size_t)b * nchunk + k];
  v = warp_sum_d(v);
  if (threadIdx.x == 0) {
    stats[(size_t)b * 4 + 0] = energy[b];
    stats[(size_t)b * 4 + 1] = err_max[b];
    stats[(size_t)b * 4 + 2] = sqrt(v / ((double)n * (double)n));
    stats[(size_t)b * 4 + 3] = defect[b];
  }
}

bool bad_batch(const char* fn, int nb, int n) {
  if (nb < 0 || n <= 0 || (long long)nb * n * n > (1LL << 40)) {
    set_error(std::string(fn) + ": bad batch shape");
    return true;
  }
  return false;
}

}  // namespace
}  // namespace pfe

using namespace pfe;

extern "C" {

int64_t pfe_scf_workspace(int32_t nb, int32_t n, int32_t ndiis) {
  if (nb < 0 || n <= 0 || ndiis < 0) return 0;
  const long long per = std::max<long long>({(long long)tiles_of(n), (long long)chunks_of(n) * std::max(ndiis, 1), 1LL});
  return (int64_t)nb * per;
}

int32_t pfe_scf_next_density(int32_t nb, int32_t n, int32_t ndiis, double* p, const double* p_new, const double* p_nuc,
                             const uint8_t* take, const uint8_t* restart, const double* incr, const double* live,
                             const double* p_ref, double* dp, uint8_t* valid, void* stream) {
  if (bad_batch("pfe_scf_next_density", nb, n)) return PFE_EINVAL;
  if (!p || !p_new || !take || !incr || !live || !p_ref || !dp || ndiis < 1 || ndiis > MAXD ||
      (restart && (!p_nuc || !valid))) {
    set_error("pfe_scf_next_density: bad argument");
    return PFE_EINVAL;
  }
  if (nb == 0) return PFE_OK;
  k_next_density<<<dim3(chunks_of(n), nb), 256, 0, (cudaStream_t)stream>>>(n, ndiis, p, p_new, p_nuc, take, restart,
                                                                            incr, live, p_ref, dp, valid);
  PFE_CUDA(cudaGetLastError());
  return PFE_OK;
}

int32_t pfe_scf_fock_assemble(int32_t nb, int32_t n, const double* h, const double* d_c, const double* d_x,
                              double* c_ref, double* x_ref, const double* p, double* p_ref, const double* incr,
                              const double* hfx, const double* e_nuc, double* f, double* energy, double* work,
                              void* stream) {
  if (bad_batch("pfe_scf_fock_assemble", nb, n)) return PFE_EINVAL;
  if (!h || !d_c || !d_x || !c_ref || !x_ref || !p || !p_ref || !incr || !hfx || !e_nuc || !f || !energy || !work) {
    set_error("pfe_scf_fock_assemble: null pointer");
    return PFE_EINVAL;
  }
  if (nb == 0) return PFE_OK;
  cudaStream_t s = (cudaStream_t)stream;
  const int nt = tiles_of(n);
  k_fock_assemble<<<dim3(nt, nb), dim3(TS, 8), 0, s>>>(n, h, d_c, d_x, c_ref, x_ref, p, p_ref, incr, hfx, f, work);
  k_finish_partials<false><<<nb, 32, 0, s>>>(work, nt, e_nuc, energy);
  PFE_CUDA(cudaGetLastError());
  return PFE_OK;
}

int32_t pfe_scf_commutator(int32_t nb, int32_t n, int32_t ndiis, const double* a, const double* f_o,
                           const int64_t* slot, double* hist_e, double* hist_f, uint8_t* valid, double* err_max,
                           double* work, void* stream) {
  if (bad_batch("pfe_scf_commutator", nb, n)) return PFE_EINVAL;
  if (!a || !f_o || !slot || !hist_e || !hist_f || !valid || !err_max || !work || ndiis < 1 || ndiis > MAXD) {
    set_error("pfe_scf_commutator: bad argument");
    return PFE_EINVAL;
  }
  if (nb == 0) return PFE_OK;
  cudaStream_t s = (cudaStream_t)stream;
  const int nt = tiles_of(n);
  k_commutator<<<dim3(nt, nb), dim3(TS, 8), 0, s>>>(n, ndiis, a, f_o, slot, hist_e, hist_f, valid, work);
  k_finish_partials<true><<<nb, 32, 0, s>>>(work, nt, nullptr, err_max);
  PFE_CUDA(cudaGetLastError());
  return PFE_OK;
}

int32_t pfe_scf_diis(int32_t nb, int32_t n, int32_t ndiis, const double* hist_e, const double* hist_f,
                     const uint8_t* valid, const int64_t* slot, double* gram, double* coef, double* f_x, double* work,
                     void* stream) {
  if (bad_batch("pfe_scf_diis", nb, n)) return PFE_EINVAL;
  if (!hist_e || !hist_f || !valid || !slot || !gram || !coef || !f_x || !work || ndiis < 1 || ndiis > MAXD) {
    set_error("pfe_scf_diis: bad argument");
    return PFE_EINVAL;
  }
  if (nb == 0) return PFE_OK;
  cudaStream_t s = (cudaStream_t)stream;
  const int nc = chunks_of(n);
  k_diis_row<<<dim3(nc, nb), 256, 0, s>>>(n, ndiis, hist_e, slot, work);
  k_diis_solve<<<nb, 32, 0, s>>>(ndiis, nc, work, valid, slot, gram, coef);
  k_diis_extrapolate<<<dim3(nc, nb), 256, 0, s>>>(n, ndiis, hist_f, coef, f_x);
  PFE_CUDA(cudaGetLastError());
  return PFE_OK;
}

int32_t pfe_scf_sp2_init(int32_t nb, int32_t n, const double* f, const uint8_t* pad, double* x, void* stream) {
  if (bad_batch("pfe_scf_sp2_init", nb, n)) return PFE_EINVAL;
  if (!f || !pad || !x) {
    set_error("pfe_scf_sp2_init: null pointer");
    return PFE_EINVAL;
  }
  if (nb == 0) return PFE_OK;
  k_sp2_init<<<nb, 256, 0, (cudaStream_t)stream>>>(n, f, pad, x);
  PFE_CUDA(cudaGetLastError());
  return PFE_OK;
}

int32_t pfe_scf_sp2_step(int32_t nb, int32_t n, int32_t nocc, double* x, const double* x2, double* defect, double* work,
                         void* stream) {
  if (bad_batch("pfe_scf_sp2_step", nb, n)) return PFE_EINVAL;
  if (!x || !x2 || !defect || !work || nocc < 0 || nocc > n) {
    set_error("pfe_scf_sp2_step: bad argument");
    return PFE_EINVAL;
  }
  if (nb == 0) return PFE_OK;
  cudaStream_t s = (cudaStream_t)stream;
  k_sp2_trace<<<nb, 32, 0, s>>>(n, nocc, x, x2, defect, work);
  k_sp2_update<<<dim3(chunks_of(n), nb), 256, 0, s>>>(n, x, x2, work);
  PFE_CUDA(cudaGetLastError());
  return PFE_OK;
}

int32_t pfe_scf_finish(int32_t nb, int32_t n, double scale, const double* q, const double* p, double* p_new,
                       const double* energy, const double* err_max, const double* defect, double* stats, double* work,
                       void* stream) {
  if (bad_batch("pfe_scf_finish", nb, n)) return PFE_EINVAL;
  if (!q || !p || !p_new || !energy || !err_max || !defect || !stats || !work) {
    set_error("pfe_scf_finish: null pointer");
    return PFE_EINVAL;
  }
  if (nb == 0) return PFE_OK;
  cudaStream_t s = (cudaStream_t)stream;
  const int nc = chunks_of(n);
  k_finish<<<dim3(nc, nb), 256, 0, s>>>(n, scale, q, p, p_new, work);
  k_finish_stats<<<nb, 32, 0, s>>>(n, nc, work, energy, err_max, defect, stats);
  PFE_CUDA(cudaGetLastError());
  return PFE_OK;
}

}  // extern "C"
