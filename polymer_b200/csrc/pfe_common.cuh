// Shared device helpers of libpolymer_fock: constants, error plumbing, the
// tabulated Boys function and the cumulative-shell component counts.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>
#include <string>

#include "../../include/polymer_fock.h"
#include "generated/eri_classes.cuh"

namespace pfe {

// The reference's own constant (src/pmodules.f90:7), used wherever it enters
// normalisation/prefactors so that integrals agree with it to the last digits.
constexpr double REF_PI = 3.14159265358979;
constexpr int LMAX_SUPPORTED = 2;   // cumulative s, sp, spd shells (what the workloads use)
constexpr int NPOW = 5;             // P_SHELL power extent 0..BASIS_LMAX+1
constexpr int MAXCOMP = 10;         // components of a cumulative d shell
constexpr int NIG_T = 1701;         // IGAMMA rows (T = 0..85 step 0.05)
constexpr int NIG_M = 28;           // IGAMMA orders 0..27

__host__ __device__ constexpr int ncum(int L) { return (L + 1) * (L + 2) * (L + 3) / 6; }

void set_error(const std::string& msg);

#define PFE_CUDA(call)                                                                   \
  do {                                                                                   \
    cudaError_t e_ = (call);                                                             \
    if (e_ != cudaSuccess) {                                                             \
      ::pfe::set_error(std::string(#call) + ": " + cudaGetErrorString(e_));             \
      return (e_ == cudaErrorMemoryAllocation) ? PFE_ENOMEM : PFE_ECUDA;               \
    }                                                                                    \
  } while (0)

// Switch points of the asymptotic Boys form, TF(0:21) (src/pmodules.f90:156-159).
static __constant__ const double c_TF[22] = {33, 37, 41, 43, 46, 49, 51, 54, 56, 58, 61,
                                             63, 66, 68, 70, 72, 74, 76, 78, 80, 82, 84};

// Doubles of one IGAMMA row a Boys evaluation of orders 0..L reads (L+7 rounded
// up to even: whole 16-byte loads; rows are 28 doubles, so this stays inside one).
template <int L>
struct BoysRow {
  static constexpr int NV = (L + 8) / 2;
  static constexpr int N = 2 * NV;
};

// Gather the IGAMMA row nearest T (row-major [T][m], 16-byte aligned rows); the
// index is clamped to the table so a row can be fetched before knowing whether
// the Taylor branch will read it.
template <int L>
__device__ __forceinline__ void boys_row(double T, const double* __restrict__ tab, double* __restrict__ gv) {
  int ts = (int)floor(T * 20.0 + 0.5);
  ts = ts < NIG_T - 1 ? ts : NIG_T - 1;
  const double2* g2 = reinterpret_cast<const double2*>(tab + ts * NIG_M);
#pragma unroll
  for (int k = 0; k < BoysRow<L>::NV; ++k) {
    const double2 v = __ldg(g2 + k);
    gv[2 * k] = v.x;
    gv[2 * k + 1] = v.y;
  }
}

// F_m(T)*pref for m = 0..L exactly as the reference evaluates it
// (src/pfourindexdirect.f90:543-553): below TF(m) a 6-term Taylor series about
// the nearest tabulated point of IGAMMA (its row gv, from boys_row), above it
// the asymptotic form.  The asymptotic power T^(-m-1/2) is formed as
// rsqrt(T)*(1/T)^m instead of exp((-m-1/2) log T): same function, rounding
// differs in the last bit.
template <int L>
__device__ __forceinline__ void boys_eval(double T, double pref, const double* __restrict__ gv,
                                          double* __restrict__ F) {
  if (T < c_TF[L]) {
    const int ts = (int)floor(T * 20.0 + 0.5);  // NINT for T >= 0
    const double h = 0.05 * (double)ts - T;
#pragma unroll
    for (int m = 0; m <= L; ++m) {
      if (T < c_TF[m]) {
        F[m] = ((((((gv[m + 6] * h * 0.166666666666667 + gv[m + 5]) * h * 0.2 + gv[m + 4]) * h * 0.25 +
                   gv[m + 3]) * h * 0.333333333333333 + gv[m + 2]) * h * 0.5 + gv[m + 1]) * h + gv[m]) * pref;
      } else {
        // asymptotic prefactor F1(m) = (2m-1)!!/2^m * sqrt(PI)/2 (src/pfourindexdirect.f90:75-81)
        double v = pref * PFE_F1_0 * rsqrt(T);
        const double it = 1.0 / T;
        for (int k = 1; k <= m; ++k) v *= it * (0.5 * (double)(2 * k - 1));
        F[m] = v;
      }
    }
  } else {
    const double it = 1.0 / T;
    double v = pref * PFE_F1_0 * rsqrt(T);
    F[0] = v;
#pragma unroll
    for (int m = 1; m <= L; ++m) {
      v *= it * (0.5 * (double)(2 * m - 1));
      F[m] = v;
    }
  }
}

// Both steps; the row is read only on the Taylor branch.
template <int L>
__device__ __forceinline__ void boys_tab(double T, double pref, const double* __restrict__ tab,
                                         double* __restrict__ F) {
  double gv[BoysRow<L>::N];
  if (T < c_TF[L]) boys_row<L>(T, tab, gv);
  boys_eval<L>(T, pref, gv, F);
}

// Coefficients 1/(k! (2L+2k+1)), k = 0..17, of the Maclaurin series
// F_L(T) = sum_k (-T)^k / (k! (2L+2k+1)); at T <= 1 the omitted terms are below 1e-17.
template <int L>
struct BoysSeries {
  double c[18];
  constexpr BoysSeries() : c() {
    double f = 1.0;   // k!
    for (int k = 0; k < 18; ++k) {
      if (k > 0) f *= (double)k;
      c[k] = 1.0 / (f * (double)(2 * L + 2 * k + 1));
    }
  }
};

// F_m(T)*pref for m = 0..L (L <= 2) without reading the table, for kernels whose
// per-lane table-row gathers are what their L1 spends its wavefronts on:
//  * T >= 1: F_0 = F1(0) erf(sqrt T)/sqrt T (F1(0) = sqrt(PI)/2, the constant of the
//    asymptotic form) and upward recursion F_{m+1} = ((2m+1) F_m - e^-T)/(2T), whose
//    error grows by at most (2m+1)/(2T) <= 3/2 per step here;
//  * T < 1: the series above for F_L and downward recursion
//    F_{m-1} = (2T F_m + e^-T)/(2m-1), which is stable.
// The reference tabulates and Taylor-expands every order (boys_eval); the two agree to
// the table's own accuracy (about 1e-14 relative), far inside the build's tolerance.
template <int L>
__device__ __forceinline__ void boys_direct(double T, double pref, double* __restrict__ F) {
  static_assert(L <= 2, "boys_direct: orders 0..2");
  if (T >= 1.0) {
    const double r = rsqrt(T);
    F[0] = pref * PFE_F1_0 * erf(T * r) * r;
    if (L >= 1) {
      const double e = pref * exp(-T), h = 0.5 * r * r;
#pragma unroll
      for (int m = 0; m < L; ++m) F[m + 1] = ((double)(2 * m + 1) * F[m] - e) * h;
    }
  } else {
    constexpr BoysSeries<L> S{};
    double v = S.c[17];
#pragma unroll
    for (int k = 16; k >= 0; --k) v = fma(v, -T, S.c[k]);
    F[L] = pref * v;
    if (L >= 1) {
      const double e = pref * exp(-T);
#pragma unroll
      for (int m = L; m > 0; --m) F[m - 1] = (2.0 * T * F[m] + e) * (1.0 / (double)(2 * m - 1));
    }
  }
}

// The part of IGAMMA a Boys evaluation of orders 0..L can read -- rows 0..20*TF(L)
// (the Taylor branch is taken below TF(L)), BoysRow<L>::N columns -- staged in
// shared memory by a kernel, so that the per-lane row gathers of the quartet
// loops hit shared memory instead of L1.  `use`: it fits next to the other
// blocks of an SM (at most 96 KB).
constexpr int kTF[22] = {33, 37, 41, 43, 46, 49, 51, 54, 56, 58, 61, 63, 66, 68, 70, 72, 74, 76, 78, 80, 82, 84};

template <int L>
struct BoysSmem {
  static constexpr int ROWS = 20 * kTF[L] + 1;
  static constexpr int COLS = BoysRow<L>::N;
  static constexpr size_t BYTES = sizeof(double) * (size_t)ROWS * COLS;
  static constexpr bool use = BYTES <= 96 * 1024;
};

// Copy the rows and columns of BoysSmem<L> from the row-major table (all threads of the block).
template <int L>
__device__ __forceinline__ void boys_stage(const double* __restrict__ tab, double* __restrict__ s) {
  using B = BoysSmem<L>;
  for (int i = threadIdx.x; i < B::ROWS * B::COLS / 2; i += blockDim.x) {
    const int r = i / (B::COLS / 2), c = i % (B::COLS / 2);
    reinterpret_cast<double2*>(s)[i] = __ldg(reinterpret_cast<const double2*>(tab + (size_t)r * NIG_M) + c);
  }
}

// boys_tab with the row read from the staged copy.
template <int L>
__device__ __forceinline__ void boys_tab_smem(double T, double pref, const double* __restrict__ s,
                                              double* __restrict__ F) {
  using B = BoysSmem<L>;
  double gv[B::COLS];
  if (T < c_TF[L]) {
    const int ts = (int)floor(T * 20.0 + 0.5);   // <= 20*TF(L) = ROWS-1
    const double2* r2 = reinterpret_cast<const double2*>(s + (size_t)ts * B::COLS);
#pragma unroll
    for (int k = 0; k < B::COLS / 2; ++k) {
      const double2 v = r2[k];
      gv[2 * k] = v.x;
      gv[2 * k + 1] = v.y;
    }
  }
  boys_eval<L>(T, pref, gv, F);
}

}  // namespace pfe
