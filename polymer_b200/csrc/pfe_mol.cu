// Molecular path of the Fock build (all cells 0, HELIX 0).
//
// Set-up (device):
//   * every unordered primitive-shell pair, oriented higher L first, then
//     higher contracted block, then higher shell index, with the reference's
//     Schwarz bound (component 1 excluded, src/pfourindexdirect.f90:326-363);
//   * pairs grouped by ordered contracted block pair ("group"): the pairs of a
//     group feed the same contracted J/K elements;
//   * sorted by (class, group's largest bound desc, group, bound desc), so the
//     groups a bra can reach form a prefix of each ket class and the pairs of a
//     group are adjacent;
//   * per (bra class, ket class) the screened triangle in 32-ket chunks.
// Build:
//   * k_quartets (straight-line, one quartet per lane): the reference's screen
//     IJIJ*KLKL >= INTTOL per lane (src/pfourindexdirect.f90:529); digestion with
//     8-fold symmetry into contracted targets; lanes of one group reduce with a
//     segmented warp reduction before one FP64 atomic per segment;
//   * k_quartets_warp / k_quartets_big (op-table interpreter, one quartet per
//     warp / block) for the larger classes, accumulating a group's quartets in
//     registers before its atomics;
//   * C_C = J' + J'^T and X_C = K' + K'^T (contracted targets), or the cuBLAS
//     contraction CC (J'+J'^T) CC^T when CC is a general contraction.

#include <cublas_v2.h>
#include <cub/cub.cuh>

#include <algorithm>
#include <vector>

#include "pfe_common.cuh"
#include "pfe_context.cuh"
#include "pfe_interp.cuh"
#include "generated/eri_classes.cuh"

namespace pfe {

struct MolLaunch {
  PairArrays pairs;
  const int* prim;       // shell components -> primitive
  const int* tidx;       // primitive -> target row (-1: none)
  const double* tcoef;   // primitive -> coefficient
  const double* boys;
  const double* density; // P_P (npgs x npgs, column-major)
  double* jt;            // J' targets (nt x nt)
  double* kt;            // K' targets
  const int4* chunks;    // (bra pair, first ket, end ket, 0)
  const int* nchunks;
  double inttol;
  int npgs, nt;
  int myid, numprocs;
};

static const int kCL[6][2] = {{0, 0}, {1, 0}, {1, 1}, {2, 0}, {2, 1}, {2, 2}};

// ------------------------------------------------------------------ set-up

__global__ void k_mol_pairs(DevShells sh, const int* __restrict__ blk, int nblk, const double* __restrict__ sss,
                            const double* __restrict__ tab, const double* __restrict__ maxc, PairArrays out,
                            int* __restrict__ class_count, long long npairs) {
  const long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (t >= npairs) return;
  long long i = (long long)((sqrt(8.0 * (double)t + 1.0) - 1.0) * 0.5);
  while ((i + 1) * (i + 2) / 2 <= t) ++i;
  while (i * (i + 1) / 2 > t) --i;
  int I = (int)i, J = (int)(t - i * (i + 1) / 2);
  // orientation: higher L first; equal L: higher block; equal block: higher index
  bool swap = false;
  if (sh.L[J] != sh.L[I]) swap = sh.L[J] > sh.L[I];
  else if (blk[J] != blk[I]) swap = blk[J] > blk[I];
  if (swap) { const int x = I; I = J; J = x; }
  const double za = sh.zeta[I], zb = sh.zeta[J];
  const double ax = sh.x[I], ay = sh.y[I], az = sh.z[I];
  const double bx = sh.x[J], by = sh.y[J], bz = sh.z[J];
  const double z = za + zb;
  const double px = (ax * za + bx * zb) / z, py = (ay * za + by * zb) / z, pz = (az * za + bz * zb) / z;
  const double S = sss[(size_t)I + (size_t)sh.n * J];
  const double PA[3] = {px - ax, py - ay, pz - az}, AB[3] = {ax - bx, ay - by, az - bz};
  const int la = sh.L[I], lb = sh.L[J];
  const int* pa = sh.prim + (size_t)I * MAXCOMP;
  const int* pb = sh.prim + (size_t)J * MAXCOMP;
  const int cls = pair_class(la, lb);
  double sch = 0.0;
  switch (cls) {
    case 0: sch = schwarz_pair<0, 0>(tab, z, S, PA, AB, pa, pb, maxc); break;
    case 1: sch = schwarz_pair<1, 0>(tab, z, S, PA, AB, pa, pb, maxc); break;
    case 2: sch = schwarz_pair<1, 1>(tab, z, S, PA, AB, pa, pb, maxc); break;
    case 3: sch = schwarz_pair<2, 0>(tab, z, S, PA, AB, pa, pb, maxc); break;
    default: sch = 0.0; break;  // (21), (22): k_schwarz_big
  }
  out.P[0][t] = px; out.P[1][t] = py; out.P[2][t] = pz;
  out.PA[0][t] = PA[0]; out.PA[1][t] = PA[1]; out.PA[2][t] = PA[2];
  out.AB[0][t] = AB[0]; out.AB[1][t] = AB[1]; out.AB[2][t] = AB[2];
  out.zeta[t] = z;
  out.S[t] = S;
  out.schwarz[t] = sch;
  out.si[t] = I;
  out.sj[t] = J;
  out.cls[t] = (unsigned char)cls;
  out.gid[t] = blk[I] * nblk + blk[J];
  atomicAdd(class_count + cls, 1);
}

__global__ void k_mol_groupmax(const double* __restrict__ sch, const int* __restrict__ gid,
                               unsigned long long* __restrict__ gmax_bits, long long n) {
  const long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (t < n) atomicMax(gmax_bits + gid[t], (unsigned long long)__double_as_longlong(sch[t]));
}

__global__ void k_mol_keys(const double* __restrict__ sch, const int* __restrict__ gid,
                           const unsigned long long* __restrict__ gmax_bits, unsigned long long* __restrict__ k_sch,
                           unsigned long long* __restrict__ k_gmax, double* __restrict__ gmax, long long n) {
  const long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (t >= n) return;
  k_sch[t] = ~(unsigned long long)__double_as_longlong(sch[t]);   // descending bound
  const unsigned long long gb = gmax_bits[gid[t]];
  k_gmax[t] = ~gb;                                                // descending group max
  gmax[t] = __longlong_as_double((long long)gb);
}

template <typename T>
__global__ void k_gather_t(const T* __restrict__ src, const int* __restrict__ perm, T* __restrict__ dst, long long n) {
  const long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (t < n) dst[t] = src[perm[t]];
}

__global__ void k_mol_iota(int* p, long long n) {
  const long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (t < n) p[t] = (int)t;
}

__global__ void k_mol_gather(PairArrays src, PairArrays dst, const int* __restrict__ perm, long long n) {
  const long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (t >= n) return;
  const int s = perm[t];
  for (int k = 0; k < 3; ++k) {
    dst.P[k][t] = src.P[k][s];
    dst.PA[k][t] = src.PA[k][s];
    dst.AB[k][t] = src.AB[k][s];
  }
  dst.zeta[t] = src.zeta[s];
  dst.S[t] = src.S[s];
  dst.schwarz[t] = src.schwarz[s];
  dst.si[t] = src.si[s];
  dst.sj[t] = src.sj[s];
  dst.cls[t] = src.cls[s];
  dst.gid[t] = src.gid[s];
  dst.gmax[t] = src.gmax[s];
}

// Ket range of bra p: the groups whose largest bound passes the screen with p
// (a prefix, groups being ordered by that bound), cut at q <= p for one class;
// also counts the quartets that pass individually.
__global__ void k_mol_count(const double* __restrict__ sch, const double* __restrict__ gmax, int b0, int nb, int k0,
                            int nk, bool same, double inttol, int* __restrict__ nrange, int* __restrict__ nchunk,
                            int* __restrict__ nquart) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= nb) return;
  const double sp = sch[b0 + p];
  int lo = 0, hi = nk;
  while (lo < hi) {
    const int mid = (lo + hi) >> 1;
    if (sp * gmax[k0 + mid] < inttol) hi = mid; else lo = mid + 1;
  }
  int e = lo;
  if (same && e > p + 1) e = p + 1;
  int nq = 0;
  for (int q = 0; q < e; ++q) nq += (sp * sch[k0 + q] < inttol) ? 0 : 1;
  nrange[p] = e;
  nchunk[p] = (e + 31) >> 5;
  nquart[p] = nq;
}

__global__ void k_mol_fill(const int* __restrict__ nrange, const int* __restrict__ off, int b0, int k0, int nb,
                           int4* __restrict__ chunks) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= nb) return;
  const int e = nrange[p];
  int o = off[p];
  for (int q = 0; q < e; q += 32, ++o) chunks[o] = make_int4(b0 + p, k0 + q, k0 + min(q + 32, e), 0);
}

// ------------------------------------------------------------------ digestion helpers

// Sum over the lanes of this lane's segment [lane, seg_end] (segments are
// contiguous lane ranges); the segment's first lane ends with the full sum.
__device__ __forceinline__ double seg_sum(double v, int lane, int seg_end) {
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const double w = __shfl_down_sync(0xffffffffu, v, o);
    if (lane + o <= seg_end) v += w;
  }
  return v;
}

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

__device__ __forceinline__ void add_target(double* __restrict__ M, int nt, int r, int c, double v) {
  if (r >= 0 && c >= 0 && v != 0.0) atomicAdd(M + r + (size_t)nt * c, v);
}

template <int NA, int NB, int NC, int ND>
struct Digest {
  double Pab[NA * NB], Pcd[NC * ND], Pac[NA * NC], Pad[NA * ND], Pbc[NB * NC], Pbd[NB * ND];
  double jab[NA * NB], jcd[NC * ND], kad[NA * ND], kbd[NB * ND], kac[NA * NC], kbc[NB * NC];
};

// ------------------------------------------------------------------ straight-line classes

template <int LA, int LB, int LC, int LD>
__global__ void __launch_bounds__(128) k_quartets(MolLaunch ql) {
  constexpr int NA = ncum(LA), NB = ncum(LB), NC = ncum(LC), ND = ncum(LD);
  constexpr int NI = NA * NB * NC * ND;
  constexpr int LT = LA + LB + LC + LD;
  const int lane = threadIdx.x & 31;
  const int wpb = blockDim.x >> 5;
  const int nchunks = *ql.nchunks;
  const int stride = gridDim.x * wpb * ql.numprocs;
  const double c2pi = 2.0 / sqrt(REF_PI);
  const PairArrays pr = ql.pairs;
  const int npgs = ql.npgs, nt = ql.nt;
  const double* __restrict__ D = ql.density;
  for (int c = (blockIdx.x * wpb + (threadIdx.x >> 5)) * ql.numprocs + ql.myid; c < nchunks; c += stride) {
    const int4 ch = ql.chunks[c];
    const int p = ch.x;
    const int q = ch.y + lane;
    const bool act = q < ch.z;
    const int qq = act ? q : ch.y;
    const double sp = pr.schwarz[p];
    const bool valid = act && !(sp * pr.schwarz[qq] < ql.inttol);
    const double zb = pr.zeta[p], ze = pr.zeta[qq];
    const double Px = pr.P[0][p], Py = pr.P[1][p], Pz = pr.P[2][p];
    const double Qx = pr.P[0][qq], Qy = pr.P[1][qq], Qz = pr.P[2][qq];
    const double zz = zb + ze;
    const double rho = zb * ze / zz;
    const double dx = Px - Qx, dy = Py - Qy, dz = Pz - Qz;
    const double T = rho * (dx * dx + dy * dy + dz * dz);
    const double pref = c2pi * pr.S[p] * pr.S[qq] * sqrt(rho);
    double F[LT + 1];
    boys_tab<LT>(T, pref, ql.boys, F);
    double out[NI];
    if constexpr (LT == 0) {
      out[0] = F[0];
    } else {
      EriGeom<double> g;
      const double Wx = (zb * Px + ze * Qx) / zz, Wy = (zb * Py + ze * Qy) / zz, Wz = (zb * Pz + ze * Qz) / zz;
      g.PA[0] = pr.PA[0][p]; g.PA[1] = pr.PA[1][p]; g.PA[2] = pr.PA[2][p];
      g.QC[0] = pr.PA[0][qq]; g.QC[1] = pr.PA[1][qq]; g.QC[2] = pr.PA[2][qq];
      g.AB[0] = pr.AB[0][p]; g.AB[1] = pr.AB[1][p]; g.AB[2] = pr.AB[2][p];
      g.CD[0] = pr.AB[0][qq]; g.CD[1] = pr.AB[1][qq]; g.CD[2] = pr.AB[2][qq];
      g.WP[0] = Wx - Px; g.WP[1] = Wy - Py; g.WP[2] = Wz - Pz;
      g.WQ[0] = Wx - Qx; g.WQ[1] = Wy - Qy; g.WQ[2] = Wz - Qz;
      g.oz = 0.5 / zb; g.oe = 0.5 / ze; g.oze = 0.5 / zz; g.roz = rho / zb; g.roe = rho / ze;
      eri_dispatch<LA, LB, LC, LD>(F, g, out);
    }
    const int I = pr.si[p], J = pr.sj[p], K = pr.si[qq], L = pr.sj[qq];
    const double deg = (I != J ? 2.0 : 1.0) * (K != L ? 2.0 : 1.0) * (p != qq ? 2.0 : 1.0);
    const double wj = valid ? 0.25 * deg : 0.0, wk = valid ? 0.125 * deg : 0.0;
    int pa[NA], pb[NB], pc[NC], pd[ND];
#pragma unroll
    for (int x = 0; x < NA; ++x) pa[x] = ql.prim[I * MAXCOMP + x];
#pragma unroll
    for (int x = 0; x < NB; ++x) pb[x] = ql.prim[J * MAXCOMP + x];
#pragma unroll
    for (int x = 0; x < NC; ++x) pc[x] = ql.prim[K * MAXCOMP + x];
#pragma unroll
    for (int x = 0; x < ND; ++x) pd[x] = ql.prim[L * MAXCOMP + x];
    Digest<NA, NB, NC, ND> dg;
#pragma unroll
    for (int a = 0; a < NA; ++a) {
#pragma unroll
      for (int b = 0; b < NB; ++b) { dg.Pab[a * NB + b] = dens_at(D, npgs, pa[a], pb[b]); dg.jab[a * NB + b] = 0.0; }
#pragma unroll
      for (int cc = 0; cc < NC; ++cc) { dg.Pac[a * NC + cc] = dens_at(D, npgs, pa[a], pc[cc]); dg.kac[a * NC + cc] = 0.0; }
#pragma unroll
      for (int d = 0; d < ND; ++d) { dg.Pad[a * ND + d] = dens_at(D, npgs, pa[a], pd[d]); dg.kad[a * ND + d] = 0.0; }
    }
#pragma unroll
    for (int b = 0; b < NB; ++b) {
#pragma unroll
      for (int cc = 0; cc < NC; ++cc) { dg.Pbc[b * NC + cc] = dens_at(D, npgs, pb[b], pc[cc]); dg.kbc[b * NC + cc] = 0.0; }
#pragma unroll
      for (int d = 0; d < ND; ++d) { dg.Pbd[b * ND + d] = dens_at(D, npgs, pb[b], pd[d]); dg.kbd[b * ND + d] = 0.0; }
    }
#pragma unroll
    for (int cc = 0; cc < NC; ++cc)
#pragma unroll
      for (int d = 0; d < ND; ++d) { dg.Pcd[cc * ND + d] = dens_at(D, npgs, pc[cc], pd[d]); dg.jcd[cc * ND + d] = 0.0; }
#pragma unroll
    for (int a = 0; a < NA; ++a)
#pragma unroll
      for (int b = 0; b < NB; ++b)
#pragma unroll
        for (int cc = 0; cc < NC; ++cc)
#pragma unroll
          for (int d = 0; d < ND; ++d) {
            const double v = out[((a * NB + b) * NC + cc) * ND + d];
            dg.jab[a * NB + b] += dg.Pcd[cc * ND + d] * v;
            dg.jcd[cc * ND + d] += dg.Pab[a * NB + b] * v;
            dg.kad[a * ND + d] += dg.Pbc[b * NC + cc] * v;
            dg.kbd[b * ND + d] += dg.Pac[a * NC + cc] * v;
            dg.kac[a * NC + cc] += dg.Pbd[b * ND + d] * v;
            dg.kbc[b * NC + cc] += dg.Pad[a * ND + d] * v;
          }
    // targets and coefficients of every component
    int ta[NA], tb[NB], tc[NC], td[ND];
    double ca[NA], cb[NB], cc_[NC], cd[ND];
#pragma unroll
    for (int x = 0; x < NA; ++x) { ta[x] = ql.tidx[pa[x]]; ca[x] = ql.tcoef[pa[x]]; }
#pragma unroll
    for (int x = 0; x < NB; ++x) { tb[x] = ql.tidx[pb[x]]; cb[x] = ql.tcoef[pb[x]]; }
#pragma unroll
    for (int x = 0; x < NC; ++x) { tc[x] = ql.tidx[pc[x]]; cc_[x] = ql.tcoef[pc[x]]; }
#pragma unroll
    for (int x = 0; x < ND; ++x) { td[x] = ql.tidx[pd[x]]; cd[x] = ql.tcoef[pd[x]]; }
    // segments: consecutive lanes of one contracted block pair share every target
    const int g = act ? pr.gid[qq] : -1 - lane;
    const unsigned seg = __match_any_sync(0xffffffffu, g);
    const int seg_end = 31 - __clz(seg);
    const bool head = lane == (__ffs(seg) - 1);
    // J'(ab): the whole warp shares the bra (and its coefficients)
#pragma unroll
    for (int a = 0; a < NA; ++a)
#pragma unroll
      for (int b = 0; b < NB; ++b) {
        const double v = warp_sum(dg.jab[a * NB + b] * wj);
        if (lane == 0) add_target(ql.jt, nt, ta[a], tb[b], v * ca[a] * cb[b]);
      }
    // the rest: every lane weighs by its own ket coefficients, then the
    // segment sums and its first lane adds
#pragma unroll
    for (int cc = 0; cc < NC; ++cc)
#pragma unroll
      for (int d = 0; d < ND; ++d) {
        const double v = seg_sum(dg.jcd[cc * ND + d] * wj * cc_[cc] * cd[d], lane, seg_end);
        if (head) add_target(ql.jt, nt, tc[cc], td[d], v);
      }
#pragma unroll
    for (int a = 0; a < NA; ++a) {
#pragma unroll
      for (int d = 0; d < ND; ++d) {
        const double v = seg_sum(dg.kad[a * ND + d] * wk * cd[d], lane, seg_end);
        if (head) add_target(ql.kt, nt, ta[a], td[d], v * ca[a]);
      }
#pragma unroll
      for (int cc = 0; cc < NC; ++cc) {
        const double v = seg_sum(dg.kac[a * NC + cc] * wk * cc_[cc], lane, seg_end);
        if (head) add_target(ql.kt, nt, ta[a], tc[cc], v * ca[a]);
      }
    }
#pragma unroll
    for (int b = 0; b < NB; ++b) {
#pragma unroll
      for (int d = 0; d < ND; ++d) {
        const double v = seg_sum(dg.kbd[b * ND + d] * wk * cd[d], lane, seg_end);
        if (head) add_target(ql.kt, nt, tb[b], td[d], v * cb[b]);
      }
#pragma unroll
      for (int cc = 0; cc < NC; ++cc) {
        const double v = seg_sum(dg.kbc[b * NC + cc] * wk * cc_[cc], lane, seg_end);
        if (head) add_target(ql.kt, nt, tb[b], tc[cc], v * cb[b]);
      }
    }
  }
}

// ------------------------------------------------------------------ interpreted classes

// Digestion targets of one quartet, t in [0, NT): J'(ab), J'(cd), K'(ad),
// K'(bd), K'(ac), K'(bc).  slots(): the matrix (0 = J', 1 = K') and the two
// component slots (a: 0.., b: NA.., c: NA+NB.., d: NA+NB+NC..) of target t;
// value(): its density-weighted sum over the quartet's integrals.
template <int NA, int NB, int NC, int ND>
struct Targets {
  static constexpr int NT = NA * NB + NC * ND + (NA + NB) * (NC + ND);
  static constexpr int SB = NA, SC = NA + NB, SD = NA + NB + NC;
  __device__ static void slots(int t, int* kind, int* s1, int* s2) {
    int r = t;
    if (r < NA * NB) { *kind = 0; *s1 = r / NB; *s2 = SB + r % NB; return; }
    r -= NA * NB;
    if (r < NC * ND) { *kind = 0; *s1 = SC + r / ND; *s2 = SD + r % ND; return; }
    r -= NC * ND;
    if (r < NA * ND) { *kind = 1; *s1 = r / ND; *s2 = SD + r % ND; return; }
    r -= NA * ND;
    if (r < NB * ND) { *kind = 1; *s1 = SB + r / ND; *s2 = SD + r % ND; return; }
    r -= NB * ND;
    if (r < NA * NC) { *kind = 1; *s1 = r / NC; *s2 = SC + r % NC; return; }
    r -= NA * NC;
    *kind = 1; *s1 = SB + r / NC; *s2 = SC + r % NC;
  }
  __device__ static double value(int t, const double* __restrict__ v, const unsigned short* __restrict__ out,
                                 const double* Pab, const double* Pcd, const double* Pac, const double* Pad,
                                 const double* Pbc, const double* Pbd) {
    double acc = 0.0;
    int r = t;
    if (r < NA * NB) {
      const int a = r / NB, b = r % NB;
      for (int cc = 0; cc < NC; ++cc)
        for (int d = 0; d < ND; ++d) acc += Pcd[cc * ND + d] * v[out[((a * NB + b) * NC + cc) * ND + d]];
      return acc;
    }
    r -= NA * NB;
    if (r < NC * ND) {
      const int cc = r / ND, d = r % ND;
      for (int a = 0; a < NA; ++a)
        for (int b = 0; b < NB; ++b) acc += Pab[a * NB + b] * v[out[((a * NB + b) * NC + cc) * ND + d]];
      return acc;
    }
    r -= NC * ND;
    if (r < NA * ND) {
      const int a = r / ND, d = r % ND;
      for (int b = 0; b < NB; ++b)
        for (int cc = 0; cc < NC; ++cc) acc += Pbc[b * NC + cc] * v[out[((a * NB + b) * NC + cc) * ND + d]];
      return acc;
    }
    r -= NA * ND;
    if (r < NB * ND) {
      const int b = r / ND, d = r % ND;
      for (int a = 0; a < NA; ++a)
        for (int cc = 0; cc < NC; ++cc) acc += Pac[a * NC + cc] * v[out[((a * NB + b) * NC + cc) * ND + d]];
      return acc;
    }
    r -= NB * ND;
    if (r < NA * NC) {
      const int a = r / NC, cc = r % NC;
      for (int b = 0; b < NB; ++b)
        for (int d = 0; d < ND; ++d) acc += Pbd[b * ND + d] * v[out[((a * NB + b) * NC + cc) * ND + d]];
      return acc;
    }
    r -= NA * NC;
    const int b = r / NC, cc = r % NC;
    for (int a = 0; a < NA; ++a)
      for (int d = 0; d < ND; ++d) acc += Pad[a * ND + d] * v[out[((a * NB + b) * NC + cc) * ND + d]];
    return acc;
  }
};

// One quartet per warp (several warps per block) on the level-scheduled op
// table.  When a class has at most 256 targets, each lane keeps its targets'
// coefficient-weighted sums in registers while consecutive kets belong to one
// contracted block pair (same contracted targets) and adds them once per run;
// the bra's J'(ab) is added once per chunk.
template <int LA, int LB, int LC, int LD>
__global__ void __launch_bounds__(256) k_quartets_warp(MolLaunch ql, OpTableDev tab, int per_warp) {
  constexpr int NA = ncum(LA), NB = ncum(LB), NC = ncum(LC), ND = ncum(LD);
  constexpr int LT = LA + LB + LC + LD;
  using TG = Targets<NA, NB, NC, ND>;
  constexpr int NT = TG::NT;
  constexpr int NPRM = NA + NB + NC + ND;
  constexpr int NR = (NT + 31) / 32;
  constexpr bool HOLD = NR <= 8;
  extern __shared__ double smem[];
  __shared__ OpGeom s_geo[8];
  __shared__ int s_prm[8][NPRM];
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, wpb = blockDim.x >> 5;
  double* v = smem + (size_t)wid * per_warp;
  double* Pab = v + tab.nslots;
  double* Pcd = Pab + NA * NB;
  double* Pac = Pcd + NC * ND;
  double* Pad = Pac + NA * NC;
  double* Pbc = Pad + NA * ND;
  double* Pbd = Pbc + NB * NC;
  OpGeom& geo = s_geo[wid];
  int* prm = s_prm[wid];
  const PairArrays pr = ql.pairs;
  const int npgs = ql.npgs, nt = ql.nt;
  const double* __restrict__ D = ql.density;
  const int nchunks = *ql.nchunks;
  const double c2pi = 2.0 / sqrt(REF_PI);
  const int base = LT + 2;
  const int stride = gridDim.x * wpb * ql.numprocs;
  double hold[HOLD ? NR : 1];
  // adds the held sums of this lane's targets; ket slots of prm still hold a
  // member of the run being flushed (all members share their targets)
  auto flush = [&](bool with_bra) {
#pragma unroll
    for (int r = 0; r < (HOLD ? NR : 0); ++r) {
      const int t = lane + 32 * r;
      if (t < NT && (with_bra || t >= NA * NB)) {
        int kind, s1, s2;
        TG::slots(t, &kind, &s1, &s2);
        add_target(kind == 0 ? ql.jt : ql.kt, nt, ql.tidx[prm[s1]], ql.tidx[prm[s2]], hold[r]);
        hold[r] = 0.0;
      }
    }
  };
  for (int c = (blockIdx.x * wpb + wid) * ql.numprocs + ql.myid; c < nchunks; c += stride) {
    const int4 ch = ql.chunks[c];
    const int p = ch.x;
    const int I = pr.si[p], J = pr.sj[p];
    for (int x = lane; x < NA; x += 32) prm[x] = ql.prim[I * MAXCOMP + x];
    for (int x = lane; x < NB; x += 32) prm[TG::SB + x] = ql.prim[J * MAXCOMP + x];
    __syncwarp();
    for (int t = lane; t < NA * NB; t += 32) Pab[t] = dens_at(D, npgs, prm[t / NB], prm[TG::SB + t % NB]);
    const double zb = pr.zeta[p], sp = pr.schwarz[p];
    const double Px = pr.P[0][p], Py = pr.P[1][p], Pz = pr.P[2][p];
#pragma unroll
    for (int r = 0; r < (HOLD ? NR : 1); ++r) hold[r] = 0.0;
    int run = -1;  // contracted block pair of the held sums
    for (int qq = ch.y; qq < ch.z; ++qq) {
      if (sp * pr.schwarz[qq] < ql.inttol) continue;   // the reference's screen (warp-uniform)
      const int K = pr.si[qq], L = pr.sj[qq];
      if (HOLD) {
        const int g = pr.gid[qq];
        if (g != run) {
          if (run >= 0) flush(false);
          run = g;
          __syncwarp();
        }
      }
      const double ze = pr.zeta[qq];
      const double Qx = pr.P[0][qq], Qy = pr.P[1][qq], Qz = pr.P[2][qq];
      const double zz = zb + ze, rho = zb * ze / zz;
      const double T = rho * ((Px - Qx) * (Px - Qx) + (Py - Qy) * (Py - Qy) + (Pz - Qz) * (Pz - Qz));
      const double pref = c2pi * pr.S[p] * pr.S[qq] * sqrt(rho);
      if (lane == 0) {
        double F[LT + 1];
        boys_tab<LT>(T, pref, ql.boys, F);
        v[0] = 0.0;
#pragma unroll
        for (int m = 0; m <= LT; ++m) v[1 + m] = F[m];
      } else if (lane == 1) {
        const double W[3] = {(zb * Px + ze * Qx) / zz, (zb * Py + ze * Qy) / zz, (zb * Pz + ze * Qz) / zz};
        const double Pv[3] = {Px, Py, Pz}, Qv[3] = {Qx, Qy, Qz};
        double PA[3], QC[3], AB[3], CD[3], WP[3], WQ[3];
        for (int k = 0; k < 3; ++k) {
          PA[k] = pr.PA[k][p]; QC[k] = pr.PA[k][qq]; AB[k] = pr.AB[k][p]; CD[k] = pr.AB[k][qq];
          WP[k] = W[k] - Pv[k]; WQ[k] = W[k] - Qv[k];
        }
        set_geom(geo, PA, WP, QC, WQ, AB, CD, 0.5 / zb, 0.5 / ze, 0.5 / zz, rho / zb, rho / ze);
      }
      for (int x = lane; x < NC; x += 32) prm[TG::SC + x] = ql.prim[K * MAXCOMP + x];
      for (int x = lane; x < ND; x += 32) prm[TG::SD + x] = ql.prim[L * MAXCOMP + x];
      __syncwarp();
      const int* pa = prm;
      const int* pb = prm + TG::SB;
      const int* pc = prm + TG::SC;
      const int* pd = prm + TG::SD;
      for (int t = lane; t < NC * ND; t += 32) Pcd[t] = dens_at(D, npgs, pc[t / ND], pd[t % ND]);
      for (int t = lane; t < NA * NC; t += 32) Pac[t] = dens_at(D, npgs, pa[t / NC], pc[t % NC]);
      for (int t = lane; t < NA * ND; t += 32) Pad[t] = dens_at(D, npgs, pa[t / ND], pd[t % ND]);
      for (int t = lane; t < NB * NC; t += 32) Pbc[t] = dens_at(D, npgs, pb[t / NC], pc[t % NC]);
      for (int t = lane; t < NB * ND; t += 32) Pbd[t] = dens_at(D, npgs, pb[t / ND], pd[t % ND]);
      for (int l = 0; l < tab.nlevels; ++l) {
        const int o0 = tab.levels[l], o1 = tab.levels[l + 1];
        for (int o = o0 + lane; o < o1; o += 32) {
          const unsigned short* op = tab.ops + 6 * o;
          const int h = op[0];
          const int kind = h >> 12, ax = (h >> 10) & 3, cA = (h >> 5) & 31, cB = h & 31;
          double val = geo.G1[kind][ax] * v[op[1]] + geo.G2[kind][ax] * v[op[2]];
          if (cA) val += (double)cA * geo.X[kind] * (v[op[3]] - geo.Y[kind] * v[op[4]]);
          if (cB) val += (double)cB * geo.Z * v[op[5]];
          v[base + o] = val;
        }
        __syncwarp();
      }
      const double deg = (I != J ? 2.0 : 1.0) * (K != L ? 2.0 : 1.0) * (p != qq ? 2.0 : 1.0);
      const double wj = 0.25 * deg, wk = 0.125 * deg;
#pragma unroll
      for (int r = 0; r < NR; ++r) {
        const int t = lane + 32 * r;
        if (t < NT) {
          int kind, s1, s2;
          TG::slots(t, &kind, &s1, &s2);
          const int p1 = prm[s1], p2 = prm[s2];
          const double w = (kind == 0 ? wj : wk) * ql.tcoef[p1] * ql.tcoef[p2] *
                           TG::value(t, v, tab.out, Pab, Pcd, Pac, Pad, Pbc, Pbd);
          if constexpr (HOLD) hold[r] += w;
          else add_target(kind == 0 ? ql.jt : ql.kt, nt, ql.tidx[p1], ql.tidx[p2], w);
        }
      }
      __syncwarp();
    }
    if (HOLD && run >= 0) flush(true);
    __syncwarp();
  }
}

// One quartet at a time per block (the largest classes).
template <int LA, int LB, int LC, int LD>
__global__ void __launch_bounds__(256) k_quartets_big(MolLaunch ql, OpTableDev tab) {
  constexpr int NA = ncum(LA), NB = ncum(LB), NC = ncum(LC), ND = ncum(LD);
  constexpr int LT = LA + LB + LC + LD;
  constexpr int NT = Targets<NA, NB, NC, ND>::NT;
  extern __shared__ double smem[];
  double* v = smem;
  double* Pab = smem + tab.nslots;
  double* Pcd = Pab + NA * NB;
  double* Pac = Pcd + NC * ND;
  double* Pad = Pac + NA * NC;
  double* Pbc = Pad + NA * ND;
  double* Pbd = Pbc + NB * NC;
  __shared__ OpGeom geo;
  __shared__ int prm[NA + NB + NC + ND];
  __shared__ double s_w[2];
  const PairArrays pr = ql.pairs;
  const int npgs = ql.npgs, nt = ql.nt;
  const double* __restrict__ D = ql.density;
  const int nchunks = *ql.nchunks;
  const double c2pi = 2.0 / sqrt(REF_PI);
  const int base = LT + 2;
  for (int c = blockIdx.x * ql.numprocs + ql.myid; c < nchunks; c += gridDim.x * ql.numprocs) {
    const int4 ch = ql.chunks[c];
    const int p = ch.x;
    const double sp = pr.schwarz[p];
    for (int qq = ch.y; qq < ch.z; ++qq) {
      if (sp * pr.schwarz[qq] < ql.inttol) continue;
      if (threadIdx.x == 0) {
        const double zb = pr.zeta[p], ze = pr.zeta[qq];
        const double Pv[3] = {pr.P[0][p], pr.P[1][p], pr.P[2][p]};
        const double Qv[3] = {pr.P[0][qq], pr.P[1][qq], pr.P[2][qq]};
        const double zz = zb + ze, rho = zb * ze / zz;
        const double T = rho * ((Pv[0] - Qv[0]) * (Pv[0] - Qv[0]) + (Pv[1] - Qv[1]) * (Pv[1] - Qv[1]) +
                                (Pv[2] - Qv[2]) * (Pv[2] - Qv[2]));
        const double pref = c2pi * pr.S[p] * pr.S[qq] * sqrt(rho);
        double F[LT + 1];
        boys_tab<LT>(T, pref, ql.boys, F);
        v[0] = 0.0;
        for (int m = 0; m <= LT; ++m) v[1 + m] = F[m];
        double PA[3], QC[3], AB[3], CD[3], WP[3], WQ[3];
        for (int k = 0; k < 3; ++k) {
          const double W = (zb * Pv[k] + ze * Qv[k]) / zz;
          PA[k] = pr.PA[k][p]; QC[k] = pr.PA[k][qq]; AB[k] = pr.AB[k][p]; CD[k] = pr.AB[k][qq];
          WP[k] = W - Pv[k]; WQ[k] = W - Qv[k];
        }
        set_geom(geo, PA, WP, QC, WQ, AB, CD, 0.5 / zb, 0.5 / ze, 0.5 / zz, rho / zb, rho / ze);
        const int I = pr.si[p], J = pr.sj[p], K = pr.si[qq], L = pr.sj[qq];
        const double deg = (I != J ? 2.0 : 1.0) * (K != L ? 2.0 : 1.0) * (p != qq ? 2.0 : 1.0);
        s_w[0] = 0.25 * deg;
        s_w[1] = 0.125 * deg;
        for (int x = 0; x < NA; ++x) prm[x] = ql.prim[I * MAXCOMP + x];
        for (int x = 0; x < NB; ++x) prm[NA + x] = ql.prim[J * MAXCOMP + x];
        for (int x = 0; x < NC; ++x) prm[NA + NB + x] = ql.prim[K * MAXCOMP + x];
        for (int x = 0; x < ND; ++x) prm[NA + NB + NC + x] = ql.prim[L * MAXCOMP + x];
      }
      __syncthreads();
      const int* pa = prm;
      const int* pb = prm + NA;
      const int* pc = prm + NA + NB;
      const int* pd = prm + NA + NB + NC;
      for (int t = threadIdx.x; t < NA * NB; t += blockDim.x) Pab[t] = dens_at(D, npgs, pa[t / NB], pb[t % NB]);
      for (int t = threadIdx.x; t < NC * ND; t += blockDim.x) Pcd[t] = dens_at(D, npgs, pc[t / ND], pd[t % ND]);
      for (int t = threadIdx.x; t < NA * NC; t += blockDim.x) Pac[t] = dens_at(D, npgs, pa[t / NC], pc[t % NC]);
      for (int t = threadIdx.x; t < NA * ND; t += blockDim.x) Pad[t] = dens_at(D, npgs, pa[t / ND], pd[t % ND]);
      for (int t = threadIdx.x; t < NB * NC; t += blockDim.x) Pbc[t] = dens_at(D, npgs, pb[t / NC], pc[t % NC]);
      for (int t = threadIdx.x; t < NB * ND; t += blockDim.x) Pbd[t] = dens_at(D, npgs, pb[t / ND], pd[t % ND]);
      run_optable(tab, v, geo, base);
      for (int t = threadIdx.x; t < NT; t += blockDim.x) {
        int kind, r1, r2;
        Targets<NA, NB, NC, ND>::slots(t, &kind, &r1, &r2);
        const double val = Targets<NA, NB, NC, ND>::value(t, v, tab.out, Pab, Pcd, Pac, Pad, Pbc, Pbd);
        const int p1 = prm[r1], p2 = prm[r2];
        add_target(kind == 0 ? ql.jt : ql.kt, nt, ql.tidx[p1], ql.tidx[p2],
                   (kind == 0 ? s_w[0] : s_w[1]) * val * ql.tcoef[p1] * ql.tcoef[p2]);
      }
      __syncthreads();
    }
  }
}

// ------------------------------------------------------------------ launch tables

using LaunchFn = void (*)(const MolLaunch&, int grid, cudaStream_t);

template <int LA, int LB, int LC, int LD>
static void launch_q(const MolLaunch& ql, int grid, cudaStream_t s) {
  k_quartets<LA, LB, LC, LD><<<grid, 128, 0, s>>>(ql);
}

static LaunchFn straight_launcher(int cb, int ck) {
#define Q(A, B, C, D) &launch_q<A, B, C, D>
  static const LaunchFn table[6][6] = {
      {Q(0, 0, 0, 0), nullptr, nullptr, nullptr, nullptr, nullptr},
      {Q(1, 0, 0, 0), Q(1, 0, 1, 0), nullptr, nullptr, nullptr, nullptr},
      {Q(1, 1, 0, 0), Q(1, 1, 1, 0), Q(1, 1, 1, 1), nullptr, nullptr, nullptr},
      {Q(2, 0, 0, 0), Q(2, 0, 1, 0), Q(2, 0, 1, 1), Q(2, 0, 2, 0), nullptr, nullptr},
      {Q(2, 1, 0, 0), Q(2, 1, 1, 0), nullptr, nullptr, nullptr, nullptr},
      {Q(2, 2, 0, 0), nullptr, nullptr, nullptr, nullptr, nullptr}};
#undef Q
  return table[cb][ck];
}

using BigFn = void (*)(const MolLaunch&, const OpTableDev&, int grid, size_t smem, cudaStream_t);
using WarpFn = void (*)(const MolLaunch&, const OpTableDev&, int grid, int wpb, int per_warp, size_t smem, cudaStream_t);

template <int LA, int LB, int LC, int LD>
static void launch_big(const MolLaunch& ql, const OpTableDev& t, int grid, size_t smem, cudaStream_t s) {
  k_quartets_big<LA, LB, LC, LD><<<grid, 256, smem, s>>>(ql, t);
}

template <int LA, int LB, int LC, int LD>
static void launch_warp(const MolLaunch& ql, const OpTableDev& t, int grid, int wpb, int per_warp, size_t smem,
                        cudaStream_t s) {
  k_quartets_warp<LA, LB, LC, LD><<<grid, 32 * wpb, smem, s>>>(ql, t, per_warp);
}

template <int LA, int LB, int LC, int LD>
static cudaError_t allow_smem_both(size_t big, size_t warp) {
  cudaError_t e = cudaFuncSetAttribute(k_quartets_big<LA, LB, LC, LD>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)big);
  if (e != cudaSuccess) return e;
  return cudaFuncSetAttribute(k_quartets_warp<LA, LB, LC, LD>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)warp);
}

struct Variants {
  BigFn big;
  WarpFn warp;
  cudaError_t (*allow)(size_t, size_t);
};

static Variants variants(int cb, int ck) {
#define V(A, B, C, D) Variants{&launch_big<A, B, C, D>, &launch_warp<A, B, C, D>, &allow_smem_both<A, B, C, D>}
  switch (cb * 8 + ck) {
    case 0: return V(0, 0, 0, 0);
    case 8: return V(1, 0, 0, 0);
    case 9: return V(1, 0, 1, 0);
    case 16: return V(1, 1, 0, 0);
    case 17: return V(1, 1, 1, 0);
    case 18: return V(1, 1, 1, 1);
    case 24: return V(2, 0, 0, 0);
    case 25: return V(2, 0, 1, 0);
    case 26: return V(2, 0, 1, 1);
    case 27: return V(2, 0, 2, 0);
    case 32: return V(2, 1, 0, 0);
    case 33: return V(2, 1, 1, 0);
    case 34: return V(2, 1, 1, 1);
    case 35: return V(2, 1, 2, 0);
    case 36: return V(2, 1, 2, 1);
    case 40: return V(2, 2, 0, 0);
    case 41: return V(2, 2, 1, 0);
    case 42: return V(2, 2, 1, 1);
    case 43: return V(2, 2, 2, 0);
    case 44: return V(2, 2, 2, 1);
    case 45: return V(2, 2, 2, 2);
    default: return Variants{nullptr, nullptr, nullptr};
  }
#undef V
}

static int density_block_doubles(int cb, int ck) {
  const int NA = ncum(kCL[cb][0]), NB = ncum(kCL[cb][1]), NC = ncum(kCL[ck][0]), ND = ncum(kCL[ck][1]);
  return NA * NB + NC * ND + NA * NC + NA * ND + NB * NC + NB * ND;
}

// ------------------------------------------------------------------ set-up

int molecular_setup(pfe_context* ctx, const pfe_args* a) {
  (void)a;
  cudaStream_t s = ctx->stream;
  const int nsh = ctx->npshell;
  const long long npairs = (long long)nsh * (nsh + 1) / 2;
  ctx->npairs = npairs;
  PairArrays raw{};
  int rc;
  if ((rc = alloc_pairs(ctx, &raw, npairs)) != PFE_OK) return rc;
  if ((rc = alloc_pairs(ctx, &ctx->pairs, npairs)) != PFE_OK) return rc;
  int* d_count = nullptr;
  PFE_CUDA(ctx->alloc((void**)&d_count, sizeof(int) * 8));
  PFE_CUDA(cudaMemsetAsync(d_count, 0, sizeof(int) * 8, s));
  const unsigned nb256 = (unsigned)((npairs + 255) / 256);
  k_mol_pairs<<<(unsigned)((npairs + 127) / 128), 128, 0, s>>>(ctx->shells, ctx->d_blk, ctx->nblk, ctx->d_sss,
                                                                ctx->d_boys, ctx->d_maxc, raw, d_count, npairs);
  PFE_CUDA(cudaGetLastError());
  // bounds of the (21) and (22) pair classes on the interpreter
  {
    int *list = nullptr, *cnt = nullptr;
    PFE_CUDA(ctx->alloc((void**)&list, sizeof(int) * npairs));
    PFE_CUDA(ctx->alloc((void**)&cnt, sizeof(int)));
    for (int cls = 4; cls <= 5; ++cls) {
      PFE_CUDA(cudaMemsetAsync(cnt, 0, sizeof(int), s));
      launch_select_class(raw.cls, cls, list, cnt, npairs, s);
      int hn = 0;
      PFE_CUDA(cudaMemcpyAsync(&hn, cnt, sizeof(int), cudaMemcpyDeviceToHost, s));
      PFE_CUDA(cudaStreamSynchronize(s));
      if (hn == 0) continue;
      const OpTableHost* h = host_optable(cls, cls);
      OpTableDev d{};
      if ((rc = upload_optable(ctx, h, &d)) != PFE_OK) return rc;
      const size_t smem = sizeof(double) * (size_t)h->nslots;
      if (cls == 4) {
        PFE_CUDA(cudaFuncSetAttribute(k_schwarz_big<2, 1>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        k_schwarz_big<2, 1><<<std::min(hn, 4 * ctx->num_sms), 256, smem, s>>>(raw, ctx->shells.prim, ctx->d_maxc, list, hn, d);
      } else {
        PFE_CUDA(cudaFuncSetAttribute(k_schwarz_big<2, 2>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        k_schwarz_big<2, 2><<<std::min(hn, 4 * ctx->num_sms), 256, smem, s>>>(raw, ctx->shells.prim, ctx->d_maxc, list, hn, d);
      }
      PFE_CUDA(cudaGetLastError());
      PFE_CUDA(cudaStreamSynchronize(s));
    }
    ctx->free_now(list);
    ctx->free_now(cnt);
  }
  // group maxima and the four sort keys
  const long long ngroups = (long long)ctx->nblk * ctx->nblk;
  unsigned long long *gbits = nullptr, *k_sch = nullptr, *k_gmax = nullptr, *k64 = nullptr;
  int *perm_a = nullptr, *perm_b = nullptr, *k32 = nullptr, *k32b = nullptr;
  unsigned char *k8 = nullptr, *k8b = nullptr;
  PFE_CUDA(ctx->alloc((void**)&gbits, sizeof(unsigned long long) * ngroups));
  PFE_CUDA(ctx->alloc((void**)&k_sch, sizeof(unsigned long long) * npairs));
  PFE_CUDA(ctx->alloc((void**)&k_gmax, sizeof(unsigned long long) * npairs));
  PFE_CUDA(ctx->alloc((void**)&k64, sizeof(unsigned long long) * npairs));
  PFE_CUDA(ctx->alloc((void**)&perm_a, sizeof(int) * npairs));
  PFE_CUDA(ctx->alloc((void**)&perm_b, sizeof(int) * npairs));
  PFE_CUDA(ctx->alloc((void**)&k32, sizeof(int) * npairs));
  PFE_CUDA(ctx->alloc((void**)&k32b, sizeof(int) * npairs));
  PFE_CUDA(ctx->alloc((void**)&k8, npairs));
  PFE_CUDA(ctx->alloc((void**)&k8b, npairs));
  PFE_CUDA(cudaMemsetAsync(gbits, 0, sizeof(unsigned long long) * ngroups, s));
  k_mol_groupmax<<<nb256, 256, 0, s>>>(raw.schwarz, raw.gid, gbits, npairs);
  k_mol_keys<<<nb256, 256, 0, s>>>(raw.schwarz, raw.gid, gbits, k_sch, k_gmax, raw.gmax, npairs);
  k_mol_iota<<<nb256, 256, 0, s>>>(perm_a, npairs);
  PFE_CUDA(cudaGetLastError());
  {
    const int n = (int)npairs;
    size_t t1 = 0, t2 = 0, t3 = 0;
    cub::DeviceRadixSort::SortPairs(nullptr, t1, k_sch, k64, perm_a, perm_b, n, 0, 64, s);
    cub::DeviceRadixSort::SortPairs(nullptr, t2, k32, k32b, perm_b, perm_a, n, 0, 32, s);
    cub::DeviceRadixSort::SortPairs(nullptr, t3, k8, k8b, perm_a, perm_b, n, 0, 8, s);
    const size_t tb = std::max(t1, std::max(t2, t3)) + 16;
    void* tmp = nullptr;
    PFE_CUDA(ctx->alloc(&tmp, tb));
    size_t tt = tb;
    // 1: bound descending
    PFE_CUDA(cub::DeviceRadixSort::SortPairs(tmp, tt, k_sch, k64, perm_a, perm_b, n, 0, 64, s));
    // 2: group (stable)
    k_gather_t<int><<<nb256, 256, 0, s>>>(raw.gid, perm_b, k32, npairs);
    tt = tb;
    PFE_CUDA(cub::DeviceRadixSort::SortPairs(tmp, tt, k32, k32b, perm_b, perm_a, n, 0, 32, s));
    // 3: group maximum descending (stable)
    k_gather_t<unsigned long long><<<nb256, 256, 0, s>>>(k_gmax, perm_a, k_sch, npairs);
    tt = tb;
    PFE_CUDA(cub::DeviceRadixSort::SortPairs(tmp, tt, k_sch, k64, perm_a, perm_b, n, 0, 64, s));
    // 4: class (stable)
    k_gather_t<unsigned char><<<nb256, 256, 0, s>>>(raw.cls, perm_b, k8, npairs);
    tt = tb;
    PFE_CUDA(cub::DeviceRadixSort::SortPairs(tmp, tt, k8, k8b, perm_b, perm_a, n, 0, 8, s));
    k_mol_gather<<<(unsigned)((npairs + 127) / 128), 128, 0, s>>>(raw, ctx->pairs, perm_a, npairs);
    PFE_CUDA(cudaGetLastError());
    PFE_CUDA(cudaStreamSynchronize(s));
    ctx->free_now(tmp);
  }
  for (void* p : {(void*)gbits, (void*)k_sch, (void*)k_gmax, (void*)k64, (void*)perm_a, (void*)perm_b, (void*)k32,
                  (void*)k32b, (void*)k8, (void*)k8b})
    ctx->free_now(p);
  int hcount[8] = {0};
  PFE_CUDA(cudaMemcpy(hcount, d_count, sizeof(int) * 8, cudaMemcpyDeviceToHost));
  ctx->free_now(d_count);
  free_pairs(ctx, &raw);
  int off = 0;
  for (int c = 0; c < 6; ++c) {
    ctx->class_off[c] = off;
    ctx->class_n[c] = hcount[c];
    off += hcount[c];
  }
  // chunk lists for every class pair cb >= ck
  ctx->nlaunch = 0;
  ctx->census_quartets = ctx->census_flops = ctx->census_ref = 0.0;
  const int maxn = *std::max_element(ctx->class_n, ctx->class_n + 6);
  int *nrange = nullptr, *nchunk = nullptr, *offs = nullptr, *nquart = nullptr;
  long long* d_sum = nullptr;
  PFE_CUDA(ctx->alloc((void**)&nrange, sizeof(int) * (maxn + 1)));
  PFE_CUDA(ctx->alloc((void**)&nchunk, sizeof(int) * (maxn + 1)));
  PFE_CUDA(ctx->alloc((void**)&offs, sizeof(int) * (maxn + 1)));
  PFE_CUDA(ctx->alloc((void**)&nquart, sizeof(int) * (maxn + 1)));
  PFE_CUDA(ctx->alloc((void**)&d_sum, sizeof(long long)));
  for (int cb = 0; cb < 6; ++cb)
    for (int ck = 0; ck <= cb; ++ck) {
      const int nb = ctx->class_n[cb], nk = ctx->class_n[ck];
      if (nb == 0 || nk == 0) continue;
      const int b0 = ctx->class_off[cb], k0 = ctx->class_off[ck];
      k_mol_count<<<(nb + 127) / 128, 128, 0, s>>>(ctx->pairs.schwarz, ctx->pairs.gmax, b0, nb, k0, nk, cb == ck,
                                                   ctx->inttol, nrange, nchunk, nquart);
      PFE_CUDA(cudaGetLastError());
      PFE_CUDA(cudaMemsetAsync(nchunk + nb, 0, sizeof(int), s));
      size_t sb = 0;
      cub::DeviceScan::ExclusiveSum(nullptr, sb, nchunk, offs, nb + 1, s);
      void* st = nullptr;
      PFE_CUDA(ctx->alloc(&st, sb + 16));
      PFE_CUDA(cub::DeviceScan::ExclusiveSum(st, sb, nchunk, offs, nb + 1, s));
      size_t rb = 0;
      cub::DeviceReduce::Sum(nullptr, rb, nquart, d_sum, nb, s);
      void* rt = nullptr;
      PFE_CUDA(ctx->alloc(&rt, rb + 16));
      PFE_CUDA(cub::DeviceReduce::Sum(rt, rb, nquart, d_sum, nb, s));
      int total = 0;
      long long nq = 0;
      PFE_CUDA(cudaMemcpyAsync(&total, offs + nb, sizeof(int), cudaMemcpyDeviceToHost, s));
      PFE_CUDA(cudaMemcpyAsync(&nq, d_sum, sizeof(long long), cudaMemcpyDeviceToHost, s));
      PFE_CUDA(cudaStreamSynchronize(s));
      ctx->free_now(st);
      ctx->free_now(rt);
      if (total == 0) continue;
      ClassLaunch cl{};
      cl.cb = cb;
      cl.ck = ck;
      cl.nchunks_host = total;
      cl.quartets = (double)nq;
      PFE_CUDA(ctx->alloc((void**)&cl.chunks, sizeof(int4) * total));
      PFE_CUDA(ctx->alloc((void**)&cl.d_nchunks, sizeof(int)));
      PFE_CUDA(cudaMemcpyAsync(cl.d_nchunks, &cl.nchunks_host, sizeof(int), cudaMemcpyHostToDevice, s));
      k_mol_fill<<<(nb + 127) / 128, 128, 0, s>>>(nrange, offs, b0, k0, nb, cl.chunks);
      PFE_CUDA(cudaGetLastError());
      PFE_CUDA(cudaStreamSynchronize(s));
      cl.has_straight = straight_launcher(cb, ck) != nullptr;
      cl.has_table = false;
      cl.variant = 0;
      if (const OpTableHost* h = host_optable(cb, ck)) {
        OpTableDev d{};
        if ((rc = upload_optable(ctx, h, &d)) != PFE_OK) return rc;
        cl.has_table = true;
        cl.ops = d.ops; cl.levels = d.levels; cl.out = d.out;
        cl.nlevels = d.nlevels; cl.nout = d.nout; cl.nslots = d.nslots;
        cl.smem_big = sizeof(double) * ((size_t)h->nslots + density_block_doubles(cb, ck));
        cl.per_warp = h->nslots + density_block_doubles(cb, ck);
        cl.wpb = (int)std::max<size_t>(1, std::min<size_t>(8, (200 * 1024) / (sizeof(double) * cl.per_warp)));
        cl.smem_warp = sizeof(double) * (size_t)cl.per_warp * cl.wpb;
        PFE_CUDA(variants(cb, ck).allow(cl.smem_big, cl.smem_warp));
        cl.variant = (cl.has_straight && h->nout <= 100) ? 0 : (sizeof(double) * cl.per_warp <= 100 * 1024 ? 1 : 2);
      }
      for (int v = 0; v < 3; ++v) cl.tuned_ms[v] = 0.f;
      ctx->launches[ctx->nlaunch++] = cl;
      ctx->census_quartets += (double)nq;
      ctx->census_flops += (double)nq * class_flops(cb, ck);
    }
  for (void* p : {(void*)nrange, (void*)nchunk, (void*)offs, (void*)nquart, (void*)d_sum}) ctx->free_now(p);
  // the reference's loop visits both orders of every pair and of bra/ket: 8x the unique quartets
  ctx->census_ref = 0.0;
  ctx->free_pending();
  return PFE_OK;
}

// ------------------------------------------------------------------ build

static MolLaunch make_launch(pfe_context* ctx, const double* d_pp) {
  MolLaunch ql{};
  ql.pairs = ctx->pairs;
  ql.prim = ctx->shells.prim;
  ql.tidx = ctx->d_tidx;
  ql.tcoef = ctx->d_tcoef;
  ql.boys = ctx->d_boys;
  ql.density = d_pp;
  ql.jt = ctx->d_jp;
  ql.kt = ctx->d_kp;
  ql.inttol = ctx->inttol;
  ql.npgs = ctx->npgs;
  ql.nt = ctx->nt;
  ql.myid = ctx->myid;
  ql.numprocs = ctx->numprocs;
  return ql;
}

static void launch_class(pfe_context* ctx, const ClassLaunch& cl, MolLaunch ql, int variant, cudaStream_t s) {
  ql.chunks = cl.chunks;
  ql.nchunks = cl.d_nchunks;
  const int work = (cl.nchunks_host + ctx->numprocs - 1) / ctx->numprocs;
  if (variant == 0 || !cl.has_table) {
    const int grid = std::min((work + 3) / 4, ctx->num_sms * 16);
    straight_launcher(cl.cb, cl.ck)(ql, std::max(grid, 1), s);
    return;
  }
  OpTableDev t{cl.ops, cl.levels, cl.out, cl.nlevels, cl.nout, cl.nslots};
  if (variant == 1) {
    const int grid = std::min((work + cl.wpb - 1) / cl.wpb, ctx->num_sms * 8);
    variants(cl.cb, cl.ck).warp(ql, t, std::max(grid, 1), cl.wpb, cl.per_warp, cl.smem_warp, s);
  } else {
    const int grid = std::min(work, ctx->num_sms * 2);
    variants(cl.cb, cl.ck).big(ql, t, std::max(grid, 1), cl.smem_big, s);
  }
}

static size_t target_bytes(const pfe_context* ctx) { return sizeof(double) * (size_t)ctx->nt * ctx->nt; }

int autotune(pfe_context* ctx, const double* d_pp, cudaStream_t s) {
  const MolLaunch ql = make_launch(ctx, d_pp);
  cudaEvent_t e0, e1;
  PFE_CUDA(cudaEventCreate(&e0));
  PFE_CUDA(cudaEventCreate(&e1));
  for (int i = 0; i < ctx->nlaunch; ++i) {
    ClassLaunch& cl = ctx->launches[i];
    float best = 1e30f;
    int bestv = cl.variant;
    for (int v = 0; v < 3; ++v) {
      if ((v == 0 && !cl.has_straight) || (v > 0 && !cl.has_table)) continue;
      if (v == 1 && sizeof(double) * (size_t)cl.per_warp > 200 * 1024) continue;
      launch_class(ctx, cl, ql, v, s);
      float t = 1e30f;
      for (int r = 0; r < 2; ++r) {
        PFE_CUDA(cudaEventRecord(e0, s));
        launch_class(ctx, cl, ql, v, s);
        PFE_CUDA(cudaEventRecord(e1, s));
        PFE_CUDA(cudaEventSynchronize(e1));
        float ms = 0.f;
        PFE_CUDA(cudaEventElapsedTime(&ms, e0, e1));
        t = std::min(t, ms);
      }
      PFE_CUDA(cudaGetLastError());
      cl.tuned_ms[v] = t;
      if (t < best) { best = t; bestv = v; }
    }
    cl.variant = bestv;
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  PFE_CUDA(cudaMemsetAsync(ctx->d_jp, 0, target_bytes(ctx), s));
  PFE_CUDA(cudaMemsetAsync(ctx->d_kp, 0, target_bytes(ctx), s));
  PFE_CUDA(cudaStreamSynchronize(s));
  ctx->tuned = true;
  return PFE_OK;
}

int molecular_fock(pfe_context* ctx, const double* d_pp, double* d_cc, double* d_xc, cudaStream_t s) {
  PFE_CUDA(cudaMemsetAsync(ctx->d_jp, 0, target_bytes(ctx), s));
  PFE_CUDA(cudaMemsetAsync(ctx->d_kp, 0, target_bytes(ctx), s));
  const MolLaunch ql = make_launch(ctx, d_pp);
  if (ctx->profile) {
    for (int i = 0; i <= ctx->nlaunch && i < 64; ++i)
      if (!ctx->ev[i]) PFE_CUDA(cudaEventCreate(&ctx->ev[i]));
    ctx->nprof = ctx->nlaunch;
    PFE_CUDA(cudaEventRecord(ctx->ev[0], s));
  }
  for (int i = 0; i < ctx->nlaunch; ++i) {
    const ClassLaunch& cl = ctx->launches[i];
    launch_class(ctx, cl, ql, cl.variant, s);
    PFE_CUDA(cudaGetLastError());
    if (ctx->profile) {
      PFE_CUDA(cudaEventRecord(ctx->ev[i + 1], s));
      ctx->ev_cls[i] = 1000 * kCL[cl.cb][0] + 100 * kCL[cl.cb][1] + 10 * kCL[cl.ck][0] + kCL[cl.ck][1];
      ctx->ev_quartets[i] = cl.quartets;
      ctx->ev_flops[i] = cl.quartets * class_flops(cl.cb, cl.ck);
      ctx->ev_variant[i] = cl.variant;
      for (int v = 0; v < 3; ++v) ctx->ev_tuned[i][v] = cl.tuned_ms[v];
    }
  }
  if (ctx->contracted) {
    launch_symmetrize(ctx->d_jp, d_cc, ctx->ncgs, 1, s);
    launch_symmetrize(ctx->d_kp, d_xc, ctx->ncgs, 1, s);
    PFE_CUDA(cudaGetLastError());
    return PFE_OK;
  }
  return contract_outputs(ctx, ctx->d_jp, ctx->d_kp, d_cc, d_xc, /*symmetrize=*/true, 1, s);
}

}  // namespace pfe
