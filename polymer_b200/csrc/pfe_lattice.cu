// General path of the Fock build: lattices (CEL1/CEL2 > 0) and helices.
//
// Follows the reference's loop semantics (src/pfourindexdirect.f90:224-760)
// without permutational symmetry: for every (Q1,Q2) cell-pair ticket owned by
// this rank (the TICKET round robin, :224-240), every bra pair (I@0, J@Q1),
// every Q3 in the CEL2 box and every ket pair (K@Q3, L@Q3+Q2) -- the screw
// image of (K@0, L@Q2) -- that passes IJIJ*KLKL >= INTTOL (:529):
//   C_P(i,j,Q1)    += D(k,l) (ij|kl),  D = P_P(:,:,Q2)   or P_P_HELIX(:,:,Q3,Q3+Q2)
//   X_P(i,l,Q3+Q2) += D(k,j) (ij|kl),  D = P_P(:,:,Q1-Q3) or P_P_HELIX(:,:,Q3,Q1)
// the second only where Q3+Q2 and Q1-Q3 lie inside CUTOFF1 (LCEL1, :248-259);
// then C_C = CC C_P CC^T per cell (:765-782) and, with HELIX, C_C <- C_C C2H^T
// along the screw axis (:784-803).
//
// KLKL is the bound of the ket's own geometry (K@0, L@Q2).  IJIJ reproduces
// the reference's reuse of the ket scratch QI_CI (:436-447): it is evaluated
// with the exponents and S_P(I,J,Q1) of the bra but with the component
// geometry of (I@0, J@Q2) for the first bra pair of a ticket and of the last Q3
// image (I@Q3max, J@Q3max+Q2) for all others -- exact for molecules, and the
// reason the bound depends on the ticket.
//
// Device layout: one list of ordered shell pairs (I@0, J@q) per cell q of the
// REDUCED_CEL1 box, canonically oriented (higher L first, orientation flag
// kept) and sorted by (cell, class, bound descending); chunks of up to 32 kets
// per (ticket, bra pair); one quartet per warp on the generated op tables.

#include <cublas_v2.h>
#include <cub/cub.cuh>

#include <algorithm>
#include <vector>

#include "pfe_common.cuh"
#include "pfe_context.cuh"
#include "pfe_interp.cuh"
#include "pfe_lattice.cuh"

namespace pfe {

struct LatticeLaunch {
  int cb, ck;            // bra class, ket class (canonical pair classes)
  int ncells_chunks;
  int* d_nchunks;
  int4* chunks;          // (bra pair, first ket, end ket, ticket)
  OpTableDev tab;        // of the evaluated class (max(cb,ck) | min(cb,ck))
  int per_warp, wpb;
  size_t smem;
  double quartets;
};

struct LatticeState {
  int nq = 0;                  // cells of the REDUCED_CEL1 box
  std::vector<int> qcell;      // 3 ints per list cell
  int npl = 0;                 // pairs per list (npshell^2)
  int cls_off[6] = {0}, cls_n[6] = {0};   // per list, identical for every cell
  PairArrays pairs{};          // nq * npl, sorted by (cell, class, bound desc)
  unsigned char* swp = nullptr;  // orientation flag: 1 when the first centre is J
  int ntk = 0;                 // owned tickets
  int4* d_tickets = nullptr;   // (Q1 list, Q2 list, 0, 0)
  std::vector<int4> h_tickets;
  int* d_qcell = nullptr;      // 3 ints per list cell
  double* d_quirk = nullptr;   // ntk * npl bra bounds (sorted order of the Q1 list)
  LatticeLaunch launches[36];
  int nlaunch = 0;
  int* d_queue = nullptr;      // kLatQueueSlots chunk counters per launch (straight-line kernels, per pass)
  bool interpret_only = false; // every class on the op-table interpreter (tests)
  double quartets = 0.0, flops = 0.0;
};

// ---------------------------------------------------------------- set-up kernels

__device__ __forceinline__ void screw(const LatGeom& g, double x, double y, double z, int qx, int qy, int qz,
                                      double* o) {
  const double a = qx * g.helix;
  const double c = cos(a), s = sin(a);
  o[0] = x + qx * g.period[0];
  o[1] = y * c - z * s + qy * g.period[1];
  o[2] = y * s + z * c + qz * g.period[2];
}

// Fill pair record t for shells (I at cell A, J at cell B) with overlap S.
__device__ void fill_pair(const DevShells& sh, const LatGeom& g, int I, int J, const int qa[3], const int qb[3],
                          double S, PairArrays out, long long t, unsigned char* swp) {
  double A[3], B[3];
  screw(g, sh.x[I], sh.y[I], sh.z[I], qa[0], qa[1], qa[2], A);
  screw(g, sh.x[J], sh.y[J], sh.z[J], qb[0], qb[1], qb[2], B);
  int f = I, sc = J;
  const double *F = A, *Sc = B;
  unsigned char sw = 0;
  if (sh.L[J] > sh.L[I]) { f = J; sc = I; F = B; Sc = A; sw = 1; }
  const double zf = sh.zeta[f], zs = sh.zeta[sc], z = zf + zs;
  for (int k = 0; k < 3; ++k) {
    const double p = (F[k] * zf + Sc[k] * zs) / z;
    out.P[k][t] = p;
    out.PA[k][t] = p - F[k];
    out.AB[k][t] = F[k] - Sc[k];
  }
  out.zeta[t] = z;
  out.S[t] = S;
  out.si[t] = f;
  out.sj[t] = sc;
  out.cls[t] = (unsigned char)pair_class(sh.L[f], sh.L[sc]);
  if (swp) swp[t] = sw;
}

// Ordered pairs (I@0, J@q) of every list cell q.
__global__ void k_lat_pairs(DevShells sh, LatGeom g, const int* __restrict__ qcell, int nq, const double* __restrict__ sss,
                            PairArrays out, unsigned char* swp) {
  const int n = sh.n;
  const long long npl = (long long)n * n;
  const long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (t >= npl * nq) return;
  const int qi = (int)(t / npl);
  const int r = (int)(t % npl);
  const int I = r % n, J = r / n;
  const int q[3] = {qcell[3 * qi], qcell[3 * qi + 1], qcell[3 * qi + 2]};
  const int z0[3] = {0, 0, 0};
  const double S = sss[(size_t)I + (size_t)n * J + (size_t)n * n * cell1_index(g, q[0], q[1], q[2])];
  fill_pair(sh, g, I, J, z0, q, S, out, t, swp);
  out.schwarz[t] = 0.0;
}

// Schwarz bound of every record (thread per record) for pair classes 0..3.
__global__ void k_schwarz_small(PairArrays pr, const int* __restrict__ prim, const double* __restrict__ maxc,
                                const double* __restrict__ tab, long long n) {
  const long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (t >= n) return;
  const double PA[3] = {pr.PA[0][t], pr.PA[1][t], pr.PA[2][t]};
  const double AB[3] = {pr.AB[0][t], pr.AB[1][t], pr.AB[2][t]};
  const int* pa = prim + (size_t)pr.si[t] * MAXCOMP;
  const int* pb = prim + (size_t)pr.sj[t] * MAXCOMP;
  double b = 0.0;
  switch (pr.cls[t]) {
    case 0: b = schwarz_pair<0, 0>(tab, pr.zeta[t], pr.S[t], PA, AB, pa, pb, maxc); break;
    case 1: b = schwarz_pair<1, 0>(tab, pr.zeta[t], pr.S[t], PA, AB, pa, pb, maxc); break;
    case 2: b = schwarz_pair<1, 1>(tab, pr.zeta[t], pr.S[t], PA, AB, pa, pb, maxc); break;
    case 3: b = schwarz_pair<2, 0>(tab, pr.zeta[t], pr.S[t], PA, AB, pa, pb, maxc); break;
    default: return;  // classes 4, 5 on the interpreter
  }
  pr.schwarz[t] = b;
  pr.key[t] = ~(unsigned long long)__double_as_longlong(b);
}

__global__ void k_lat_keys(PairArrays pr, long long n) {
  const long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (t < n) pr.key[t] = ~(unsigned long long)__double_as_longlong(pr.schwarz[t]);
}

__global__ void k_select_cls(const unsigned char* __restrict__ cls, int want, int* __restrict__ list,
                             int* __restrict__ count, long long n) {
  const long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (t < n && cls[t] == want) list[atomicAdd(count, 1)] = (int)t;
}

// Stale-geometry bra records of every owned ticket, one per (ticket, bra) in
// the sorted order of the Q1 list; the bound is written to quirk[].
__global__ void k_lat_quirk_jobs(DevShells sh, LatGeom g, const int4* __restrict__ tickets, int ntk,
                                 const int* __restrict__ qcell, PairArrays lists, int npl,
                                 const unsigned char* __restrict__ swp, const double* __restrict__ sss,
                                 PairArrays jobs) {
  const long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (t >= (long long)ntk * npl) return;
  const int tk = (int)(t / npl), p = (int)(t % npl);
  const int4 tt = tickets[tk];
  const long long gp = (long long)tt.x * npl + p;           // bra record in the Q1 list
  const int f = lists.si[gp], sc = lists.sj[gp];
  const int I = swp[gp] ? sc : f, J = swp[gp] ? f : sc;     // reference order
  const int q2[3] = {qcell[3 * tt.y], qcell[3 * tt.y + 1], qcell[3 * tt.y + 2]};
  const int q1[3] = {qcell[3 * tt.x], qcell[3 * tt.x + 1], qcell[3 * tt.x + 2]};
  int qa[3] = {0, 0, 0}, qb[3] = {q2[0], q2[1], q2[2]};
  if (!(I == 0 && J == 0)) {
    for (int k = 0; k < 3; ++k) {
      qa[k] = g.c2[k];
      qb[k] = g.c2[k] + q2[k];
    }
  }
  const int n = sh.n;
  const double S = sss[(size_t)I + (size_t)n * J + (size_t)n * n * cell1_index(g, q1[0], q1[1], q1[2])];
  fill_pair(sh, g, I, J, qa, qb, S, jobs, t, nullptr);
  jobs.schwarz[t] = 0.0;
}

__global__ void k_lat_count(const double* __restrict__ quirk, const double* __restrict__ ksch, int npl, int b0, int nb,
                            int k0, int nk, int ntk, const int4* __restrict__ tickets, double inttol,
                            int* __restrict__ nvalid, int* __restrict__ nchunk) {
  const long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (t >= (long long)ntk * nb) return;
  const int tk = (int)(t / nb), p = (int)(t % nb);
  const double b = quirk[(long long)tk * npl + b0 + p];
  const double* ks = ksch + (long long)tickets[tk].y * npl + k0;
  int lo = 0, hi = nk;
  while (lo < hi) {
    const int mid = (lo + hi) >> 1;
    if (b * ks[mid] < inttol) hi = mid; else lo = mid + 1;
  }
  nvalid[t] = lo;
  nchunk[t] = (lo + 31) >> 5;
}

__global__ void k_lat_fill(const int* __restrict__ nvalid, const int* __restrict__ off, int npl, int b0, int nb, int k0,
                           int ntk, const int4* __restrict__ tickets, int4* __restrict__ chunks) {
  const long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (t >= (long long)ntk * nb) return;
  const int tk = (int)(t / nb), p = (int)(t % nb);
  const int nv = nvalid[t];
  int o = off[t];
  const int bra = tickets[tk].x * npl + b0 + p;
  const int kbase = tickets[tk].y * npl + k0;
  for (int q = 0; q < nv; q += 32, ++o) chunks[o] = make_int4(bra, kbase + q, kbase + min(q + 32, nv), tk);
}

// ---------------------------------------------------------------- build kernel

// (LA LB|LC LD) is the evaluated canonical class; SWAP: its first pair is the ket.
template <int LA, int LB, int LC, int LD, bool SWAP>
__global__ void __launch_bounds__(256) k_lattice(LatticeRun R, OpTableDev tab, int per_warp) {
  constexpr int NA = ncum(LA), NB = ncum(LB), NC = ncum(LC), ND = ncum(LD);
  constexpr int LT = LA + LB + LC + LD;
  // component counts of the bra pair's and the ket pair's canonical centres
  constexpr int N1 = SWAP ? NC : NA, N2 = SWAP ? ND : NB;   // bra first, second
  constexpr int M1 = SWAP ? NA : NC, M2 = SWAP ? NB : ND;   // ket first, second
  constexpr int NBRA = N1 * N2;
  extern __shared__ double smem[];
  __shared__ OpGeom s_geo[8];
  __shared__ OpGeomF s_geof[8];
  __shared__ int s_prm[8][N1 + N2 + M1 + M2];
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, wpb = blockDim.x >> 5;
  double* v = smem + (size_t)wid * per_warp;
  double* DJ = v + tab.nslots;      // D(k,l), [c][d] over ket canonical comps
  double* DK = DJ + M1 * M2;        // D(k,j), [ket comp of K][bra comp of J]
  OpGeom& geo = s_geo[wid];
  OpGeomF& geof = s_geof[wid];
  float* vf = reinterpret_cast<float*>(v);   // the slots as floats on the FP32 path
  unsigned long long n32 = 0;
  int* b1 = s_prm[wid];             // bra first centre prims
  int* b2 = b1 + N1;
  int* k1 = b2 + N2;
  int* k2 = k1 + M1;
  const PairArrays pr = R.pairs;
  const int npgs = R.npgs;
  const size_t pp2 = (size_t)npgs * npgs;
  const LatGeom& g = R.g;
  const int nchunks = *R.nchunks;
  const double c2pi = 2.0 / sqrt(REF_PI);
  const int h3 = g.c2[0] + g.c1[0];
  const bool helix = R.pph != nullptr;
  for (int c = blockIdx.x * wpb + wid; c < nchunks; c += gridDim.x * wpb) {
    const int4 ch = R.chunks[c];
    const int p = ch.x;
    const int4 tk = R.tickets[ch.w];
    const int q1[3] = {R.qcell[3 * tk.x], R.qcell[3 * tk.x + 1], R.qcell[3 * tk.x + 2]};
    const int q2[3] = {R.qcell[3 * tk.y], R.qcell[3 * tk.y + 1], R.qcell[3 * tk.y + 2]};
    const bool swb = R.swp[p] != 0;
    for (int x = lane; x < N1; x += 32) b1[x] = R.prim[pr.si[p] * MAXCOMP + x];
    for (int x = lane; x < N2; x += 32) b2[x] = R.prim[pr.sj[p] * MAXCOMP + x];
    // bra J comps are b2 (first = I) or b1 (first = J)
    const int nI = swb ? N2 : N1, nJ = swb ? N1 : N2;
    double jacc[4] = {0.0, 0.0, 0.0, 0.0};
    const double zb = pr.zeta[p];
    const double Pb[3] = {pr.P[0][p], pr.P[1][p], pr.P[2][p]};
    const double PAb[3] = {pr.PA[0][p], pr.PA[1][p], pr.PA[2][p]};
    const double ABb[3] = {pr.AB[0][p], pr.AB[1][p], pr.AB[2][p]};
    const int c1q1 = cell1_index(g, q1[0], q1[1], q1[2]);
    for (int q3z = -g.c2[2]; q3z <= g.c2[2]; ++q3z)
    for (int q3y = -g.c2[1]; q3y <= g.c2[1]; ++q3y)
    for (int q3x = -g.c2[0]; q3x <= g.c2[0]; ++q3x) {
      const int q3[3] = {q3x, q3y, q3z};
      bool lcel = true;
      for (int k = 0; k < 3; ++k)
        lcel = lcel && (q3[k] + q2[k] >= -g.c1[k]) && (q3[k] + q2[k] <= g.c1[k]) && (q1[k] - q3[k] >= -g.c1[k]) &&
               (q1[k] - q3[k] <= g.c1[k]);
      const double ang = q3x * g.helix, cs = cos(ang), sn = sin(ang);
      const double tr[3] = {q3x * g.period[0], q3y * g.period[1], q3z * g.period[2]};
      // warp-uniform: the whole chunk's kets are images in the same cell Q3
      const bool f32 = R.far32 && LT > 0 &&
                       (abs(q3x) > g.c1[0] || abs(q3y) > g.c1[1] || abs(q3z) > g.c1[2]);
      for (int qq = ch.y; qq < ch.z; ++qq) {
        const bool swk = R.swp[qq] != 0;
        const double ze = pr.zeta[qq];
        const double Qb[3] = {pr.P[0][qq], pr.P[1][qq], pr.P[2][qq]};
        // screw image of the ket pair: rotate about x, then translate
        const double Q[3] = {Qb[0] + tr[0], Qb[1] * cs - Qb[2] * sn + tr[1], Qb[1] * sn + Qb[2] * cs + tr[2]};
        const double QC[3] = {pr.PA[0][qq], pr.PA[1][qq] * cs - pr.PA[2][qq] * sn, pr.PA[1][qq] * sn + pr.PA[2][qq] * cs};
        const double CD[3] = {pr.AB[0][qq], pr.AB[1][qq] * cs - pr.AB[2][qq] * sn, pr.AB[1][qq] * sn + pr.AB[2][qq] * cs};
        const double zz = zb + ze, rho = zb * ze / zz;
        const double T = rho * ((Pb[0] - Q[0]) * (Pb[0] - Q[0]) + (Pb[1] - Q[1]) * (Pb[1] - Q[1]) +
                                (Pb[2] - Q[2]) * (Pb[2] - Q[2]));
        const double pref = c2pi * pr.S[p] * pr.S[qq] * sqrt(rho);
        if (lane == 0) {
          // FP32: the recursion runs on F_m/pref (values of order one); the
          // outputs are scaled back by pref in FP64
          double F[LT + 1];
          boys_tab<LT>(T, f32 ? 1.0 : pref, R.boys, F);
          if (f32) {
            vf[0] = 0.0f;
#pragma unroll
            for (int m = 0; m <= LT; ++m) vf[1 + m] = (float)F[m];
          } else {
            v[0] = 0.0;
#pragma unroll
            for (int m = 0; m <= LT; ++m) v[1 + m] = F[m];
          }
        } else if (lane == 1) {
          double WP[3], WQ[3];
          for (int k = 0; k < 3; ++k) {
            const double W = (zb * Pb[k] + ze * Q[k]) / zz;
            WP[k] = W - Pb[k];
            WQ[k] = W - Q[k];
          }
          if (!SWAP)
            set_geom(geo, PAb, WP, QC, WQ, ABb, CD, 0.5 / zb, 0.5 / ze, 0.5 / zz, rho / zb, rho / ze);
          else
            set_geom(geo, QC, WQ, PAb, WP, CD, ABb, 0.5 / ze, 0.5 / zb, 0.5 / zz, rho / ze, rho / zb);
          if (f32) geom_to_float(geo, geof);
        }
        for (int x = lane; x < M1; x += 32) k1[x] = R.prim[pr.si[qq] * MAXCOMP + x];
        for (int x = lane; x < M2; x += 32) k2[x] = R.prim[pr.sj[qq] * MAXCOMP + x];
        __syncwarp();
        // densities: DJ(c,d) = D(k,l), DK(k comp, j comp) = D(k,j)
        for (int t = lane; t < M1 * M2; t += 32) {
          const int cc = t / M2, d = t % M2;
          const int kp = swk ? k2[d] : k1[cc], lp = swk ? k1[cc] : k2[d];
          double val = 0.0;
          if (kp >= 0 && lp >= 0)
            val = helix ? __ldg(R.pph + kp + (size_t)npgs * lp + pp2 * ((size_t)(q3x + g.c2[0]) + (size_t)(2 * g.c2[0] + 1) * (q3x + q2[0] + h3)))
                        : __ldg(R.pp + kp + (size_t)npgs * lp + pp2 * cell1_index(g, q2[0], q2[1], q2[2]));
          DJ[t] = val;
        }
        const int nK = swk ? M2 : M1, nL = swk ? M1 : M2;
        if (lcel) {
          for (int t = lane; t < nK * nJ; t += 32) {
            const int kc = t / nJ, jc = t % nJ;
            const int kp = swk ? k2[kc] : k1[kc];
            const int jp = swb ? b1[jc] : b2[jc];
            double val = 0.0;
            if (kp >= 0 && jp >= 0)
              val = helix ? __ldg(R.pph + kp + (size_t)npgs * jp + pp2 * ((size_t)(q3x + g.c2[0]) + (size_t)(2 * g.c2[0] + 1) * (q1[0] + h3)))
                          : __ldg(R.pp + kp + (size_t)npgs * jp + pp2 * cell1_index(g, q1[0] - q3x, q1[1] - q3y, q1[2] - q3z));
            DK[t] = val;
          }
        }
        if (f32) {
          ++n32;
          for (int l = 0; l < tab.nlevels; ++l) {
            const int o0 = tab.levels[l], o1 = tab.levels[l + 1];
            run_level(tab.ops, o0, o1, vf, geof, lane, 32, EvalF{});
            __syncwarp();
          }
        } else {
          for (int l = 0; l < tab.nlevels; ++l) {
            const int o0 = tab.levels[l], o1 = tab.levels[l + 1];
            run_level(tab.ops, o0, o1, v, geo, lane, 32, EvalD{});
            __syncwarp();
          }
        }
        // integral of bra comps (a over first, b over second) and ket comps (c, d)
        auto E = [&](int a, int b, int cc, int d) -> double {
          const int idx = SWAP ? ((cc * M2 + d) * N1 + a) * N2 + b : ((a * N2 + b) * M1 + cc) * M2 + d;
          return f32 ? pref * (double)vf[tab.out[idx]] : v[tab.out[idx]];
        };
        // J: C(i,j,Q1) += sum_kl DJ(k,l) (ij|kl), accumulated over the whole chunk
#pragma unroll
        for (int r = 0; r < 4; ++r) {
          const int t = lane + 32 * r;
          if (t < NBRA) {
            const int a = t / N2, b = t % N2;
            double acc = 0.0;
            for (int cc = 0; cc < M1; ++cc)
              for (int d = 0; d < M2; ++d) acc += DJ[cc * M2 + d] * E(a, b, cc, d);
            jacc[r] += acc;
          }
        }
        // K: X(i,l,Q3+Q2) += sum_{j,k} D(k,j) (ij|kl)
        if (lcel) {
          const int cx = cell1_index(g, q3x + q2[0], q3y + q2[1], q3z + q2[2]);
          for (int t = lane; t < nI * nL; t += 32) {
            const int ic = t / nL, lc = t % nL;
            double acc = 0.0;
            for (int jc = 0; jc < nJ; ++jc)
              for (int kc = 0; kc < nK; ++kc) {
                const int a = swb ? jc : ic, b = swb ? ic : jc;
                const int cc = swk ? lc : kc, d = swk ? kc : lc;
                acc += DK[kc * nJ + jc] * E(a, b, cc, d);
              }
            const int ip = swb ? b2[ic] : b1[ic];
            const int lp = swk ? k1[lc] : k2[lc];
            if (ip >= 0 && lp >= 0) atomicAdd(R.xp + ip + (size_t)npgs * lp + pp2 * cx, acc);
          }
        }
        __syncwarp();
      }
    }
    // flush J of this chunk
    if (lane == 0 && n32) atomicAdd(R.n32, n32);
    n32 = 0;
#pragma unroll
    for (int r = 0; r < 4; ++r) {
      const int t = lane + 32 * r;
      if (t < NBRA) {
        const int a = t / N2, b = t % N2;
        const int ip = swb ? b2[b] : b1[a], jp = swb ? b1[a] : b2[b];
        if (ip >= 0 && jp >= 0) atomicAdd(R.cp + ip + (size_t)npgs * jp + pp2 * c1q1, jacc[r]);
      }
    }
    __syncwarp();
  }
}

// ---------------------------------------------------------------- host side

using LatFn = void (*)(const LatticeRun&, const OpTableDev&, int grid, int wpb, int per_warp, size_t smem, cudaStream_t);
using LatAllow = cudaError_t (*)(size_t);

template <int LA, int LB, int LC, int LD, bool SW>
static void launch_lat(const LatticeRun& r, const OpTableDev& t, int grid, int wpb, int per_warp, size_t smem,
                       cudaStream_t s) {
  k_lattice<LA, LB, LC, LD, SW><<<grid, 32 * wpb, smem, s>>>(r, t, per_warp);
}
template <int LA, int LB, int LC, int LD, bool SW>
static cudaError_t allow_lat(size_t smem) {
  return cudaFuncSetAttribute(k_lattice<LA, LB, LC, LD, SW>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
}

struct LatVariant {
  LatFn fn;
  LatAllow allow;
};

// evaluated class (e1 >= e2), swap flag
static LatVariant lat_variant(int e1, int e2, bool sw) {
#define LV(A, B, C, D)                                                                        \
  (sw ? LatVariant{&launch_lat<A, B, C, D, true>, &allow_lat<A, B, C, D, true>}               \
      : LatVariant{&launch_lat<A, B, C, D, false>, &allow_lat<A, B, C, D, false>})
  switch (e1 * 8 + e2) {
    case 0: return LV(0, 0, 0, 0);
    case 8: return LV(1, 0, 0, 0);
    case 9: return LV(1, 0, 1, 0);
    case 16: return LV(1, 1, 0, 0);
    case 17: return LV(1, 1, 1, 0);
    case 18: return LV(1, 1, 1, 1);
    case 24: return LV(2, 0, 0, 0);
    case 25: return LV(2, 0, 1, 0);
    case 26: return LV(2, 0, 1, 1);
    case 27: return LV(2, 0, 2, 0);
    case 32: return LV(2, 1, 0, 0);
    case 33: return LV(2, 1, 1, 0);
    case 34: return LV(2, 1, 1, 1);
    case 35: return LV(2, 1, 2, 0);
    case 36: return LV(2, 1, 2, 1);
    case 40: return LV(2, 2, 0, 0);
    case 41: return LV(2, 2, 1, 0);
    case 42: return LV(2, 2, 1, 1);
    case 43: return LV(2, 2, 2, 0);
    case 44: return LV(2, 2, 2, 1);
    default: return LV(2, 2, 2, 2);
  }
#undef LV
}

static LatGeom make_geom(const pfe_context* ctx) {
  LatGeom g{};
  for (int k = 0; k < 3; ++k) {
    g.c1[k] = ctx->cel1[k];
    g.c2[k] = ctx->cel2[k];
    g.n1[k] = 2 * ctx->cel1[k] + 1;
    g.period[k] = ctx->period[k];
  }
  g.helix = ctx->helix;
  return g;
}

static int compute_schwarz(pfe_context* ctx, PairArrays recs, long long n, cudaStream_t s) {
  const int bs = 128;
  k_schwarz_small<<<(unsigned)((n + bs - 1) / bs), bs, 0, s>>>(recs, ctx->shells.prim, ctx->d_maxc, ctx->d_boys, n);
  PFE_CUDA(cudaGetLastError());
  int *list = nullptr, *cnt = nullptr;
  PFE_CUDA(ctx->alloc((void**)&list, sizeof(int) * n));
  PFE_CUDA(ctx->alloc((void**)&cnt, sizeof(int)));
  for (int cls = 4; cls <= 5; ++cls) {
    PFE_CUDA(cudaMemsetAsync(cnt, 0, sizeof(int), s));
    k_select_cls<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(recs.cls, cls, list, cnt, n);
    int hn = 0;
    PFE_CUDA(cudaMemcpyAsync(&hn, cnt, sizeof(int), cudaMemcpyDeviceToHost, s));
    PFE_CUDA(cudaStreamSynchronize(s));
    if (hn == 0) continue;
    const OpTableHost* h = host_optable(cls, cls);
    OpTableDev d{};
    int rc;
    if ((rc = upload_optable(ctx, h, &d)) != PFE_OK) return rc;
    const size_t smem = sizeof(double) * (size_t)h->nslots;
    if (cls == 4) {
      PFE_CUDA(cudaFuncSetAttribute(k_schwarz_big<2, 1>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
      k_schwarz_big<2, 1><<<std::min(hn, 4 * ctx->num_sms), 256, smem, s>>>(recs, ctx->shells.prim, ctx->d_maxc, list, hn, d);
    } else {
      PFE_CUDA(cudaFuncSetAttribute(k_schwarz_big<2, 2>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
      k_schwarz_big<2, 2><<<std::min(hn, 4 * ctx->num_sms), 256, smem, s>>>(recs, ctx->shells.prim, ctx->d_maxc, list, hn, d);
    }
    PFE_CUDA(cudaGetLastError());
    PFE_CUDA(cudaStreamSynchronize(s));
  }
  ctx->free_now(list);
  ctx->free_now(cnt);
  k_lat_keys<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(recs, n);
  PFE_CUDA(cudaGetLastError());
  return PFE_OK;
}

__global__ void k_lat_gather(PairArrays src, const unsigned char* sws, PairArrays dst, unsigned char* swd,
                             const int* __restrict__ perm, long long n) {
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
  swd[t] = sws[s];
}

__global__ void k_iota_lat(int* p, long long n) {
  const long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (t < n) p[t] = (int)t;
}

__global__ void k_lat_listkey(unsigned short* key, long long npl, long long n) {
  const long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (t < n) key[t] = (unsigned short)(t / npl);
}

__global__ void k_gather_u8_lat(const unsigned char* src, const int* perm, unsigned char* dst, long long n) {
  const long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (t < n) dst[t] = src[perm[t]];
}

__global__ void k_gather_u16(const unsigned short* src, const int* perm, unsigned short* dst, long long n) {
  const long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (t < n) dst[t] = src[perm[t]];
}

int lattice_setup(pfe_context* ctx, const pfe_args* a) {
  cudaStream_t s = ctx->stream;
  LatticeState* L = new LatticeState();
  ctx->lattice = L;
  PFE_CUDA(ctx->alloc((void**)&L->d_queue, sizeof(int) * 64 * kLatQueueSlots));
  if (!ctx->d_n32) {   // FP32 quartet counter of the mixed-precision path
    PFE_CUDA(ctx->alloc((void**)&ctx->d_n32, sizeof(unsigned long long)));
    PFE_CUDA(cudaMemset(ctx->d_n32, 0, sizeof(unsigned long long)));
  }
  const LatGeom g = make_geom(ctx);
  const int n = ctx->npshell;
  // cells of the REDUCED_CEL1 box, x fastest within the list index
  for (int qz = -ctx->rc1[2]; qz <= ctx->rc1[2]; ++qz)
    for (int qy = -ctx->rc1[1]; qy <= ctx->rc1[1]; ++qy)
      for (int qx = -ctx->rc1[0]; qx <= ctx->rc1[0]; ++qx) {
        L->qcell.push_back(qx);
        L->qcell.push_back(qy);
        L->qcell.push_back(qz);
      }
  L->nq = (int)L->qcell.size() / 3;
  L->npl = n * n;
  const long long ntot = (long long)L->nq * L->npl;
  if (ntot >= (1ll << 31)) { set_error("lattice pair lists too large"); return PFE_EUNSUPPORTED; }
  auto list_of = [&](int qx, int qy, int qz) {
    const int nx = 2 * ctx->rc1[0] + 1, ny = 2 * ctx->rc1[1] + 1;
    return (qx + ctx->rc1[0]) + nx * ((qy + ctx->rc1[1]) + ny * (qz + ctx->rc1[2]));
  };
  PFE_CUDA(ctx->alloc((void**)&L->d_qcell, sizeof(int) * L->qcell.size()));
  PFE_CUDA(cudaMemcpy(L->d_qcell, L->qcell.data(), sizeof(int) * L->qcell.size(), cudaMemcpyHostToDevice));
  int rc;
  PairArrays raw{};
  if ((rc = alloc_pairs(ctx, &raw, ntot)) != PFE_OK) return rc;
  if ((rc = alloc_pairs(ctx, &L->pairs, ntot)) != PFE_OK) return rc;
  unsigned char *sw_raw = nullptr;
  PFE_CUDA(ctx->alloc((void**)&sw_raw, ntot));
  PFE_CUDA(ctx->alloc((void**)&L->swp, ntot));
  k_lat_pairs<<<(unsigned)((ntot + 127) / 128), 128, 0, s>>>(ctx->shells, g, L->d_qcell, L->nq, ctx->d_sss, raw, sw_raw);
  PFE_CUDA(cudaGetLastError());
  if ((rc = compute_schwarz(ctx, raw, ntot, s)) != PFE_OK) return rc;
  // sort: bound descending, then class, then list cell (each pass stable)
  {
    int *pa = nullptr, *pb = nullptr;
    unsigned long long* kb = nullptr;
    unsigned char *c1 = nullptr, *c2 = nullptr;
    unsigned short *l1 = nullptr, *l2 = nullptr;
    PFE_CUDA(ctx->alloc((void**)&pa, sizeof(int) * ntot));
    PFE_CUDA(ctx->alloc((void**)&pb, sizeof(int) * ntot));
    PFE_CUDA(ctx->alloc((void**)&kb, sizeof(unsigned long long) * ntot));
    PFE_CUDA(ctx->alloc((void**)&c1, ntot));
    PFE_CUDA(ctx->alloc((void**)&c2, ntot));
    PFE_CUDA(ctx->alloc((void**)&l1, sizeof(unsigned short) * ntot));
    PFE_CUDA(ctx->alloc((void**)&l2, sizeof(unsigned short) * ntot));
    k_iota_lat<<<(unsigned)((ntot + 255) / 256), 256, 0, s>>>(pa, ntot);
    size_t t1 = 0, t2 = 0, t3 = 0;
    cub::DeviceRadixSort::SortPairs(nullptr, t1, raw.key, kb, pa, pb, (int)ntot, 0, 64, s);
    cub::DeviceRadixSort::SortPairs(nullptr, t2, c1, c2, pb, pa, (int)ntot, 0, 8, s);
    cub::DeviceRadixSort::SortPairs(nullptr, t3, l1, l2, pa, pb, (int)ntot, 0, 16, s);
    const size_t tb = std::max(t1, std::max(t2, t3)) + 16;
    void* tmp = nullptr;
    PFE_CUDA(ctx->alloc(&tmp, tb));
    size_t tbb = tb;
    PFE_CUDA(cub::DeviceRadixSort::SortPairs(tmp, tbb, raw.key, kb, pa, pb, (int)ntot, 0, 64, s));
    k_gather_u8_lat<<<(unsigned)((ntot + 255) / 256), 256, 0, s>>>(raw.cls, pb, c1, ntot);
    tbb = tb;
    PFE_CUDA(cub::DeviceRadixSort::SortPairs(tmp, tbb, c1, c2, pb, pa, (int)ntot, 0, 8, s));
    k_lat_listkey<<<(unsigned)((ntot + 255) / 256), 256, 0, s>>>(l2, L->npl, ntot);
    k_gather_u16<<<(unsigned)((ntot + 255) / 256), 256, 0, s>>>(l2, pa, l1, ntot);
    tbb = tb;
    PFE_CUDA(cub::DeviceRadixSort::SortPairs(tmp, tbb, l1, l2, pa, pb, (int)ntot, 0, 16, s));
    k_lat_gather<<<(unsigned)((ntot + 127) / 128), 128, 0, s>>>(raw, sw_raw, L->pairs, L->swp, pb, ntot);
    PFE_CUDA(cudaGetLastError());
    PFE_CUDA(cudaStreamSynchronize(s));
    for (void* p : {(void*)pa, (void*)pb, (void*)kb, (void*)c1, (void*)c2, (void*)l1, (void*)l2, tmp}) ctx->free_now(p);
  }
  free_pairs(ctx, &raw);
  ctx->free_now(sw_raw);
  // per-list class offsets (identical for every list)
  {
    std::vector<int> cnt(6, 0);
    std::vector<int> L_sh(n);
    for (int i = 0; i < n; ++i) L_sh[i] = 0;
    PFE_CUDA(cudaMemcpy(L_sh.data(), ctx->shells.L, sizeof(int) * n, cudaMemcpyDeviceToHost));
    for (int I = 0; I < n; ++I)
      for (int J = 0; J < n; ++J) {
        const int la = std::max(L_sh[I], L_sh[J]), lb = std::min(L_sh[I], L_sh[J]);
        cnt[pair_class(la, lb)]++;
      }
    int off = 0;
    for (int c = 0; c < 6; ++c) {
      L->cls_off[c] = off;
      L->cls_n[c] = cnt[c];
      off += cnt[c];
    }
  }
  // tickets in the reference's round-robin order
  {
    int ticket = 0;
    for (int q1x = -ctx->rc1[0]; q1x <= ctx->rc1[0]; ++q1x)
      for (int q1y = -ctx->rc1[1]; q1y <= ctx->rc1[1]; ++q1y)
        for (int q1z = -ctx->rc1[2]; q1z <= ctx->rc1[2]; ++q1z)
          for (int q2x = -ctx->rc1[0]; q2x <= ctx->rc1[0]; ++q2x)
            for (int q2y = -ctx->rc1[1]; q2y <= ctx->rc1[1]; ++q2y)
              for (int q2z = -ctx->rc1[2]; q2z <= ctx->rc1[2]; ++q2z) {
                ticket += 1;
                if (ticket == ctx->numprocs) ticket -= ctx->numprocs;
                if (ctx->myid != ticket) continue;
                L->h_tickets.push_back(make_int4(list_of(q1x, q1y, q1z), list_of(q2x, q2y, q2z), 0, 0));
              }
    L->ntk = (int)L->h_tickets.size();
  }
  if (L->ntk == 0) { L->nlaunch = 0; return PFE_OK; }
  PFE_CUDA(ctx->alloc((void**)&L->d_tickets, sizeof(int4) * L->ntk));
  PFE_CUDA(cudaMemcpy(L->d_tickets, L->h_tickets.data(), sizeof(int4) * L->ntk, cudaMemcpyHostToDevice));
  // the reference's bra bounds per ticket
  {
    const long long nj = (long long)L->ntk * L->npl;
    PairArrays jobs{};
    if ((rc = alloc_pairs(ctx, &jobs, nj)) != PFE_OK) return rc;
    k_lat_quirk_jobs<<<(unsigned)((nj + 127) / 128), 128, 0, s>>>(ctx->shells, g, L->d_tickets, L->ntk, L->d_qcell,
                                                                  L->pairs, L->npl, L->swp, ctx->d_sss, jobs);
    PFE_CUDA(cudaGetLastError());
    if ((rc = compute_schwarz(ctx, jobs, nj, s)) != PFE_OK) return rc;
    PFE_CUDA(ctx->alloc((void**)&L->d_quirk, sizeof(double) * nj));
    PFE_CUDA(cudaMemcpyAsync(L->d_quirk, jobs.schwarz, sizeof(double) * nj, cudaMemcpyDeviceToDevice, s));
    PFE_CUDA(cudaStreamSynchronize(s));
    free_pairs(ctx, &jobs);
  }
  // chunk lists per (bra class, ket class)
  const int maxn = *std::max_element(L->cls_n, L->cls_n + 6);
  const long long maxt = (long long)L->ntk * maxn + 1;
  int *nvalid = nullptr, *nchunk = nullptr, *offs = nullptr;
  long long* d_sum = nullptr;
  PFE_CUDA(ctx->alloc((void**)&nvalid, sizeof(int) * maxt));
  PFE_CUDA(ctx->alloc((void**)&nchunk, sizeof(int) * maxt));
  PFE_CUDA(ctx->alloc((void**)&offs, sizeof(int) * maxt));
  PFE_CUDA(ctx->alloc((void**)&d_sum, sizeof(long long)));
  L->nlaunch = 0;
  int ncell3 = (2 * ctx->cel2[0] + 1) * (2 * ctx->cel2[1] + 1) * (2 * ctx->cel2[2] + 1);
  for (int cb = 0; cb < 6; ++cb)
    for (int ck = 0; ck < 6; ++ck) {
      const int nb = L->cls_n[cb], nk = L->cls_n[ck];
      if (nb == 0 || nk == 0) continue;
      const long long nt = (long long)L->ntk * nb;
      k_lat_count<<<(unsigned)((nt + 127) / 128), 128, 0, s>>>(L->d_quirk, L->pairs.schwarz, L->npl, L->cls_off[cb], nb,
                                                               L->cls_off[ck], nk, L->ntk, L->d_tickets, ctx->inttol,
                                                               nvalid, nchunk);
      PFE_CUDA(cudaGetLastError());
      PFE_CUDA(cudaMemsetAsync(nchunk + nt, 0, sizeof(int), s));
      size_t sb = 0;
      cub::DeviceScan::ExclusiveSum(nullptr, sb, nchunk, offs, (int)(nt + 1), s);
      void* st = nullptr;
      PFE_CUDA(ctx->alloc(&st, sb + 16));
      PFE_CUDA(cub::DeviceScan::ExclusiveSum(st, sb, nchunk, offs, (int)(nt + 1), s));
      size_t rb = 0;
      cub::DeviceReduce::Sum(nullptr, rb, nvalid, d_sum, (int)nt, s);
      void* rt = nullptr;
      PFE_CUDA(ctx->alloc(&rt, rb + 16));
      PFE_CUDA(cub::DeviceReduce::Sum(rt, rb, nvalid, d_sum, (int)nt, s));
      int total = 0;
      long long nq = 0;
      PFE_CUDA(cudaMemcpyAsync(&total, offs + nt, sizeof(int), cudaMemcpyDeviceToHost, s));
      PFE_CUDA(cudaMemcpyAsync(&nq, d_sum, sizeof(long long), cudaMemcpyDeviceToHost, s));
      PFE_CUDA(cudaStreamSynchronize(s));
      ctx->free_now(st);
      ctx->free_now(rt);
      if (total == 0) continue;
      LatticeLaunch& ll = L->launches[L->nlaunch];
      ll = LatticeLaunch{};
      ll.cb = cb;
      ll.ck = ck;
      ll.ncells_chunks = total;
      ll.quartets = (double)nq * ncell3;
      PFE_CUDA(ctx->alloc((void**)&ll.chunks, sizeof(int4) * total));
      PFE_CUDA(ctx->alloc((void**)&ll.d_nchunks, sizeof(int)));
      PFE_CUDA(cudaMemcpyAsync(ll.d_nchunks, &total, sizeof(int), cudaMemcpyHostToDevice, s));
      k_lat_fill<<<(unsigned)((nt + 127) / 128), 128, 0, s>>>(nvalid, offs, L->npl, L->cls_off[cb], nb, L->cls_off[ck],
                                                              L->ntk, L->d_tickets, ll.chunks);
      PFE_CUDA(cudaGetLastError());
      const int e1 = std::max(cb, ck), e2 = std::min(cb, ck);
      const OpTableHost* h = host_optable(e1, e2);
      if ((rc = upload_optable(ctx, h, &ll.tab)) != PFE_OK) return rc;
      static const int Lc[6][2] = {{0, 0}, {1, 0}, {1, 1}, {2, 0}, {2, 1}, {2, 2}};
      const int nbra = ncum(Lc[cb][0]) * ncum(Lc[cb][1]);
      const int nket = ncum(Lc[ck][0]) * ncum(Lc[ck][1]);
      const int maxc = std::max(ncum(Lc[ck][0]), ncum(Lc[ck][1]));
      const int maxj = std::max(ncum(Lc[cb][0]), ncum(Lc[cb][1]));
      ll.per_warp = h->nslots + nket + maxc * maxj;
      ll.wpb = (int)std::max<size_t>(1, std::min<size_t>(8, (200 * 1024) / (sizeof(double) * ll.per_warp)));
      ll.smem = sizeof(double) * (size_t)ll.per_warp * ll.wpb;
      (void)nbra;
      PFE_CUDA(lat_variant(e1, e2, cb < ck).allow(ll.smem));
      PFE_CUDA(cudaStreamSynchronize(s));
      L->quartets += ll.quartets;
      L->flops += ll.quartets * class_flops(e1, e2);
      L->nlaunch++;
    }
  ctx->free_now(nvalid);
  ctx->free_now(nchunk);
  ctx->free_now(offs);
  ctx->free_now(d_sum);
  ctx->census_quartets = L->quartets;
  ctx->census_ref = L->quartets;
  ctx->census_flops = L->flops;
  ctx->npairs = ntot;
  ctx->nlaunch = L->nlaunch;
  return PFE_OK;
}

int lattice_fock(pfe_context* ctx, const double* d_pp, const double* d_pph, double* d_cc, double* d_xc,
                 cudaStream_t s) {
  LatticeState* L = (LatticeState*)ctx->lattice;
  const size_t pp = (size_t)ctx->npgs * ctx->npgs * ctx->ncell1;
  PFE_CUDA(cudaMemsetAsync(ctx->d_jp, 0, sizeof(double) * pp, s));
  PFE_CUDA(cudaMemsetAsync(ctx->d_kp, 0, sizeof(double) * pp, s));
  LatticeRun R{};
  R.pairs = L->pairs;
  R.swp = L->swp;
  R.prim = ctx->shells.prim;
  R.boys = ctx->d_boys;
  R.pp = d_pp;
  R.pph = ctx->helix != 0.0 ? d_pph : nullptr;
  R.cp = ctx->d_jp;
  R.xp = ctx->d_kp;
  R.tickets = L->d_tickets;
  R.qcell = L->d_qcell;
  R.g = make_geom(ctx);
  R.npgs = ctx->npgs;
  R.far32 = ctx->mcut > 0.0 ? 1 : 0;
  R.n32 = ctx->d_n32;
  PFE_CUDA(cudaMemsetAsync(ctx->d_n32, 0, sizeof(unsigned long long), s));
  PFE_CUDA(cudaMemsetAsync(L->d_queue, 0, sizeof(int) * 64 * kLatQueueSlots, s));
  for (int i = 0; i < L->nlaunch; ++i) {
    const LatticeLaunch& ll = L->launches[i];
    R.chunks = ll.chunks;
    R.nchunks = ll.d_nchunks;
    R.queue = L->d_queue + kLatQueueSlots * i;
    const int e1 = std::max(ll.cb, ll.ck), e2 = std::min(ll.cb, ll.ck);
    if (LatSlFn f = L->interpret_only ? nullptr : lattice_sl_launcher(e1, e2, ll.cb < ll.ck)) {
      // straight-line: one chunk per warp from the queue, a persistent grid of 16 blocks per SM
      const int grid = std::min((ll.ncells_chunks + 3) / 4, ctx->num_sms * 16);
      f(R, std::max(grid, 1), s);
    } else {
      int grid = std::min((ll.ncells_chunks + ll.wpb - 1) / ll.wpb, ctx->num_sms * 8);
      lat_variant(e1, e2, ll.cb < ll.ck).fn(R, ll.tab, std::max(grid, 1), ll.wpb, ll.per_warp, ll.smem, s);
    }
    PFE_CUDA(cudaGetLastError());
  }
  int rc = contract_outputs(ctx, ctx->d_jp, ctx->d_kp, d_cc, d_xc, /*symmetrize=*/false, ctx->ncell1, s);
  if (rc != PFE_OK) return rc;
  if (ctx->helix != 0.0) {
    // C_C(:,:,q) <- C_C(:,:,q) C2H(:,:,q)^T along the screw axis (cells are x only)
    const int nc = ctx->ncgs, nx = 2 * ctx->cel1[0] + 1, h3 = ctx->cel2[0] + ctx->cel1[0];
    const double one = 1.0, zero = 0.0;
    if (!ensure_blas(ctx)) { set_error("cublasCreate failed"); return PFE_ECUDA; }
    cublasSetStream(ctx->blas, s);
    double* outs[2] = {d_cc, d_xc};
    for (int o = 0; o < 2; ++o) {
      cublasStatus_t st = cublasDgemmStridedBatched(
          ctx->blas, CUBLAS_OP_N, CUBLAS_OP_T, nc, nc, nc, &one, outs[o], nc, (long long)nc * nc,
          ctx->d_c2h + (size_t)(h3 - ctx->cel1[0]) * nc * nc, nc, (long long)nc * nc, &zero, ctx->d_w2, nc,
          (long long)nc * nc, nx);
      if (st != CUBLAS_STATUS_SUCCESS) { set_error("cublasDgemmStridedBatched (C2H) failed"); return PFE_ECUDA; }
      PFE_CUDA(cudaMemcpyAsync(outs[o], ctx->d_w2, sizeof(double) * (size_t)nc * nc * nx, cudaMemcpyDeviceToDevice, s));
    }
  }
  return PFE_OK;
}

// Class kernel launches of one lattice build: a straight-line class's register
// passes, one launch for an interpreted class.
int lattice_class_launches(pfe_context* ctx) {
  const LatticeState* L = (const LatticeState*)ctx->lattice;
  if (!L) return 0;
  int n = 0;
  for (int i = 0; i < L->nlaunch; ++i) {
    const LatticeLaunch& ll = L->launches[i];
    const int e1 = std::max(ll.cb, ll.ck), e2 = std::min(ll.cb, ll.ck);
    n += L->interpret_only ? 1 : std::max(1, lattice_sl_passes(e1, e2));
  }
  return n;
}

void lattice_force_interpreter(pfe_context* ctx, bool on) {
  if (ctx->lattice) ((LatticeState*)ctx->lattice)->interpret_only = on;
}

void lattice_release(pfe_context* ctx) {
  delete (LatticeState*)ctx->lattice;
  ctx->lattice = nullptr;
}

}  // namespace pfe
