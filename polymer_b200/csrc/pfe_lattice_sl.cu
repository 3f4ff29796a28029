// Straight-line lattice/helix quartet kernels: one (ticket, bra pair) chunk per
// warp and one of its kets per lane.
//
// The lattice path (pfe_lattice.cu) follows the reference's loop without
// permutational symmetry: for the chunk's bra pair (I@0, J@Q1) and every ket
// pair (K@0, L@Q2) of the chunk, every image cell Q3 of the CUTOFF2 box gives
// the quartet (I@0 J@Q1 | K@Q3 L@Q3+Q2) (the screw image of the ket about the
// helix axis), digested as
//   C_P(i,j,Q1)    += D(k,l) (ij|kl),  D = P_P(:,:,Q2)   or P_P_HELIX(:,:,Q3,Q3+Q2)
//   X_P(i,l,Q3+Q2) += D(k,j) (ij|kl),  D = P_P(:,:,Q1-Q3) or P_P_HELIX(:,:,Q3,Q1)
// (src/pfourindexdirect.f90:691-740), the second only where Q3+Q2 and Q1-Q3
// lie inside CUTOFF1.  Here every lane evaluates its own ket's quartet of one
// cell Q3 at a time with the generated straight-line recursion (the integrals
// stay in registers and are digested as they are produced): the J sums of the
// bra's components accumulate in registers over the chunk's kets and cells and
// are reduced over the warp once, the K contributions go straight to the
// atomics.  Classes of up to 64 integrals in one launch; (11|11) in four
// register passes, pass p keeping the chunk bra's first component a = p (64
// integrals each; the K sums of a pass are partial sums over the kept
// components, so the passes' atomics add up to the full digestion).  Larger
// classes keep the interpreter.
// With mixed precision the cells Q3 outside the CUTOFF1 box (the far cells)
// run the recursion in FP32 on F_m/pref, the rest in FP64.

#include "pfe_common.cuh"
#include "pfe_context.cuh"
#include "pfe_interp.cuh"
#include "pfe_lattice.cuh"
#include "pfe_mol_kernels.cuh"

namespace pfe {

namespace {

// K digestion of one quartet: X(i,l,cell) += sum_{j,k} D(k,j) (ij|kl), with the
// bra's (SWB) and the ket's (SWK) centre order fixed at compile time so that
// every integral index is a constant (the integrals stay in registers); only the
// integrals whose chunk-bra first component lies in [A0, A1) (this pass's).
template <int N1, int N2, int M1, int M2, bool SWAP, bool SWB, bool SWK, int A0, int A1>
__device__ __forceinline__ void lat_k(const double* out, const int* b1, const int* b2, const int* k1, const int* k2,
                                      const double* __restrict__ Dk, size_t ck, double* __restrict__ xp, size_t cx,
                                      int npgs) {
  constexpr int nI = SWB ? N2 : N1, nJ = SWB ? N1 : N2;
  constexpr int nK = SWK ? M2 : M1, nL = SWK ? M1 : M2;
  double dk[nK * nJ];
#pragma unroll
  for (int kc = 0; kc < nK; ++kc)
#pragma unroll
    for (int jc = 0; jc < nJ; ++jc) {
      const int kp = SWK ? k2[kc] : k1[kc];
      const int jp = SWB ? b1[jc] : b2[jc];
      dk[kc * nJ + jc] = (kp >= 0 && jp >= 0) ? __ldg(Dk + kp + (size_t)npgs * jp + ck) : 0.0;
    }
#pragma unroll
  for (int ic = 0; ic < nI; ++ic) {
    if (!SWB && (ic < A0 || ic >= A1)) continue;
#pragma unroll
    for (int lc = 0; lc < nL; ++lc) {
      double acc = 0.0;
#pragma unroll
      for (int jc = 0; jc < nJ; ++jc) {
        if (SWB && (jc < A0 || jc >= A1)) continue;
#pragma unroll
        for (int kc = 0; kc < nK; ++kc) {
          const int a = SWB ? jc : ic, b = SWB ? ic : jc;
          const int cc = SWK ? lc : kc, d = SWK ? kc : lc;
          const int idx = SWAP ? ((cc * M2 + d) * N1 + a) * N2 + b : ((a * N2 + b) * M1 + cc) * M2 + d;
          acc = fma(dk[kc * nJ + jc], out[idx], acc);
        }
      }
      const int ip = SWB ? b2[ic] : b1[ic];
      const int lp = SWK ? k1[lc] : k2[lc];
      if (ip >= 0 && lp >= 0 && acc != 0.0) atomicAdd(xp + ip + (size_t)npgs * lp + cx, acc);
    }
  }
}

// (LA LB|LC LD) is the evaluated canonical class; SWAP: the chunk's bra pair is
// its ket pair (the chunk's bra class is the lower one).  Register pass PASS of
// NPASS keeps the chunk bra's first components [A0, A1).
template <int LA, int LB, int LC, int LD, bool SWAP, int NPASS = 1, int PASS = 0>
__global__ void __launch_bounds__(128) k_lat_sl(LatticeRun R) {
  constexpr int NA = ncum(LA), NB = ncum(LB), NC = ncum(LC), ND = ncum(LD);
  constexpr int LT = LA + LB + LC + LD;
  constexpr int NI = NA * NB * NC * ND;
  constexpr int N1 = SWAP ? NC : NA, N2 = SWAP ? ND : NB;   // the chunk's bra: first, second centre
  constexpr int M1 = SWAP ? NA : NC, M2 = SWAP ? NB : ND;   // the lane's ket: first, second centre
  constexpr int NBRA = N1 * N2;
  constexpr int A0 = PASS * N1 / NPASS, A1 = (PASS + 1) * N1 / NPASS;
  static_assert(A0 < A1, "every pass keeps a component");
  const int lane = threadIdx.x & 31;
  const PairArrays pr = R.pairs;
  const int npgs = R.npgs;
  const size_t pp2 = (size_t)npgs * npgs;
  const LatGeom& g = R.g;
  const int nchunks = *R.nchunks;
  const double c2pi = 2.0 / sqrt(REF_PI);
  const int h3 = g.c2[0] + g.c1[0];
  const bool helix = R.pph != nullptr;
  unsigned long long n32 = 0;
  // cos and sin of the screw angle of every image cell along x, once per block
  // (the same functions of the same arguments the lanes would evaluate per cell)
  constexpr int kMaxRot = 257;
  __shared__ double s_cs[kMaxRot], s_sn[kMaxRot];
  const int nrot = 2 * g.c2[0] + 1;
  const bool rot_tab = nrot <= kMaxRot;
  if (rot_tab)
    for (int i = threadIdx.x; i < nrot; i += blockDim.x) {
      const double ang = (i - g.c2[0]) * g.helix;
      s_cs[i] = cos(ang);
      s_sn[i] = sin(ang);
    }
  __syncthreads();
  for (;;) {
    int tk = 0;
    if (lane == 0) tk = atomicAdd(R.queue, 1);
    const int c = __shfl_sync(0xffffffffu, tk, 0);
    if (c >= nchunks) break;
    const int4 ch = R.chunks[c];
    const int p = ch.x;
    const int4 tkt = R.tickets[ch.w];
    const int q1[3] = {R.qcell[3 * tkt.x], R.qcell[3 * tkt.x + 1], R.qcell[3 * tkt.x + 2]};
    const int q2[3] = {R.qcell[3 * tkt.y], R.qcell[3 * tkt.y + 1], R.qcell[3 * tkt.y + 2]};
    const bool swb = R.swp[p] != 0;
    int b1[N1], b2[N2];
#pragma unroll
    for (int x = 0; x < N1; ++x) b1[x] = R.prim[pr.si[p] * MAXCOMP + x];
#pragma unroll
    for (int x = 0; x < N2; ++x) b2[x] = R.prim[pr.sj[p] * MAXCOMP + x];
    const double zb = pr.zeta[p], Sb = pr.S[p];
    const double Pb[3] = {pr.P[0][p], pr.P[1][p], pr.P[2][p]};
    const double PAb[3] = {pr.PA[0][p], pr.PA[1][p], pr.PA[2][p]};
    const double ABb[3] = {pr.AB[0][p], pr.AB[1][p], pr.AB[2][p]};
    // this lane's ket
    const int qq = ch.y + lane;
    const bool act = qq < ch.z;
    const int qk = act ? qq : ch.y;
    const bool swk = R.swp[qk] != 0;
    int k1[M1], k2[M2];
#pragma unroll
    for (int x = 0; x < M1; ++x) k1[x] = R.prim[pr.si[qk] * MAXCOMP + x];
#pragma unroll
    for (int x = 0; x < M2; ++x) k2[x] = R.prim[pr.sj[qk] * MAXCOMP + x];
    const double ze = pr.zeta[qk], Sk = pr.S[qk];
    const double Qb[3] = {pr.P[0][qk], pr.P[1][qk], pr.P[2][qk]};
    const double QCb[3] = {pr.PA[0][qk], pr.PA[1][qk], pr.PA[2][qk]};
    const double CDb[3] = {pr.AB[0][qk], pr.AB[1][qk], pr.AB[2][qk]};
    const double zz = zb + ze, rzz = 1.0 / zz, rho = zb * ze * rzz;
    const double pref = c2pi * Sb * Sk * sqrt(rho);
    double jacc[NBRA];
#pragma unroll
    for (int t = 0; t < NBRA; ++t) jacc[t] = 0.0;
    // translational J density D(k,l) of the ket: the same for every cell Q3
    double dj[M1 * M2];
    if (!helix) {
#pragma unroll
      for (int t = 0; t < M1 * M2; ++t) {
        const int cc = t / M2, d = t % M2;
        const int kp = swk ? k2[d] : k1[cc], lp = swk ? k1[cc] : k2[d];
        dj[t] = (act && kp >= 0 && lp >= 0)
                    ? __ldg(R.pp + kp + (size_t)npgs * lp + pp2 * cell1_index(g, q2[0], q2[1], q2[2]))
                    : 0.0;
      }
    }
    for (int q3z = -g.c2[2]; q3z <= g.c2[2]; ++q3z)
    for (int q3y = -g.c2[1]; q3y <= g.c2[1]; ++q3y)
    for (int q3x = -g.c2[0]; q3x <= g.c2[0]; ++q3x) {
      const int q3[3] = {q3x, q3y, q3z};
      bool lcel = true;
#pragma unroll
      for (int k = 0; k < 3; ++k)
        lcel = lcel && (q3[k] + q2[k] >= -g.c1[k]) && (q3[k] + q2[k] <= g.c1[k]) && (q1[k] - q3[k] >= -g.c1[k]) &&
               (q1[k] - q3[k] <= g.c1[k]);
      const bool f32 = R.far32 && LT > 0 && (abs(q3x) > g.c1[0] || abs(q3y) > g.c1[1] || abs(q3z) > g.c1[2]);
      if (!act) continue;
      double cs, sn;
      if (rot_tab) {
        cs = s_cs[q3x + g.c2[0]];
        sn = s_sn[q3x + g.c2[0]];
      } else {
        const double ang = q3x * g.helix;
        cs = cos(ang);
        sn = sin(ang);
      }
      // screw image of the ket pair: rotate about x, then translate
      const double Q[3] = {Qb[0] + q3x * g.period[0], Qb[1] * cs - Qb[2] * sn + q3y * g.period[1],
                           Qb[1] * sn + Qb[2] * cs + q3z * g.period[2]};
      const double QC[3] = {QCb[0], QCb[1] * cs - QCb[2] * sn, QCb[1] * sn + QCb[2] * cs};
      const double CD[3] = {CDb[0], CDb[1] * cs - CDb[2] * sn, CDb[1] * sn + CDb[2] * cs};
      const double dx = Pb[0] - Q[0], dy = Pb[1] - Q[1], dz = Pb[2] - Q[2];
      const double T = rho * (dx * dx + dy * dy + dz * dz);
      double F[LT + 1];
      boys_tab<LT>(T, f32 ? 1.0 : pref, R.boys, F);
      double out[NI];
      if constexpr (LT == 0) {
        out[0] = F[0];
      } else {
        EriGeom<double> e;
        const double W[3] = {(zb * Pb[0] + ze * Q[0]) * rzz, (zb * Pb[1] + ze * Q[1]) * rzz,
                             (zb * Pb[2] + ze * Q[2]) * rzz};
#pragma unroll
        for (int k = 0; k < 3; ++k) {
          if (!SWAP) {
            e.PA[k] = PAb[k]; e.WP[k] = W[k] - Pb[k]; e.QC[k] = QC[k]; e.WQ[k] = W[k] - Q[k];
            e.AB[k] = ABb[k]; e.CD[k] = CD[k];
          } else {
            e.PA[k] = QC[k]; e.WP[k] = W[k] - Q[k]; e.QC[k] = PAb[k]; e.WQ[k] = W[k] - Pb[k];
            e.AB[k] = CD[k]; e.CD[k] = ABb[k];
          }
        }
        const double ozb = 0.5 / zb, oze = 0.5 / ze;
        e.oz = SWAP ? oze : ozb;
        e.oe = SWAP ? ozb : oze;
        e.oze = 0.5 * rzz;
        e.roz = SWAP ? zb * rzz : ze * rzz;
        e.roe = SWAP ? ze * rzz : zb * rzz;
        if (f32) eri_prec<float, LA, LB, LC, LD>(F, pref, e, out);
        else eri_prec<double, LA, LB, LC, LD>(F, pref, e, out);
      }
      n32 += (f32 && PASS == 0) ? 1u : 0u;
      // integral of the bra's components (a first, b second) and the ket's (c, d)
      auto E = [&](int a, int b, int cc, int d) -> double {
        return out[SWAP ? ((cc * M2 + d) * N1 + a) * N2 + b : ((a * N2 + b) * M1 + cc) * M2 + d];
      };
      if (helix) {
        const size_t cj = pp2 * ((size_t)(q3x + g.c2[0]) + (size_t)(2 * g.c2[0] + 1) * (q3x + q2[0] + h3));
#pragma unroll
        for (int t = 0; t < M1 * M2; ++t) {
          const int cc = t / M2, d = t % M2;
          const int kp = swk ? k2[d] : k1[cc], lp = swk ? k1[cc] : k2[d];
          dj[t] = (kp >= 0 && lp >= 0) ? __ldg(R.pph + kp + (size_t)npgs * lp + cj) : 0.0;
        }
      }
      // J: sum over the ket's components, accumulated over cells and kets
#pragma unroll
      for (int a = A0; a < A1; ++a)
#pragma unroll
        for (int b = 0; b < N2; ++b) {
          double acc = 0.0;
#pragma unroll
          for (int cc = 0; cc < M1; ++cc)
#pragma unroll
            for (int d = 0; d < M2; ++d) acc = fma(dj[cc * M2 + d], E(a, b, cc, d), acc);
          jacc[a * N2 + b] += acc;
        }
      // K: X(i,l,Q3+Q2) += sum_{j,k} D(k,j) (ij|kl)
      if (lcel) {
        const size_t ck = helix ? pp2 * ((size_t)(q3x + g.c2[0]) + (size_t)(2 * g.c2[0] + 1) * (q1[0] + h3))
                                : pp2 * cell1_index(g, q1[0] - q3x, q1[1] - q3y, q1[2] - q3z);
        const double* __restrict__ Dk = helix ? R.pph : R.pp;
        const size_t cx = pp2 * cell1_index(g, q3x + q2[0], q3y + q2[1], q3z + q2[2]);
        if (!swb && !swk) lat_k<N1, N2, M1, M2, SWAP, false, false, A0, A1>(out, b1, b2, k1, k2, Dk, ck, R.xp, cx, npgs);
        else if (!swb) lat_k<N1, N2, M1, M2, SWAP, false, true, A0, A1>(out, b1, b2, k1, k2, Dk, ck, R.xp, cx, npgs);
        else if (!swk) lat_k<N1, N2, M1, M2, SWAP, true, false, A0, A1>(out, b1, b2, k1, k2, Dk, ck, R.xp, cx, npgs);
        else lat_k<N1, N2, M1, M2, SWAP, true, true, A0, A1>(out, b1, b2, k1, k2, Dk, ck, R.xp, cx, npgs);
      }
    }
    // J of this chunk: reduce the lanes' sums, one atomic per bra component pair
    const size_t c1q1 = pp2 * cell1_index(g, q1[0], q1[1], q1[2]);
#pragma unroll
    for (int a = A0; a < A1; ++a)
#pragma unroll
      for (int b = 0; b < N2; ++b) {
        const double v = warp_sum(jacc[a * N2 + b]);
        const int ip = swb ? b2[b] : b1[a], jp = swb ? b1[a] : b2[b];
        if (lane == 0 && ip >= 0 && jp >= 0 && v != 0.0) atomicAdd(R.cp + ip + (size_t)npgs * jp + c1q1, v);
      }
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) n32 += __shfl_xor_sync(0xffffffffu, n32, o);
  if (lane == 0 && n32) atomicAdd(R.n32, n32);
}

template <int LA, int LB, int LC, int LD, bool SW>
void launch_sl(const LatticeRun& r, int grid, cudaStream_t s) {
  k_lat_sl<LA, LB, LC, LD, SW><<<grid, 128, 0, s>>>(r);
}

// The register passes of a class, one launch each on its own work-queue counter
// (r.queue + PASS: the lattice build zeroes kLatQueueSlots counters per class).
template <int LA, int LB, int LC, int LD, bool SW, int NPASS, int PASS = 0>
void launch_sl_passes(const LatticeRun& r, int grid, cudaStream_t s) {
  static_assert(NPASS <= kLatQueueSlots, "a counter per pass");
  LatticeRun rp = r;
  rp.queue = r.queue + PASS;
  k_lat_sl<LA, LB, LC, LD, SW, NPASS, PASS><<<grid, 128, 0, s>>>(rp);
  if constexpr (PASS + 1 < NPASS) launch_sl_passes<LA, LB, LC, LD, SW, NPASS, PASS + 1>(r, grid, s);
}

}  // namespace

int lattice_sl_passes(int e1, int e2) {
  if (!lattice_sl_launcher(e1, e2, false)) return 0;
  return (e1 == 2 && e2 == 2) ? 4 : 1;
}

// evaluated class (e1 >= e2) and swap flag -> straight-line launcher, or null
LatSlFn lattice_sl_launcher(int e1, int e2, bool sw) {
#define L2(A, B, C, D) (sw ? &launch_sl<A, B, C, D, true> : &launch_sl<A, B, C, D, false>)
  switch (e1 * 8 + e2) {
    case 0: return L2(0, 0, 0, 0);
    case 8: return L2(1, 0, 0, 0);
    case 9: return L2(1, 0, 1, 0);
    case 16: return L2(1, 1, 0, 0);
    case 17: return L2(1, 1, 1, 0);
    case 18: return sw ? &launch_sl_passes<1, 1, 1, 1, true, 4> : &launch_sl_passes<1, 1, 1, 1, false, 4>;
    case 24: return L2(2, 0, 0, 0);
    case 25: return L2(2, 0, 1, 0);
    case 32: return L2(2, 1, 0, 0);
    default: return nullptr;
  }
#undef L2
}

}  // namespace pfe
