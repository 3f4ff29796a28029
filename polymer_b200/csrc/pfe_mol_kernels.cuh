// Molecular quartet kernels shared by the FP64 and mixed-precision
// instantiations (pfe_mol.cu, pfe_mol_mixed.cu): the launch block, density
// bounds, the precision switch of the recursion, the digestion helpers and the
// straight-line group-quartet kernel with its pass launchers.
#pragma once

#include "pfe_common.cuh"
#include "pfe_context.cuh"
#include "generated/eri_classes.cuh"

namespace pfe {

// One shell pair as the quartet kernels read it, 128 bytes (seven 16-byte
// loads): P[3], PA[3], AB[3], zeta, S, Schwarz bound, (si, sj), 1/(2 zeta),
// padding.
struct __align__(16) PairRec {
  double P[3], PA[3], AB[3];
  double zeta, S, schwarz;
  int si, sj;
  double oz;
  double pad[2];
};
static_assert(sizeof(PairRec) == 128, "PairRec layout");

struct PairView {
  double P[3], PA[3], AB[3], zeta, S, oz, bound;
  int si, sj;
};

// the record of pair t with its Schwarz bound (the quartet loops load the whole
// record before screening on the bound: one load latency per pair, not two)
__device__ __forceinline__ PairView load_pair(const PairRec* __restrict__ rec, int t) {
  const double2* r = reinterpret_cast<const double2*>(rec + t);
  const double2 a = __ldg(r), b = __ldg(r + 1), c = __ldg(r + 2), d = __ldg(r + 3), e = __ldg(r + 4),
                f = __ldg(r + 5), g = __ldg(r + 6);
  PairView v;
  v.P[0] = a.x; v.P[1] = a.y; v.P[2] = b.x;
  v.PA[0] = b.y; v.PA[1] = c.x; v.PA[2] = c.y;
  v.AB[0] = d.x; v.AB[1] = d.y; v.AB[2] = e.x;
  v.zeta = e.y; v.S = f.x; v.bound = f.y;
  v.si = __double2loint(g.x); v.sj = __double2hiint(g.x);
  v.oz = g.y;
  return v;
}

__device__ __forceinline__ double pair_bound(const PairRec* __restrict__ rec, int t) {
  return __ldg(&rec[t].schwarz);
}

struct MolLaunch {
  PairArrays pairs;
  const PairRec* rec;     // the sorted pairs as records
  const int* prim;        // shell components -> primitive
  const int* stidx;       // shell x component -> target row (-1: none)
  const double* scoef;    // shell x component -> coefficient
  const double* boys;
  const double* dt;       // density in target space (nt x nt, column-major)
  double* jt;             // J' targets (nt x nt)
  double* kt;             // K' targets
  const int* gr_start;    // group -> first pair
  const int* gr_n;        // group -> number of pairs
  const double* gr_max;   // group -> largest bound
  const int* bk_list;     // ket groups by (class, bucket, group)
  const int* blk;         // shell -> contracted block
  const int* tblk;        // target -> contracted block (-1: none)
  const double* bmax;     // block-pair maxima of |P_T| (density screening / mixed precision)
  int nblk;
  double dtol;            // skip quartets with bound * max|P| < dtol (0: the reference's screen only)
  double mcut;            // FP32 recursion where bound * max|P| < mcut (0: FP64 only)
  unsigned long long* n32;  // quartets run in FP32
  const int4* chunks;     // (bra group, first list entry, end list entry, 0), costliest first
  const int* nchunks;
  int* queue;             // chunk counters (one per pass), zero at launch: warps take chunks in order
  double inttol;
  int nt;
  int myid, numprocs;
  const MolLaunch* insts;   // batches: the launch record of every instance (chunk .w), else null
  int lower_kept_bits;      // bit L: some shell of top L has a coefficient on a lower component
};

// The launch record of a set-up molecular context for target-space density d_dt.
MolLaunch molecular_launch(pfe_context* ctx, const double* d_dt);

// max|P_T| over the six density blocks a group quartet's digestion reads
__device__ __forceinline__ double quartet_pmax(const MolLaunch& ql, int I, int J, int K, int L) {
  const int bI = ql.blk[I], bJ = ql.blk[J], bK = ql.blk[K], bL = ql.blk[L], nb = ql.nblk;
  const double* bm = ql.bmax;
  return fmax(fmax(fmax(bm[bI * nb + bJ], bm[bK * nb + bL]), fmax(bm[bI * nb + bK], bm[bI * nb + bL])),
              fmax(bm[bJ * nb + bK], bm[bJ * nb + bL]));
}

// Screening threshold on Schwarz(ij)*Schwarz(kl) of a group quartet: the
// reference's INTTOL, raised to dtol/max|P| under density screening.
__device__ __forceinline__ double quartet_threshold(const MolLaunch& ql, double pmax) {
  if (ql.dtol <= 0.0) return ql.inttol;
  return pmax > 0.0 ? fmax(ql.inttol, ql.dtol / pmax) : INFINITY;
}

// Primitive-quartet integrals in FP64, or in FP32 from Boys values and geometry
// computed in FP64 (the recursion is linear in F: it runs on F/pref, and the
// outputs are scaled by pref in FP64, so FP32 sees values of order one).
template <typename R, int LA, int LB, int LC, int LD>
__device__ __forceinline__ void eri_prec(const double* F, double pref, const EriGeom<double>& g, double* out) {
  constexpr int NI = ncum(LA) * ncum(LB) * ncum(LC) * ncum(LD);
  constexpr int LT = LA + LB + LC + LD;
  if constexpr (sizeof(R) == sizeof(double)) {
    eri_dispatch<LA, LB, LC, LD>(F, g, out);
  } else {
    float Ff[LT + 1];
#pragma unroll
    for (int m = 0; m <= LT; ++m) Ff[m] = (float)F[m];
    EriGeom<float> gf;
#pragma unroll
    for (int k = 0; k < 3; ++k) {
      gf.PA[k] = (float)g.PA[k]; gf.WP[k] = (float)g.WP[k]; gf.QC[k] = (float)g.QC[k];
      gf.WQ[k] = (float)g.WQ[k]; gf.AB[k] = (float)g.AB[k]; gf.CD[k] = (float)g.CD[k];
    }
    gf.oz = (float)g.oz; gf.oe = (float)g.oe; gf.oze = (float)g.oze; gf.roz = (float)g.roz; gf.roe = (float)g.roe;
    float of[NI];
    eri_dispatch<LA, LB, LC, LD>(Ff, gf, of);
#pragma unroll
    for (int i = 0; i < NI; ++i) out[i] = pref * (double)of[i];
  }
}

// ------------------------------------------------------------------ digestion helpers

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

__device__ __forceinline__ void add_target(double* __restrict__ M, int nt, int r, int c, double v) {
  if (r >= 0 && c >= 0 && v != 0.0) atomicAdd(M + r + (size_t)nt * c, v);
}

__device__ __forceinline__ double dt_at(const double* __restrict__ D, int nt, int i, int j) {
  return (i >= 0 && j >= 0) ? __ldg(D + i + (size_t)nt * j) : 0.0;
}

// ------------------------------------------------------------------ straight-line classes

// One group quartet per lane: the warp shares the bra group, each lane owns one
// ket group of the chunk.  X(abcd) of the lane's group quartet stays in
// registers; the bra's primitive pairs are walked in step by the whole warp.
// Classes with more integrals than registers hold X in NPASS launches, pass
// PASS keeping the bra components ab in [AB0, AB1) (the recursion is repeated
// per pass; the outputs a pass does not keep are dead code in it).
// Angular momentum of component i of a cumulative shell, in the reference's
// component order (x power outer, z power inner: s, z, zz, y, yz, yy, x, xz, xy, xx).
__host__ __device__ constexpr int comp_tot(int L, int i) {
  return L == 0 ? 0 : (L == 1 ? (i == 0 ? 0 : 1) : (i == 0 ? 0 : (i == 1 || i == 3 || i == 6) ? 1 : 2));
}

// Bra component pairs ab = a*NB + b ordered by (|a|, |b|): the passes of a
// class then keep the lower (for pure shells coefficient-free) components
// together, and such passes skip their chunks.
__host__ __device__ constexpr void ab_order_fill(int LA, int LB, int* ab, int* pos) {
  const int NB = ncum(LB), N = ncum(LA) * NB;
  for (int i = 0; i < N; ++i) ab[i] = i;
  for (int i = 1; i < N; ++i)   // stable insertion sort by (|a|, |b|)
    for (int j = i; j > 0; --j) {
      const int x = ab[j - 1], y = ab[j];
      const int kx = comp_tot(LA, x / NB) * 8 + comp_tot(LB, x % NB);
      const int ky = comp_tot(LA, y / NB) * 8 + comp_tot(LB, y % NB);
      if (kx <= ky) break;
      ab[j - 1] = y;
      ab[j] = x;
    }
  for (int i = 0; i < N; ++i) pos[ab[i]] = i;
}

template <int LA, int LB>
struct AbOrder {
  static constexpr int NA = ncum(LA), NB = ncum(LB), N = NA * NB;
  int ab[N];    // k-th pair
  int pos[N];   // position of pair ab
  __host__ __device__ constexpr AbOrder() : ab(), pos() { ab_order_fill(LA, LB, ab, pos); }
};

// Bra component pairs below the top level (|a| < LA or |b| < LB): in AbOrder
// they come first.
__host__ __device__ constexpr int lower_pairs(int LA, int LB) {
  int c = 0;
  for (int a = 0; a < ncum(LA); ++a)
    for (int b = 0; b < ncum(LB); ++b)
      if (comp_tot(LA, a) < LA || comp_tot(LB, b) < LB) ++c;
  return c;
}

template <int LA, int LB>
struct LowerPairs {
  static constexpr int n = lower_pairs(LA, LB);
};

// The bra component pairs [ab0, ab1) (positions in AbOrder) register pass `pass`
// of `npass` keeps.  Two-pass (d s| classes split at the level boundary: the
// lower components of the d shell first, the top-level ones second, so that a
// pure d shell (lower components coefficient-free) skips the first pass entirely.
__host__ __device__ constexpr void pass_range(int LA, int LB, int LC, int LD, int npass, int pass, int& ab0, int& ab1) {
  const int NAB = ncum(LA) * ncum(LB), NCD = ncum(LC) * ncum(LD);
  const int abp = (NAB + npass - 1) / npass;
  const int nlow = lower_pairs(LA, LB);
  const bool lsplit = npass == 2 && LA == 2 && LB == 0 && nlow * NCD <= 40 && (NAB - nlow) * NCD <= 40;
  ab0 = lsplit ? (pass == 0 ? 0 : nlow) : pass * abp;
  ab1 = lsplit ? (pass == 0 ? nlow : NAB) : ((ab0 + abp < NAB) ? ab0 + abp : NAB);
}

// Whether register pass `pass` keeps a bra component pair that can carry a
// coefficient: a component below its shell's top level has none unless bit L of
// lower_kept_bits is set (the kernel skips such chunks anyway; a pass that keeps
// none of them is not launched at all).
inline bool pass_live(int LA, int LB, int LC, int LD, int npass, int pass, int lower_kept_bits) {
  int ab[MAXCOMP * MAXCOMP] = {}, pos[MAXCOMP * MAXCOMP] = {};
  ab_order_fill(LA, LB, ab, pos);
  int ab0 = 0, ab1 = 0;
  pass_range(LA, LB, LC, LD, npass, pass, ab0, ab1);
  const int NB = ncum(LB);
  for (int k = ab0; k < ab1; ++k) {
    const int a = ab[k] / NB, b = ab[k] % NB;
    const bool ka = comp_tot(LA, a) == LA || ((lower_kept_bits >> LA) & 1);
    const bool kb = comp_tot(LB, b) == LB || ((lower_kept_bits >> LB) & 1);
    if (ka && kb) return true;
  }
  return false;
}

// resident blocks of 128 threads the register allocation aims at: 4 (at most
// 128 registers) for the classes whose working set fits, else the compiler's choice
template <int LA, int LB, int LC, int LD>
struct GqOccupancy {
  static constexpr int NI = ncum(LA) * ncum(LB) * ncum(LC) * ncum(LD);
#ifdef PFE_GQ_MINB
  static constexpr int blocks = (NI <= 16 && LA + LB + LC + LD <= 2) ? 4 : PFE_GQ_MINB;
#else
  static constexpr int blocks = (NI <= 16 && LA + LB + LC + LD <= 2) ? 4 : 1;
#endif
};

template <int LT>
struct GqSmemBoys {
#ifdef PFE_GQ_SMEM_BOYS
  static constexpr bool use = BoysSmem<LT>::use;
#else
  static constexpr bool use = false;
#endif
};

// Classes of total angular momentum up to maxl evaluate the Boys function without
// the table (boys_direct): their lanes' per-quartet table-row gathers were half of
// their L1 wavefronts.  Measured on the 32-cluster water batch: (10|00) 55.8 ->
// 53.0 ms (long-scoreboard stalls halved, instructions +60 % for erf and exp), the
// batched build 295.8 -> 287.5 ms; C20H42 unchanged.  The lattice kernels keep the
// table (their classes ran 12 % slower on it: they already spend the FP64 pipe on
// the screw rotations of every image cell).
struct GqBoysDirect {
#ifdef PFE_BOYS_DIRECT_MAXL
  static constexpr int maxl = PFE_BOYS_DIRECT_MAXL;
#else
  static constexpr int maxl = 2;
#endif
};

template <int LA, int LB, int LC, int LD, int NPASS, int PASS, bool MIXED, bool BATCH>
__global__ void __launch_bounds__(128, GqOccupancy<LA, LB, LC, LD>::blocks) k_gq(MolLaunch lq) {
  constexpr int NA = ncum(LA), NB = ncum(LB), NC = ncum(LC), ND = ncum(LD);
  constexpr int NI = NA * NB * NC * ND;
  constexpr int NAB = NA * NB;
  constexpr int NCD = NC * ND;
  constexpr int LT = LA + LB + LC + LD;
  constexpr AbOrder<LA, LB> ORD{};
  constexpr int AB0 = [] { int a = 0, b = 0; pass_range(LA, LB, LC, LD, NPASS, PASS, a, b); return a; }();
  constexpr int AB1 = [] { int a = 0, b = 0; pass_range(LA, LB, LC, LD, NPASS, PASS, a, b); return b; }();
  constexpr int XN = (AB1 - AB0) * NCD;
  static_assert(AB0 < NAB, "every pass keeps at least one bra component pair");
  // the pass keeps the pairs ab at positions [AB0, AB1) of ORD; X(k, cd) is pair ORD.ab[AB0 + k]
  auto in_pass = [&](int a, int b) { const int k = ORD.pos[a * NB + b]; return k >= AB0 && k < AB1; };
  auto xi = [&](int a, int b, int cc, int d) { return (ORD.pos[a * NB + b] - AB0) * NCD + cc * ND + d; };
  const int lane = threadIdx.x & 31;
  const int nchunks = *lq.nchunks;
  const double c2pi = 2.0 / sqrt(REF_PI);
  // with PFE_GQ_SMEM_BOYS, classes of total angular momentum up to 4 read their
  // Boys rows from a copy of the table's first rows in shared memory (the launch
  // passes its size); off by default: measured on C20H42 it cost 10-16 % on the
  // low classes (fewer resident blocks, the per-block copy), the L1-cached
  // gathers of the global table are as fast
  constexpr bool SBOYS = GqSmemBoys<LT>::use;
  extern __shared__ double s_boys[];
  if constexpr (SBOYS) {
    boys_stage<LT>(lq.boys, s_boys);
    __syncthreads();
  }
  // the warp takes the next chunk of this rank's share (every numprocs-th,
  // starting at myid) from the pass's work queue: chunks are sorted costliest
  // first, so the launch ends with the cheap ones
  for (;;) {
    int t = 0;
    if (lane == 0) t = atomicAdd(lq.queue + PASS, 1);
    const int c = __shfl_sync(0xffffffffu, t, 0) * lq.numprocs + lq.myid;
    if (c >= nchunks) break;
    const int4 ch = lq.chunks[c];
    // this chunk's instance: batches read its launch record from global memory
    const MolLaunch& ql = [&]() -> const MolLaunch& {
      if constexpr (BATCH) return lq.insts[ch.w];
      else return lq;
    }();
    // the tables the loops read, held in registers (ql may live in global memory)
    const PairRec* __restrict__ rec = ql.rec;
    const double* __restrict__ scoef = ql.scoef;
    const double* __restrict__ boys = ql.boys;
    const int* __restrict__ stidx = ql.stidx;
    const double mcut = ql.mcut;
    const int nt = ql.nt;
    const int G = ch.x;
    const int g0 = ql.gr_start[G], gn = ql.gr_n[G];
    const int2 ijg = __ldg(reinterpret_cast<const int2*>(&rec[g0].si));
    if constexpr (NPASS > 1) {
      // a pass whose bra components all lack a coefficient (the lower components of a
      // pure d or p shell) contributes nothing: skip the chunk (warp-uniform)
      bool live = false;
#pragma unroll
      for (int k = AB0; k < AB1; ++k)
        live = live || (stidx[ijg.x * MAXCOMP + ORD.ab[k] / NB] >= 0 && stidx[ijg.y * MAXCOMP + ORD.ab[k] % NB] >= 0);
      if (!live) continue;
    }
    const int li = ch.y + lane;
    const bool act = li < ch.z;
    const int H = ql.bk_list[act ? li : ch.y];
    const int h0 = ql.gr_start[H], hn = act ? ql.gr_n[H] : 0;
    const bool dens = ql.dtol > 0.0 || ql.mcut > 0.0;
    const int2 klh = __ldg(reinterpret_cast<const int2*>(&rec[h0].si));
    const double pmax = dens ? quartet_pmax(ql, ijg.x, ijg.y, klh.x, klh.y) : 0.0;
    const double thr = quartet_threshold(ql, pmax);
    unsigned n32 = 0;
    bool any = false;   // this lane evaluated a quartet
    double X[XN];
#pragma unroll
    for (int i = 0; i < XN; ++i) X[i] = 0.0;
    const double gmax = ql.gr_max[G];
    // Each lane walks its own ket group's pairs (outer loop, one gather of the ket
    // record per pair); the warp walks the bra group's pairs in step (inner loop:
    // every lane reads the same bra record, one L1 wavefront per load).  Both
    // lists are sorted by Schwarz bound, so the screens end the loops.
    for (int qi = 0;; ++qi) {
      const bool lv = qi < hn;
      const int q = h0 + (lv ? qi : 0);
      const PairView kq = load_pair(rec, q);
      const double sq = lv ? kq.bound : 0.0;
      const bool qok = lv && sq * gmax >= thr;
      if (!__any_sync(0xffffffffu, qok)) break;
      const double ze = kq.zeta;
      const double Qx = kq.P[0], Qy = kq.P[1], Qz = kq.P[2];
      const double Sq = kq.S;
      const int K = kq.si, L = kq.sj;
      const double wKL = (K != L) ? 2.0 : 1.0;
      // ket coefficients: products held when small, factors otherwise
      constexpr bool HOLD = NCD <= 16;
      double ccd[HOLD ? NCD : 1];
      double sK[NC], sL[ND];
#pragma unroll
      for (int cc = 0; cc < NC; ++cc) sK[cc] = scoef[K * MAXCOMP + cc];
#pragma unroll
      for (int d = 0; d < ND; ++d) sL[d] = scoef[L * MAXCOMP + d];
      if constexpr (HOLD) {
#pragma unroll
        for (int cc = 0; cc < NC; ++cc)
#pragma unroll
          for (int d = 0; d < ND; ++d) ccd[cc * ND + d] = wKL * sK[cc] * sL[d];
      }
      for (int p = g0; p < g0 + gn; ++p) {
        const PairView bp = load_pair(rec, p);
        const double sp = bp.bound;
        const bool pass = qok && sp * sq >= thr;
        if (!__any_sync(0xffffffffu, pass)) break;   // later bra pairs fail for every lane
        // a group paired with itself: each unordered pair of pairs once (p >= q)
        if (!pass || (G == H && p < q)) continue;
        const int I = bp.si, J = bp.sj;
        const double zb = bp.zeta;
        const double Px = bp.P[0], Py = bp.P[1], Pz = bp.P[2];
        const double zz = zb + ze;
        // one reciprocal per primitive quartet; 1/(2 zeta) of either pair comes with its record
        const double rzz = 1.0 / zz;
        const double rho = zb * ze * rzz;
        const double dx = Px - Qx, dy = Py - Qy, dz = Pz - Qz;
        const double T = rho * (dx * dx + dy * dy + dz * dz);
        const double pref = c2pi * bp.S * Sq * sqrt(rho);
        // FP32 only when every lane running this step qualifies
        bool f32 = false;
        if constexpr (MIXED && LT > 0) f32 = __all_sync(__activemask(), sp * sq * pmax < mcut);
        n32 += f32 ? 1u : 0u;
        double F[LT + 1];
        if constexpr (LT <= GqBoysDirect::maxl) boys_direct<LT>(T, f32 ? 1.0 : pref, F);
        else if constexpr (SBOYS) boys_tab_smem<LT>(T, f32 ? 1.0 : pref, s_boys, F);
        else boys_tab<LT>(T, f32 ? 1.0 : pref, boys, F);
        double out[NI];
        if constexpr (LT == 0) {
          out[0] = F[0];
        } else {
          EriGeom<double> g;
          const double Wx = (zb * Px + ze * Qx) * rzz, Wy = (zb * Py + ze * Qy) * rzz, Wz = (zb * Pz + ze * Qz) * rzz;
          g.PA[0] = bp.PA[0]; g.PA[1] = bp.PA[1]; g.PA[2] = bp.PA[2];
          g.QC[0] = kq.PA[0]; g.QC[1] = kq.PA[1]; g.QC[2] = kq.PA[2];
          g.AB[0] = bp.AB[0]; g.AB[1] = bp.AB[1]; g.AB[2] = bp.AB[2];
          g.CD[0] = kq.AB[0]; g.CD[1] = kq.AB[1]; g.CD[2] = kq.AB[2];
          g.WP[0] = Wx - Px; g.WP[1] = Wy - Py; g.WP[2] = Wz - Pz;
          g.WQ[0] = Wx - Qx; g.WQ[1] = Wy - Qy; g.WQ[2] = Wz - Qz;
          g.oz = bp.oz; g.oe = kq.oz; g.oze = 0.5 * rzz; g.roz = ze * rzz; g.roe = zb * rzz;
          if constexpr (MIXED) {
            if (f32) eri_prec<float, LA, LB, LC, LD>(F, pref, g, out);
            else eri_prec<double, LA, LB, LC, LD>(F, pref, g, out);
          } else {
            eri_prec<double, LA, LB, LC, LD>(F, pref, g, out);
          }
        }
        any = true;
        const double w = ((I != J) ? 2.0 : 1.0) * ((p != q) ? 2.0 : 1.0);
#pragma unroll
        for (int k = AB0; k < AB1; ++k) {
          const double ca = w * scoef[I * MAXCOMP + ORD.ab[k] / NB] * scoef[J * MAXCOMP + ORD.ab[k] % NB];
#pragma unroll
          for (int cc = 0; cc < NC; ++cc) {
            double cb;
            if constexpr (HOLD) cb = ca;
            else cb = ca * (wKL * sK[cc]);
#pragma unroll
            for (int d = 0; d < ND; ++d) {
              const double c4 = HOLD ? cb * ccd[cc * ND + d] : cb * sL[d];
              X[(k - AB0) * NCD + cc * ND + d] = fma(c4, out[ORD.ab[k] * NCD + cc * ND + d], X[(k - AB0) * NCD + cc * ND + d]);
            }
          }
        }
      }
    }
    if (MIXED && PASS == 0) {
      unsigned long long n = n32;
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) n += __shfl_xor_sync(0xffffffffu, n, o);
      if (lane == 0 && n) atomicAdd(ql.n32, n);
    }
    // digestion of this pass's part of X against the target-space density
    if (!__any_sync(0xffffffffu, any)) continue;   // nothing passed the screens in this chunk
    const double* __restrict__ D = ql.dt;
    const int I0 = ijg.x, J0 = ijg.y, K0 = klh.x, L0 = klh.y;
    int ta[NA], tb[NB], tc[NC], td[ND];
#pragma unroll
    for (int x = 0; x < NA; ++x) ta[x] = stidx[I0 * MAXCOMP + x];
#pragma unroll
    for (int x = 0; x < NB; ++x) tb[x] = stidx[J0 * MAXCOMP + x];
#pragma unroll
    for (int x = 0; x < NC; ++x) tc[x] = stidx[K0 * MAXCOMP + x];
#pragma unroll
    for (int x = 0; x < ND; ++x) td[x] = stidx[L0 * MAXCOMP + x];
    // J'(ab) += 1/4 sum_cd P(cd) X: the bra is the warp's, reduce over lanes first
#pragma unroll
    for (int k = AB0; k < AB1; ++k) {
      double v = 0.0;
#pragma unroll
      for (int cc = 0; cc < NC; ++cc)
#pragma unroll
        for (int d = 0; d < ND; ++d) v = fma(dt_at(D, nt, tc[cc], td[d]), X[(k - AB0) * NCD + cc * ND + d], v);
      v = warp_sum(v);
      if (lane == 0) add_target(ql.jt, nt, ta[ORD.ab[k] / NB], tb[ORD.ab[k] % NB], 0.25 * v);
    }
    if (act && any) {
      // J'(cd) += 1/4 sum_ab P(ab) X
      double Pab[NAB];
#pragma unroll
      for (int k = AB0; k < AB1; ++k) Pab[ORD.ab[k]] = dt_at(D, nt, ta[ORD.ab[k] / NB], tb[ORD.ab[k] % NB]);
#pragma unroll
      for (int cd = 0; cd < NCD; ++cd) {
        double v = 0.0;
#pragma unroll
        for (int k = AB0; k < AB1; ++k) v = fma(Pab[ORD.ab[k]], X[(k - AB0) * NCD + cd], v);
        add_target(ql.jt, nt, tc[cd / ND], td[cd % ND], 0.25 * v);
      }
      // K'(ad) += 1/8 P(bc) X ; K'(ac) += 1/8 P(bd) X   (in_pass folds at compile time)
#pragma unroll
      for (int a = 0; a < NA; ++a) {
        bool a_in = false;
#pragma unroll
        for (int b = 0; b < NB; ++b) a_in = a_in || in_pass(a, b);
        if (!a_in) continue;
#pragma unroll
        for (int d = 0; d < ND; ++d) {
          double v = 0.0;
#pragma unroll
          for (int b = 0; b < NB; ++b)
            if (in_pass(a, b))
#pragma unroll
              for (int cc = 0; cc < NC; ++cc) v = fma(dt_at(D, nt, tb[b], tc[cc]), X[xi(a, b, cc, d)], v);
          add_target(ql.kt, nt, ta[a], td[d], 0.125 * v);
        }
#pragma unroll
        for (int cc = 0; cc < NC; ++cc) {
          double v = 0.0;
#pragma unroll
          for (int b = 0; b < NB; ++b)
            if (in_pass(a, b))
#pragma unroll
              for (int d = 0; d < ND; ++d) v = fma(dt_at(D, nt, tb[b], td[d]), X[xi(a, b, cc, d)], v);
          add_target(ql.kt, nt, ta[a], tc[cc], 0.125 * v);
        }
      }
      // K'(bd) += 1/8 P(ac) X ; K'(bc) += 1/8 P(ad) X
#pragma unroll
      for (int b = 0; b < NB; ++b) {
        bool b_in = false;
#pragma unroll
        for (int a = 0; a < NA; ++a) b_in = b_in || in_pass(a, b);
        if (!b_in) continue;
#pragma unroll
        for (int d = 0; d < ND; ++d) {
          double v = 0.0;
#pragma unroll
          for (int a = 0; a < NA; ++a)
            if (in_pass(a, b))
#pragma unroll
              for (int cc = 0; cc < NC; ++cc) v = fma(dt_at(D, nt, ta[a], tc[cc]), X[xi(a, b, cc, d)], v);
          add_target(ql.kt, nt, tb[b], td[d], 0.125 * v);
        }
#pragma unroll
        for (int cc = 0; cc < NC; ++cc) {
          double v = 0.0;
#pragma unroll
          for (int a = 0; a < NA; ++a)
            if (in_pass(a, b))
#pragma unroll
              for (int d = 0; d < ND; ++d) v = fma(dt_at(D, nt, ta[a], td[d]), X[xi(a, b, cc, d)], v);
          add_target(ql.kt, nt, tb[b], tc[cc], 0.125 * v);
        }
      }
    }
  }
}

// ------------------------------------------------------------------ launch tables

using LaunchFn = void (*)(const MolLaunch&, int grid, cudaStream_t);

template <int LA, int LB, int LC, int LD, int NPASS, int PASS, bool MIXED, bool BATCH>
struct Passes {
  static void run(const MolLaunch& ql, int grid, cudaStream_t s) {
    if (NPASS > 1 && !pass_live(LA, LB, LC, LD, NPASS, PASS, ql.lower_kept_bits)) {
      if constexpr (PASS + 1 < NPASS) Passes<LA, LB, LC, LD, NPASS, PASS + 1, MIXED, BATCH>::run(ql, grid, s);
      return;
    }
    constexpr int LT = LA + LB + LC + LD;
    auto kern = k_gq<LA, LB, LC, LD, NPASS, PASS, MIXED, BATCH>;
    if constexpr (GqSmemBoys<LT>::use) {
      // the staged Boys rows: allow them once, and launch no more blocks than can be
      // resident (each block copies the rows once; the work queue spreads the chunks)
      static int resident = 0;
      if (resident == 0) {
        cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)BoysSmem<LT>::BYTES);
        int per_sm = 0, dev = 0, nsm = 0;
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, 128, BoysSmem<LT>::BYTES);
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
        resident = std::max(1, per_sm) * std::max(1, nsm);
      }
      kern<<<std::min(grid, resident), 128, BoysSmem<LT>::BYTES, s>>>(ql);
    } else {
      kern<<<grid, 128, 0, s>>>(ql);
    }
    if constexpr (PASS + 1 < NPASS) Passes<LA, LB, LC, LD, NPASS, PASS + 1, MIXED, BATCH>::run(ql, grid, s);
  }
};

template <int LA, int LB, int LC, int LD, int NPASS, bool MIXED, bool BATCH = false>
void launch_q(const MolLaunch& ql, int grid, cudaStream_t s) {
  Passes<LA, LB, LC, LD, NPASS, 0, MIXED, BATCH>::run(ql, grid, s);
}

// Launches per straight-line class (its passes); must match the table below.
static inline int straight_npass(int cb, int ck) {
  static const int np[6][6] = {{1, 0, 0, 0, 0, 0}, {1, 1, 0, 0, 0, 0}, {1, 2, 8, 0, 0, 0},
                               {2, 2, 5, 3, 0, 0}, {1, 4, 14, 10, 40, 0}, {3, 10, 50, 25, 0, 0}};
  return np[cb][ck];
}

// straight-line classes and their passes (X of at most 40 integrals per pass)
template <bool MIXED, bool BATCH = false>
static LaunchFn straight_launcher_t(int cb, int ck) {
#define Q(A, B, C, D, P) &launch_q<A, B, C, D, P, MIXED, BATCH>
  static const LaunchFn table[6][6] = {
      {Q(0, 0, 0, 0, 1), nullptr, nullptr, nullptr, nullptr, nullptr},
      {Q(1, 0, 0, 0, 1), Q(1, 0, 1, 0, 1), nullptr, nullptr, nullptr, nullptr},
      {Q(1, 1, 0, 0, 1), Q(1, 1, 1, 0, 2), Q(1, 1, 1, 1, 8), nullptr, nullptr, nullptr},
      {Q(2, 0, 0, 0, 2), Q(2, 0, 1, 0, 2), Q(2, 0, 1, 1, 5), Q(2, 0, 2, 0, 3), nullptr, nullptr},
      {Q(2, 1, 0, 0, 1), Q(2, 1, 1, 0, 4), nullptr, nullptr, nullptr, nullptr},
      {Q(2, 2, 0, 0, 3), nullptr, nullptr, nullptr, nullptr, nullptr}};
#undef Q
  return table[cb][ck];
}

// The large classes' FP64 passes, one translation unit each (pfe_mol_big*.cu)
// so that they compile in parallel; `batch`: the instantiations for batches.
LaunchFn straight_launcher_big(int cb, int ck, bool batch = false);

}  // namespace pfe
