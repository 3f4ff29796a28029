// Warp-per-primitive-quartet kernel for the large molecular quartet classes
// ((dd|dp), (dd|dd) and the other classes with hundreds of integrals), the
// "wide" execution variant.
//
// One warp owns a chunk (a bra group and its ket groups) and walks the group
// quartets one at a time.  For each primitive quartet every lane evaluates the
// Boys values and the geometry itself (no serial step, no block barrier), then
// the 32 lanes run the class's level-scheduled op table in shared memory with a
// warp barrier per level.  Only the components that carry a coefficient (a
// target row) are kept: pure d and p shells keep their top-level components,
// so the op table is the pure-bra (or pure bra-and-ket) one and X(abcd) of the
// group quartet holds just the kept outputs, compactly.  X is digested once per
// group quartet against the target-space density with FP64 atomics, exactly as
// the other variants do (J'(ab), J'(cd), K'(ad), K'(bd), K'(ac), K'(bc) with
// the 8-fold symmetry weights).

#include <algorithm>

#include "pfe_common.cuh"
#include "pfe_context.cuh"
#include "pfe_interp.cuh"
#include "pfe_mol_kernels.cuh"
#include "pfe_mol_wide.cuh"

namespace pfe {

namespace {

template <int NA, int NB, int NC, int ND>
struct WideLayout {
  static constexpr int NS = NA + NB + NC + ND;
  // density blocks of the kept components, at fixed offsets: Pab | Pcd | Pac | Pad | Pbc | Pbd
  static constexpr int OAB = 0, OCD = NA * NB, OAC = OCD + NC * ND, OAD = OAC + NA * NC, OBC = OAD + NA * ND,
                       OBD = OBC + NB * NC, NP = OBD + NB * ND;
  static constexpr int GEO = (int)((sizeof(OpGeom) + 7) / 8);
  static constexpr int INTS = 2 * NS + 8;   // kept components, their target rows, counts and flags
  // doubles of one warp: v[vmax] | X[xmax] | xs[xmax] (int) | P | cab | ccd | geo | ints
  static __host__ __device__ int doubles(int vmax, int xmax) {
    return vmax + xmax + (xmax + 1) / 2 + NP + NA * NB + NC * ND + GEO + (INTS + 1) / 2;
  }
};

// Kept components of shell s (those with a target row) into k[], their rows
// into t[]; returns the count and whether all of them are top-level.
template <int L>
__device__ __forceinline__ int kept_components(const int* __restrict__ stidx, int s, int* k, int* t, bool* top) {
  int n = 0;
  bool all_top = true;
#pragma unroll
  for (int x = 0; x < ncum(L); ++x) {
    const int r = stidx[s * MAXCOMP + x];
    if (r >= 0) {
      k[n] = x;
      t[n] = r;
      ++n;
      if (comp_tot(L, x) < L) all_top = false;
    }
  }
  *top = all_top;
  return n;
}

template <int LA, int LB, int LC, int LD>
__global__ void __launch_bounds__(256) k_gq_wide(MolLaunch lq, OpTableDev tab, int per_warp, int vmax, int xmax) {
  constexpr int NA = ncum(LA), NB = ncum(LB), NC = ncum(LC), ND = ncum(LD);
  constexpr int LT = LA + LB + LC + LD;
  using W = WideLayout<NA, NB, NC, ND>;
  extern __shared__ double smem[];
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  double* v = smem + (size_t)wid * per_warp;
  double* X = v + vmax;
  int* xs = reinterpret_cast<int*>(X + xmax);
  double* P = X + xmax + (xmax + 1) / 2;
  double* cab = P + W::NP;
  double* ccd = cab + NA * NB;
  OpGeom& geo = *reinterpret_cast<OpGeom*>(ccd + NC * ND);
  int* im = reinterpret_cast<int*>(ccd + NC * ND + W::GEO);
  int* kA = im;
  int* kB = kA + NA;
  int* kC = kB + NB;
  int* kD = kC + NC;
  int* tA = im + W::NS;
  int* tB = tA + NA;
  int* tC = tB + NB;
  int* tD = tC + NC;
  int* meta = im + 2 * W::NS;   // na, nb, nc, nd, bra top-level only, ket top-level only
  if (lane == 0) {
    v[0] = 0.0;
    for (int k = 0; k < 3; ++k) { geo.G1[2][k] = 1.0; geo.G1[3][k] = 1.0; }
    geo.X[2] = geo.X[3] = 0.0;
    geo.Y[2] = geo.Y[3] = 0.0;
  }
  __syncwarp();
  const double c2pi = 2.0 / sqrt(REF_PI);
  const int nchunks = *lq.nchunks;
  for (;;) {   // chunks from the launch's work queue, costliest first
    int tk = 0;
    if (lane == 0) tk = atomicAdd(lq.queue, 1);
    const int c = __shfl_sync(0xffffffffu, tk, 0) * lq.numprocs + lq.myid;
    if (c >= nchunks) break;
    const int4 ch = lq.chunks[c];
    const MolLaunch& ql = lq.insts ? lq.insts[ch.w] : lq;
    const PairRec* __restrict__ rec = ql.rec;
    const double* __restrict__ scoef = ql.scoef;
    const double* __restrict__ boys = ql.boys;
    const double* __restrict__ D = ql.dt;
    const int nt = ql.nt;
    const int G = ch.x;
    const int g0 = ql.gr_start[G], gn = ql.gr_n[G];
    const double gmax = ql.gr_max[G];
    const int2 ij0 = __ldg(reinterpret_cast<const int2*>(&rec[g0].si));
    if (lane == 0) {
      bool ta, tb;
      meta[0] = kept_components<LA>(ql.stidx, ij0.x, kA, tA, &ta);
      meta[1] = kept_components<LB>(ql.stidx, ij0.y, kB, tB, &tb);
      meta[4] = (ta && tb) ? 1 : 0;
    }
    __syncwarp();
    const int na = meta[0], nb = meta[1];
    const int nab = na * nb;
    const bool bra_top = meta[4] != 0 && tab.ops_p != nullptr;
    for (int t = lane; t < nab; t += 32) P[W::OAB + t] = dt_at(D, nt, tA[t / nb], tB[t % nb]);
    for (int k = ch.y; k < ch.z; ++k) {
      const int H = ql.bk_list[k];
      const int h0 = ql.gr_start[H], hn = ql.gr_n[H];
      const double hmax = ql.gr_max[H];
      const int2 kl0 = __ldg(reinterpret_cast<const int2*>(&rec[h0].si));
      const double thr =
          quartet_threshold(ql, ql.dtol > 0.0 ? quartet_pmax(ql, ij0.x, ij0.y, kl0.x, kl0.y) : 0.0);
      if (gmax * hmax < thr) continue;   // no primitive quartet of (G|H) passes (warp-uniform)
      __syncwarp();                      // the previous group quartet's digestion read meta and X
      if (lane == 0) {
        bool tc, td;
        meta[2] = kept_components<LC>(ql.stidx, kl0.x, kC, tC, &tc);
        meta[3] = kept_components<LD>(ql.stidx, kl0.y, kD, tD, &td);
        meta[5] = (tc && td) ? 1 : 0;
      }
      __syncwarp();
      const int nc = meta[2], nd = meta[3];
      const int ncd = nc * nd, nx = nab * ncd;
      // the op table: pure bra and ket, pure bra, or the full one
      const bool two = bra_top && meta[5] != 0 && tab.ops_p2 != nullptr;
      const unsigned short* __restrict__ ops = two ? tab.ops_p2 : (bra_top ? tab.ops_p : tab.ops);
      const int* __restrict__ levels = two ? tab.levels_p2 : (bra_top ? tab.levels_p : tab.levels);
      const unsigned short* __restrict__ outs = two ? tab.out_p2 : (bra_top ? tab.out_p : tab.out);
      const int nlev = two ? tab.nlevels_p2 : (bra_top ? tab.nlevels_p : tab.nlevels);
      const int tslots = two ? tab.nslots_p2 : (bra_top ? tab.nslots_p : tab.nslots);
      if (nx > xmax || tslots > vmax) {
        // the host sized the working set for every table and kept-component count
        // of this molecule; anything else is refused loudly in the result
        if (lane == 0) atomicAdd(ql.jt, __longlong_as_double(0x7ff8000000000000ll));
        continue;
      }
      // kept outputs: slot of the table | ab << 15 | cd << 22 (ab, cd < 100)
      for (int i = lane; i < nx; i += 32) {
        const int ab = i / ncd, cd = i - ab * ncd;
        const int ia = ab / nb, ib = ab - ia * nb, ic = cd / nd, id = cd - ic * nd;
        const int full = ((kA[ia] * NB + kB[ib]) * NC + kC[ic]) * ND + kD[id];
        xs[i] = (int)outs[full] | (ab << 15) | (cd << 22);
        X[i] = 0.0;
      }
      for (int t = lane; t < ncd; t += 32) P[W::OCD + t] = dt_at(D, nt, tC[t / nd], tD[t % nd]);
      for (int t = lane; t < na * nc; t += 32) P[W::OAC + t] = dt_at(D, nt, tA[t / nc], tC[t % nc]);
      for (int t = lane; t < na * nd; t += 32) P[W::OAD + t] = dt_at(D, nt, tA[t / nd], tD[t % nd]);
      for (int t = lane; t < nb * nc; t += 32) P[W::OBC + t] = dt_at(D, nt, tB[t / nc], tC[t % nc]);
      for (int t = lane; t < nb * nd; t += 32) P[W::OBD + t] = dt_at(D, nt, tB[t / nd], tD[t % nd]);
      bool any = false;   // warp-uniform
      for (int p = g0; p < g0 + gn; ++p) {
        const PairView bp = load_pair(rec, p);
        const double sp = bp.bound;
        if (sp * hmax < thr) break;
        const int I = bp.si, J = bp.sj;
        const double zb = bp.zeta;
        const int qe = (G == H) ? p + 1 : h0 + hn;
        bool cab_ready = false;
        for (int q = h0; q < qe; ++q) {
          const PairView kq = load_pair(rec, q);
          const double sq = kq.bound;
          if (sp * sq < thr) break;   // the reference's screen (warp-uniform)
          const int K = kq.si, L = kq.sj;
          const double ze = kq.zeta;
          const double zz = zb + ze, rzz = 1.0 / zz, rho = zb * ze * rzz;
          const double dx = bp.P[0] - kq.P[0], dy = bp.P[1] - kq.P[1], dz = bp.P[2] - kq.P[2];
          const double T = rho * (dx * dx + dy * dy + dz * dz);
          const double pref = c2pi * bp.S * kq.S * sqrt(rho);
          double F[LT + 1];
          boys_tab<LT>(T, pref, boys, F);
          const double w = ((I != J) ? 2.0 : 1.0) * ((K != L) ? 2.0 : 1.0) * ((p != q) ? 2.0 : 1.0);
          __syncwarp();   // the previous quartet's ops and X update are done with v, geo, cab, ccd
          if (!cab_ready) {
            for (int t = lane; t < nab; t += 32)
              cab[t] = scoef[I * MAXCOMP + kA[t / nb]] * scoef[J * MAXCOMP + kB[t % nb]];
            cab_ready = true;
          }
          for (int t = lane; t < ncd; t += 32)
            ccd[t] = w * scoef[K * MAXCOMP + kC[t / nd]] * scoef[L * MAXCOMP + kD[t % nd]];
#pragma unroll
          for (int m = 0; m <= LT; ++m)
            if (lane == m) v[1 + m] = F[m];
          if (lane == LT + 1) {
            for (int k2 = 0; k2 < 3; ++k2) {
              const double Wk = (zb * bp.P[k2] + ze * kq.P[k2]) * rzz;
              geo.G1[0][k2] = bp.PA[k2];
              geo.G2[0][k2] = Wk - bp.P[k2];
              geo.G1[1][k2] = kq.PA[k2];
              geo.G2[1][k2] = Wk - kq.P[k2];
              geo.G2[2][k2] = bp.AB[k2];
              geo.G2[3][k2] = kq.AB[k2];
            }
            geo.X[0] = bp.oz;
            geo.Y[0] = ze * rzz;
            geo.X[1] = kq.oz;
            geo.Y[1] = zb * rzz;
            geo.Z = 0.5 * rzz;
          }
          __syncwarp();
          for (int l = 0; l < nlev; ++l) {
            const int o1 = levels[l + 1];
            run_level(ops, levels[l], o1, v, geo, lane, 32, EvalD{});
            __syncwarp();
          }
          for (int i = lane; i < nx; i += 32) {
            const int e = xs[i];
            X[i] = fma(cab[(e >> 15) & 127] * ccd[e >> 22], v[e & 0x7fff], X[i]);
          }
          any = true;
        }
      }
      __syncwarp();
      if (!any) continue;
      // digestion: J'(ab), J'(cd), K'(ad), K'(bd), K'(ac), K'(bc) of the kept components
      const int n1 = nab, n2 = n1 + ncd, n3 = n2 + na * nd, n4 = n3 + nb * nd, n5 = n4 + na * nc,
                n6 = n5 + nb * nc;
      for (int t = lane; t < n6; t += 32) {
        double acc = 0.0;
        if (t < n1) {
          for (int cd = 0; cd < ncd; ++cd) acc = fma(P[W::OCD + cd], X[t * ncd + cd], acc);
          add_target(ql.jt, nt, tA[t / nb], tB[t % nb], 0.25 * acc);
        } else if (t < n2) {
          const int cd = t - n1;
          for (int ab = 0; ab < nab; ++ab) acc = fma(P[W::OAB + ab], X[ab * ncd + cd], acc);
          add_target(ql.jt, nt, tC[cd / nd], tD[cd % nd], 0.25 * acc);
        } else if (t < n3) {   // K'(ad) += 1/8 P(bc) X
          const int r = t - n2, ia = r / nd, id = r % nd;
          for (int ib = 0; ib < nb; ++ib)
            for (int ic = 0; ic < nc; ++ic)
              acc = fma(P[W::OBC + ib * nc + ic], X[((ia * nb + ib) * nc + ic) * nd + id], acc);
          add_target(ql.kt, nt, tA[ia], tD[id], 0.125 * acc);
        } else if (t < n4) {   // K'(bd) += 1/8 P(ac) X
          const int r = t - n3, ib = r / nd, id = r % nd;
          for (int ia = 0; ia < na; ++ia)
            for (int ic = 0; ic < nc; ++ic)
              acc = fma(P[W::OAC + ia * nc + ic], X[((ia * nb + ib) * nc + ic) * nd + id], acc);
          add_target(ql.kt, nt, tB[ib], tD[id], 0.125 * acc);
        } else if (t < n5) {   // K'(ac) += 1/8 P(bd) X
          const int r = t - n4, ia = r / nc, ic = r % nc;
          for (int ib = 0; ib < nb; ++ib)
            for (int id = 0; id < nd; ++id)
              acc = fma(P[W::OBD + ib * nd + id], X[((ia * nb + ib) * nc + ic) * nd + id], acc);
          add_target(ql.kt, nt, tA[ia], tC[ic], 0.125 * acc);
        } else {               // K'(bc) += 1/8 P(ad) X
          const int r = t - n5, ib = r / nc, ic = r % nc;
          for (int ia = 0; ia < na; ++ia)
            for (int id = 0; id < nd; ++id)
              acc = fma(P[W::OAD + ia * nd + id], X[((ia * nb + ib) * nc + ic) * nd + id], acc);
          add_target(ql.kt, nt, tB[ib], tC[ic], 0.125 * acc);
        }
      }
    }
    __syncwarp();   // meta and the bra blocks are rewritten by the next chunk
  }
}

template <int LA, int LB, int LC, int LD>
void launch_wide(const MolLaunch& ql, const OpTableDev& t, int grid, int wpb, int per_warp, int vmax, int xmax,
                 size_t smem, cudaStream_t s) {
  k_gq_wide<LA, LB, LC, LD><<<grid, 32 * wpb, smem, s>>>(ql, t, per_warp, vmax, xmax);
}

template <int LA, int LB, int LC, int LD>
cudaError_t allow_wide(size_t smem) {
  const cudaError_t e =
      cudaFuncSetAttribute(k_gq_wide<LA, LB, LC, LD>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
  // ask for no more shared memory than the blocks use: the rest of the SM's
  // 256 KB is L1, where the op table the warps read stays resident
  return cudaFuncSetAttribute(k_gq_wide<LA, LB, LC, LD>, cudaFuncAttributePreferredSharedMemoryCarveout, 70);
}

template <int LA, int LB, int LC, int LD>
int wide_doubles_t(int vmax, int xmax) {
  return WideLayout<ncum(LA), ncum(LB), ncum(LC), ncum(LD)>::doubles(vmax, xmax);
}

}  // namespace

WideVariant wide_variant(int cb, int ck) {
#define V(A, B, C, D) WideVariant{&launch_wide<A, B, C, D>, &allow_wide<A, B, C, D>, &wide_doubles_t<A, B, C, D>}
  switch (cb * 8 + ck) {
    case 4 * 8 + 2: return V(2, 1, 1, 1);
    case 4 * 8 + 3: return V(2, 1, 2, 0);
    case 4 * 8 + 4: return V(2, 1, 2, 1);
    case 5 * 8 + 1: return V(2, 2, 1, 0);
    case 5 * 8 + 2: return V(2, 2, 1, 1);
    case 5 * 8 + 3: return V(2, 2, 2, 0);
    case 5 * 8 + 4: return V(2, 2, 2, 1);
    case 5 * 8 + 5: return V(2, 2, 2, 2);
    default: return WideVariant{nullptr, nullptr, nullptr};
  }
#undef V
}

}  // namespace pfe
