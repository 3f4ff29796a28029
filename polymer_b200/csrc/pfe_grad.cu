// Two-electron part of the nuclear gradient of a molecule: the work of
// FOURINDEX_ERI_GRADIENT (src/pfourindexgradient.f90:1-1478, molecular branch).
//
// For a fixed density P (target space: contracted functions, or primitives
// under a general contraction) the two-electron energy is
//   E2 = 1/2 sum (ij|kl) P_ij P_kl  -  HFX/4 sum (ij|kl) P_ik P_jl
// and its derivative with respect to the centre A of primitive i follows from
// d/dA_x phi_a = 2 zeta_a phi_{a+1x} - a_x phi_{a-1x} (the reference's
// FN = 2 ZT(II) ERI(UP1) - 2 DOWN1_C ERI(DOWN1), :1353-1361); the derivative
// with respect to B is minus the sum of the other three (translational
// invariance, as the reference forms its J-atom force, :1396-1398).  The
// J part and the K part are returned apart (the caller weighs K by HFX):
//   grad_J = 1/2 sum' w P_ab P_cd d(ab|cd)
//   grad_K = -1/8 sum' w (P_ac P_bd + P_ad P_bc) d(ab|cd)
// over the unique primitive quartets with their 8-fold degeneracy w and the
// contraction coefficients of each component, the quartets and screening of
// the Fock build (the same chunk lists).
//
// The derivative integrals come from three op tables per class, each with one
// centre raised by one (A, C, D: opg_<class>_a/c/d, generated next to the
// Fock tables), evaluated one primitive quartet per 256-thread block with the
// slots in shared memory; each block contracts them against the density
// blocks of its group quartet and adds twelve numbers per group quartet (three
// per centre) to the atoms' gradients.  Not a hot path (once per geometry
// step): correctness and coverage first.

#include <cuda_runtime.h>

#include <algorithm>
#include <vector>

#include "pfe_common.cuh"
#include "pfe_context.cuh"
#include "pfe_interp.cuh"
#include "pfe_mol_kernels.cuh"
#include "generated/eri_grad_tables.cuh"

namespace pfe {

namespace {

// Index maps of a cumulative shell's components under x/y/z raising and
// lowering: comps(L) in the reference's order (x power outer, z inner), the
// raised/lowered component's index in comps(L+1) (-1: none), and the power.
struct GradMaps {
  signed char up[3][10][3], dn[3][10][3], pw[3][10][3];
};

constexpr int comp_index(int L, int px, int py, int pz) {
  int n = 0;
  for (int i1 = 0; i1 <= L; ++i1)
    for (int i2 = 0; i2 <= L - i1; ++i2)
      for (int i3 = 0; i3 <= L - i1 - i2; ++i3) {
        if (i1 == px && i2 == py && i3 == pz) return n;
        ++n;
      }
  return -1;
}

constexpr GradMaps make_maps() {
  GradMaps m{};
  for (int L = 0; L < 3; ++L) {
    int n = 0;
    for (int i1 = 0; i1 <= L; ++i1)
      for (int i2 = 0; i2 <= L - i1; ++i2)
        for (int i3 = 0; i3 <= L - i1 - i2; ++i3, ++n) {
          const int p[3] = {i1, i2, i3};
          for (int x = 0; x < 3; ++x) {
            int u[3] = {p[0], p[1], p[2]}, d[3] = {p[0], p[1], p[2]};
            u[x] += 1;
            d[x] -= 1;
            m.up[L][n][x] = (signed char)comp_index(L + 1, u[0], u[1], u[2]);
            m.dn[L][n][x] = (signed char)(d[x] < 0 ? -1 : comp_index(L + 1, d[0], d[1], d[2]));
            m.pw[L][n][x] = (signed char)p[x];
          }
        }
  }
  return m;
}

__constant__ GradMaps c_gmap = make_maps();

struct GradTables {
  OpTableDev t[3];   // raised centre A, C, D
};

struct GradOut {
  double* gj;          // (natom, 3) column-major: dE_J/dx of atom a at a + natom*x
  double* gk;
  int natom;
  const int* satom;    // shell -> atom (0-based)
  const double* szeta; // shell -> exponent
};

template <int NA, int NB, int NC, int ND>
struct GLayout {
  static constexpr int OAB = 0, OCD = NA * NB, OAC = OCD + NC * ND, OAD = OAC + NA * NC, OBC = OAD + NA * ND,
                       OBD = OBC + NB * NC, NP = OBD + NB * ND;
};

template <int LA, int LB, int LC, int LD>
__global__ void __launch_bounds__(256) k_grad(MolLaunch ql, GradTables tabs, GradOut go, int vmax) {
  constexpr int NA = ncum(LA), NB = ncum(LB), NC = ncum(LC), ND = ncum(LD);
  constexpr int NA1 = ncum(LA + 1), NC1 = ncum(LC + 1), ND1 = ncum(LD + 1);
  constexpr int LT = LA + LB + LC + LD + 1;   // the raised classes' total angular momentum
  using GL = GLayout<NA, NB, NC, ND>;
  extern __shared__ double smem[];
  double* v = smem;
  double* P = v + vmax;
  double* cab = P + GL::NP;
  double* ccd = cab + NA * NB;
  __shared__ OpGeom geo;
  __shared__ int kA[NA], kB[NB], kC[NC], kD[ND], tA[NA], tB[NB], tC[NC], tD[ND], cnt[4];
  __shared__ double red[8][6];
  __shared__ double zeta3[3];
  const int tid = threadIdx.x, lane = tid & 31, wid = tid >> 5;
  const double c2pi = 2.0 / sqrt(REF_PI);
  const double* __restrict__ D = ql.dt;
  const int nt = ql.nt;
  const int nchunks = *ql.nchunks;
  for (int c = blockIdx.x; c < nchunks; c += gridDim.x) {
    const int4 ch = ql.chunks[c];
    const int G = ch.x;
    const int g0 = ql.gr_start[G], gn = ql.gr_n[G];
    const PairRec* __restrict__ rec = ql.rec;
    const int2 ij0 = __ldg(reinterpret_cast<const int2*>(&rec[g0].si));
    __syncthreads();   // the previous chunk is done with the shared lists
    if (tid == 0) {
      int n = 0;
      for (int x = 0; x < NA; ++x)
        if (ql.stidx[ij0.x * MAXCOMP + x] >= 0) { kA[n] = x; tA[n] = ql.stidx[ij0.x * MAXCOMP + x]; ++n; }
      cnt[0] = n;
      n = 0;
      for (int x = 0; x < NB; ++x)
        if (ql.stidx[ij0.y * MAXCOMP + x] >= 0) { kB[n] = x; tB[n] = ql.stidx[ij0.y * MAXCOMP + x]; ++n; }
      cnt[1] = n;
    }
    __syncthreads();
    const int na = cnt[0], nb = cnt[1], nab = na * nb;
    for (int t = tid; t < nab; t += blockDim.x) P[GL::OAB + t] = dt_at(D, nt, tA[t / nb], tB[t % nb]);
    for (int k = ch.y; k < ch.z; ++k) {
      const int H = ql.bk_list[k];
      const int h0 = ql.gr_start[H], hn = ql.gr_n[H];
      const double hmax = ql.gr_max[H];
      const double thr = ql.inttol;
      if (ql.gr_max[G] * hmax < thr) continue;   // block-uniform
      const int2 kl0 = __ldg(reinterpret_cast<const int2*>(&rec[h0].si));
      __syncthreads();
      if (tid == 0) {
        int n = 0;
        for (int x = 0; x < NC; ++x)
          if (ql.stidx[kl0.x * MAXCOMP + x] >= 0) { kC[n] = x; tC[n] = ql.stidx[kl0.x * MAXCOMP + x]; ++n; }
        cnt[2] = n;
        n = 0;
        for (int x = 0; x < ND; ++x)
          if (ql.stidx[kl0.y * MAXCOMP + x] >= 0) { kD[n] = x; tD[n] = ql.stidx[kl0.y * MAXCOMP + x]; ++n; }
        cnt[3] = n;
      }
      __syncthreads();
      const int nc = cnt[2], nd = cnt[3], ncd = nc * nd, nx = nab * ncd;
      for (int t = tid; t < ncd; t += blockDim.x) P[GL::OCD + t] = dt_at(D, nt, tC[t / nd], tD[t % nd]);
      for (int t = tid; t < na * nc; t += blockDim.x) P[GL::OAC + t] = dt_at(D, nt, tA[t / nc], tC[t % nc]);
      for (int t = tid; t < na * nd; t += blockDim.x) P[GL::OAD + t] = dt_at(D, nt, tA[t / nd], tD[t % nd]);
      for (int t = tid; t < nb * nc; t += blockDim.x) P[GL::OBC + t] = dt_at(D, nt, tB[t / nc], tC[t % nc]);
      for (int t = tid; t < nb * nd; t += blockDim.x) P[GL::OBD + t] = dt_at(D, nt, tB[t / nd], tD[t % nd]);
      // this group quartet's gradient, per centre (A, C, D) and axis, J and K (thread 0)
      double g[3][3][2] = {};
      for (int p = g0; p < g0 + gn; ++p) {
        const double sp = pair_bound(rec, p);
        if (sp * hmax < thr) break;
        const PairView bp = load_pair(rec, p);
        const int qe = (G == H) ? p + 1 : h0 + hn;
        for (int q = h0; q < qe; ++q) {
          const double sq = pair_bound(rec, q);
          if (sp * sq < thr) break;
          const PairView kq = load_pair(rec, q);
          __syncthreads();   // the previous quartet's tables and contractions are done
          if (tid == 0) {
            const double zb = bp.zeta, ze = kq.zeta, zz = zb + ze, rzz = 1.0 / zz, rho = zb * ze * rzz;
            const double dx = bp.P[0] - kq.P[0], dy = bp.P[1] - kq.P[1], dz = bp.P[2] - kq.P[2];
            const double T = rho * (dx * dx + dy * dy + dz * dz);
            double F[LT + 1];
            boys_tab<LT>(T, c2pi * bp.S * kq.S * sqrt(rho), ql.boys, F);
            v[0] = 0.0;
            for (int m = 0; m <= LT; ++m) v[1 + m] = F[m];
            double W[3], WP[3], WQ[3];
            for (int x = 0; x < 3; ++x) {
              W[x] = (zb * bp.P[x] + ze * kq.P[x]) * rzz;
              WP[x] = W[x] - bp.P[x];
              WQ[x] = W[x] - kq.P[x];
            }
            set_geom(geo, bp.PA, WP, kq.PA, WQ, bp.AB, kq.AB, bp.oz, kq.oz, 0.5 * rzz, ze * rzz, zb * rzz);
            zeta3[0] = go.szeta[bp.si];
            zeta3[1] = go.szeta[kq.si];
            zeta3[2] = go.szeta[kq.sj];
          }
          const double w = ((bp.si != bp.sj) ? 2.0 : 1.0) * ((kq.si != kq.sj) ? 2.0 : 1.0) * ((p != q) ? 2.0 : 1.0);
          const double* __restrict__ scoef = ql.scoef;
          for (int t = tid; t < nab; t += blockDim.x)
            cab[t] = scoef[bp.si * MAXCOMP + kA[t / nb]] * scoef[bp.sj * MAXCOMP + kB[t % nb]];
          for (int t = tid; t < ncd; t += blockDim.x)
            ccd[t] = w * scoef[kq.si * MAXCOMP + kC[t / nd]] * scoef[kq.sj * MAXCOMP + kD[t % nd]];
#pragma unroll 1
          for (int cen = 0; cen < 3; ++cen) {
            const OpTableDev& tb = tabs.t[cen];
            __syncthreads();
            for (int l = 0; l < tb.nlevels; ++l) {
              run_level(tb.ops, tb.levels[l], tb.levels[l + 1], v, geo, tid, (int)blockDim.x, EvalD{});
              __syncthreads();
            }
            const double z2 = 2.0 * zeta3[cen];
            double aj[3] = {0.0, 0.0, 0.0}, ak[3] = {0.0, 0.0, 0.0};
            for (int i = tid; i < nx; i += blockDim.x) {
              const int ab = i / ncd, cd = i - ab * ncd;
              const int ia = ab / nb, ib = ab - ia * nb, ic = cd / nd, id = cd - ic * nd;
              const int a = kA[ia], b = kB[ib], cc = kC[ic], d = kD[id];
              const double co = cab[ab] * ccd[cd];
              const double gj = co * P[GL::OAB + ab] * P[GL::OCD + cd];
              const double gk = co * (P[GL::OAC + ia * nc + ic] * P[GL::OBD + ib * nd + id] +
                                      P[GL::OAD + ia * nd + id] * P[GL::OBC + ib * nc + ic]);
#pragma unroll
              for (int x = 0; x < 3; ++x) {
                int up, dn, pw;
                int iu, idn;
                if (cen == 0) {
                  up = c_gmap.up[LA][a][x]; dn = c_gmap.dn[LA][a][x]; pw = c_gmap.pw[LA][a][x];
                  iu = ((up * NB + b) * NC + cc) * ND + d;
                  idn = dn < 0 ? -1 : ((dn * NB + b) * NC + cc) * ND + d;
                } else if (cen == 1) {
                  up = c_gmap.up[LC][cc][x]; dn = c_gmap.dn[LC][cc][x]; pw = c_gmap.pw[LC][cc][x];
                  iu = ((a * NB + b) * NC1 + up) * ND + d;
                  idn = dn < 0 ? -1 : ((a * NB + b) * NC1 + dn) * ND + d;
                } else {
                  up = c_gmap.up[LD][d][x]; dn = c_gmap.dn[LD][d][x]; pw = c_gmap.pw[LD][d][x];
                  iu = ((a * NB + b) * NC + cc) * ND1 + up;
                  idn = dn < 0 ? -1 : ((a * NB + b) * NC + cc) * ND1 + dn;
                }
                double der = z2 * v[tb.out[iu]];
                if (idn >= 0) der -= (double)pw * v[tb.out[idn]];
                aj[x] = fma(gj, der, aj[x]);
                ak[x] = fma(gk, der, ak[x]);
              }
            }
            // block reduction of the six sums
#pragma unroll
            for (int x = 0; x < 3; ++x) {
              aj[x] = warp_sum(aj[x]);
              ak[x] = warp_sum(ak[x]);
            }
            if (lane == 0)
              for (int x = 0; x < 3; ++x) { red[wid][x] = aj[x]; red[wid][3 + x] = ak[x]; }
            __syncthreads();
            if (tid == 0) {
              for (int wv = 0; wv < (int)(blockDim.x >> 5); ++wv)
                for (int x = 0; x < 3; ++x) {
                  g[cen][x][0] += red[wv][x];
                  g[cen][x][1] += red[wv][3 + x];
                }
            }
          }
          (void)NA1;
        }
      }
      if (tid == 0) {
        // centre atoms: A, C, D from the group quartet's shells, B by translational invariance
        const int atA = go.satom[ij0.x], atB = go.satom[ij0.y], atC = go.satom[kl0.x], atD = go.satom[kl0.y];
        const int at[3] = {atA, atC, atD};
        for (int x = 0; x < 3; ++x) {
          double sj = 0.0, sk = 0.0;
          for (int cen = 0; cen < 3; ++cen) {
            const double vj = 0.5 * g[cen][x][0], vk = -0.125 * g[cen][x][1];
            sj += vj;
            sk += vk;
            if (vj != 0.0) atomicAdd(go.gj + at[cen] + (size_t)go.natom * x, vj);
            if (vk != 0.0) atomicAdd(go.gk + at[cen] + (size_t)go.natom * x, vk);
          }
          if (sj != 0.0) atomicAdd(go.gj + atB + (size_t)go.natom * x, -sj);
          if (sk != 0.0) atomicAdd(go.gk + atB + (size_t)go.natom * x, -sk);
        }
      }
    }
  }
}

using GradFn = void (*)(const MolLaunch&, const GradTables&, const GradOut&, int vmax, int grid, size_t smem,
                        cudaStream_t);

template <int LA, int LB, int LC, int LD>
void launch_grad(const MolLaunch& ql, const GradTables& t, const GradOut& go, int vmax, int grid, size_t smem,
                 cudaStream_t s) {
  k_grad<LA, LB, LC, LD><<<grid, 256, smem, s>>>(ql, t, go, vmax);
}

template <int LA, int LB, int LC, int LD>
cudaError_t allow_grad(size_t smem) {
  return cudaFuncSetAttribute(k_grad<LA, LB, LC, LD>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
}

struct GradClass {
  GradFn fn;
  cudaError_t (*allow)(size_t);
  const OpTableHost* tab[3];
  int np;   // doubles of the density blocks and coefficients
};

GradClass grad_class(int cb, int ck) {
#define GC(A, B, C, D)                                                                                      \
  GradClass{&launch_grad<A, B, C, D>, &allow_grad<A, B, C, D>,                                              \
            {&opg_##A##B##C##D##_a, &opg_##A##B##C##D##_c, &opg_##A##B##C##D##_d},                          \
            GLayout<ncum(A), ncum(B), ncum(C), ncum(D)>::NP + ncum(A) * ncum(B) + ncum(C) * ncum(D)}
  switch (cb * 8 + ck) {
    case 0: return GC(0, 0, 0, 0);
    case 8: return GC(1, 0, 0, 0);
    case 9: return GC(1, 0, 1, 0);
    case 16: return GC(1, 1, 0, 0);
    case 17: return GC(1, 1, 1, 0);
    case 18: return GC(1, 1, 1, 1);
    case 24: return GC(2, 0, 0, 0);
    case 25: return GC(2, 0, 1, 0);
    case 26: return GC(2, 0, 1, 1);
    case 27: return GC(2, 0, 2, 0);
    case 32: return GC(2, 1, 0, 0);
    case 33: return GC(2, 1, 1, 0);
    case 34: return GC(2, 1, 1, 1);
    case 35: return GC(2, 1, 2, 0);
    case 36: return GC(2, 1, 2, 1);
    case 40: return GC(2, 2, 0, 0);
    case 41: return GC(2, 2, 1, 0);
    case 42: return GC(2, 2, 1, 1);
    case 43: return GC(2, 2, 2, 0);
    case 44: return GC(2, 2, 2, 1);
    case 45: return GC(2, 2, 2, 2);
    default: return GradClass{nullptr, nullptr, {nullptr, nullptr, nullptr}, 0};
  }
#undef GC
}

}  // namespace

// dE_J/dR and dE_K/dR (natom x 3 each, column-major) of the molecule set up in
// ctx for the target-space density d_dt, into device arrays d_gj, d_gk
// (overwritten).  satom: shell -> atom on the device.
int molecular_gradient(pfe_context* ctx, const double* d_dt, const int* d_satom, int natom, double* d_gj,
                       double* d_gk, cudaStream_t s) {
  PFE_CUDA(cudaMemsetAsync(d_gj, 0, sizeof(double) * 3 * (size_t)natom, s));
  PFE_CUDA(cudaMemsetAsync(d_gk, 0, sizeof(double) * 3 * (size_t)natom, s));
  MolLaunch ql = molecular_launch(ctx, d_dt);
  GradOut go{d_gj, d_gk, natom, d_satom, ctx->shells.zeta};
  for (int i = 0; i < ctx->nlaunch; ++i) {
    const ClassLaunch& cl = ctx->launches[i];
    const GradClass gc = grad_class(cl.cb, cl.ck);
    if (!gc.fn) { set_error("no gradient kernel for a quartet class"); return PFE_EUNSUPPORTED; }
    GradTables t{};
    int vmax = 0;
    for (int k = 0; k < 3; ++k) {
      const int rc = upload_optable(ctx, gc.tab[k], &t.t[k]);
      if (rc != PFE_OK) return rc;
      vmax = std::max(vmax, gc.tab[k]->nslots);
    }
    const size_t smem = sizeof(double) * ((size_t)vmax + gc.np);
    if (smem > 227 * 1024) { set_error("gradient op table exceeds shared memory"); return PFE_EUNSUPPORTED; }
    PFE_CUDA(gc.allow(smem));
    ql.chunks = cl.chunks;
    ql.nchunks = cl.d_nchunks;
    const int per_sm = std::max(1, (int)((228 * 1024) / (smem + 2048)));
    const int grid = std::max(1, std::min(cl.nchunks_host, ctx->num_sms * std::min(per_sm, 8)));
    gc.fn(ql, t, go, vmax, grid, smem, s);
    PFE_CUDA(cudaGetLastError());
  }
  return PFE_OK;
}

}  // namespace pfe
