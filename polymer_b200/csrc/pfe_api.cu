// C ABI of libpolymer_fock (include/polymer_fock.h): argument validation, the
// static-input cache, host <-> device staging and context lifetime.

#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <map>
#include <mutex>
#include <string>
#include <vector>

#include "pfe_common.cuh"
#include "pfe_context.cuh"
#include "generated/eri_classes.cuh"

namespace pfe {

// ------------------------------------------------------------------ helpers

int alloc_pairs(pfe_context* ctx, PairArrays* pa, long long n) {
  for (int k = 0; k < 3; ++k) {
    PFE_CUDA(ctx->alloc((void**)&pa->P[k], sizeof(double) * n));
    PFE_CUDA(ctx->alloc((void**)&pa->PA[k], sizeof(double) * n));
    PFE_CUDA(ctx->alloc((void**)&pa->AB[k], sizeof(double) * n));
  }
  PFE_CUDA(ctx->alloc((void**)&pa->zeta, sizeof(double) * n));
  PFE_CUDA(ctx->alloc((void**)&pa->S, sizeof(double) * n));
  PFE_CUDA(ctx->alloc((void**)&pa->schwarz, sizeof(double) * n));
  PFE_CUDA(ctx->alloc((void**)&pa->si, sizeof(int) * n));
  PFE_CUDA(ctx->alloc((void**)&pa->sj, sizeof(int) * n));
  PFE_CUDA(ctx->alloc((void**)&pa->cls, n));
  PFE_CUDA(ctx->alloc((void**)&pa->key, sizeof(unsigned long long) * n));
  PFE_CUDA(ctx->alloc((void**)&pa->gid, sizeof(int) * n));
  PFE_CUDA(ctx->alloc((void**)&pa->gmax, sizeof(double) * n));
  return PFE_OK;
}

void free_pairs(pfe_context* ctx, PairArrays* pa) {
  for (int k = 0; k < 3; ++k) {
    ctx->free_now(pa->P[k]);
    ctx->free_now(pa->PA[k]);
    ctx->free_now(pa->AB[k]);
  }
  ctx->free_now(pa->zeta);
  ctx->free_now(pa->S);
  ctx->free_now(pa->schwarz);
  ctx->free_now(pa->si);
  ctx->free_now(pa->sj);
  ctx->free_now(pa->cls);
  ctx->free_now(pa->key);
  ctx->free_now(pa->gid);
  ctx->free_now(pa->gmax);
  *pa = PairArrays{};
}

// Per primitive-shell-quartet flops of class (bra cb, ket ck) counted by the
// roofline: generated recursion + Boys (table Taylor, 13 per order) + quartet
// geometry (~40) + digestion (6 FMAs per integral = 12 flops).
double class_flops(int cb, int ck) {
  static const int L[6][2] = {{0, 0}, {1, 0}, {1, 1}, {2, 0}, {2, 1}, {2, 2}};
  const int la = L[cb][0], lb = L[cb][1], lc = L[ck][0], ld = L[ck][1];
  const double ni = (double)(ncum(la) * ncum(lb) * ncum(lc) * ncum(ld));
  const int lt = la + lb + lc + ld;
  return eri_recursion_flops(la, lb, lc, ld) + 13.0 * (lt + 1) + 40.0 + 12.0 * ni;
}

// 64-bit-word mixing hash of the static inputs (detects any change of them):
// four independent lanes over 32-byte steps (no single multiply chain over the
// megabytes of CC), folded together at the end.
static uint64_t fnv(uint64_t h, const void* p, size_t n) {
  const unsigned char* b = (const unsigned char*)p;
  uint64_t l[4] = {h, h ^ 0x243F6A8885A308D3ull, h ^ 0x13198A2E03707344ull, h ^ 0xA4093822299F31D0ull};
  size_t i = 0;
  for (; i + 32 <= n; i += 32)
    for (int k = 0; k < 4; ++k) {
      uint64_t w;
      memcpy(&w, b + i + 8 * k, 8);
      l[k] ^= w;
      l[k] *= 0x9E3779B97F4A7C15ull;
      l[k] ^= l[k] >> 29;
    }
  for (int k = 0; k < 4; ++k) {
    h ^= l[k];
    h *= 0x9E3779B97F4A7C15ull;
    h ^= h >> 29;
  }
  for (; i + 8 <= n; i += 8) {
    uint64_t w;
    memcpy(&w, b + i, 8);
    h ^= w;
    h *= 0x9E3779B97F4A7C15ull;
    h ^= h >> 29;
  }
  for (; i < n; ++i) {
    h ^= b[i];
    h *= 1099511628211ull;
  }
  return h;
}

static inline size_t psh_index(int npshell, int s, int i1, int i2, int i3) {
  return (size_t)s + (size_t)npshell * (i1 + NPOW * (i2 + NPOW * i3));
}

// Validate the argument block and derive the shell table on the host.
struct HostShells {
  std::vector<double> x, y, z, zeta;
  std::vector<int> L, prim, head;
  int lmax = 0;
};

static int build_host_shells(const pfe_args* a, HostShells* hs) {
  if (!a) { set_error("null argument block"); return PFE_EINVAL; }
  if (a->npgs <= 0 || a->ncgs <= 0 || a->npshell <= 0) { set_error("npgs, ncgs and npshell must be positive"); return PFE_EINVAL; }
  if (a->lmax != 3) { set_error("lmax must be BASIS_LMAX = 3 (P_SHELL layout)"); return PFE_EINVAL; }
  if (!a->p_shell || !a->p_shell_ang || !a->pgsx || !a->pgsy || !a->pgsz || !a->zt || !a->cc || !a->s_p || !a->igamma) {
    set_error("a required array pointer is null");
    return PFE_EINVAL;
  }
  for (int k = 0; k < 3; ++k) {
    if (a->cel1[k] < 0 || a->cel2[k] < 0 || a->reduced_cel1[k] < 0 || a->reduced_cel1[k] > a->cel1[k]) {
      set_error("invalid CUTOFF parameters");
      return PFE_EINVAL;
    }
  }
  if (a->numprocs < 1 || a->myid < 0 || a->myid >= a->numprocs) { set_error("invalid myid/numprocs"); return PFE_EINVAL; }
  if (a->helix != 0.0 && (a->cel1[1] | a->cel1[2] | a->cel2[1] | a->cel2[2])) {
    set_error("HELICAL SYMMETRY FOR 1D CRYSTAL ONLY");
    return PFE_EINVAL;
  }
  if (a->helix != 0.0 && (!a->c2h)) { set_error("helix != 0 needs C2H"); return PFE_EINVAL; }
  const int n = a->npshell;
  hs->x.resize(n); hs->y.resize(n); hs->z.resize(n); hs->zeta.resize(n);
  hs->L.resize(n); hs->prim.assign((size_t)n * MAXCOMP, -1); hs->head.resize(n);
  for (int s = 0; s < n; ++s) {
    const int L = a->p_shell_ang[s];
    if (L < 0 || L > 3) { set_error("P_SHELL_ANG out of range"); return PFE_EINVAL; }
    if (L > LMAX_SUPPORTED) {
      set_error("f shells (P_SHELL_ANG = 3) are not implemented by the CUDA kernels");
      return PFE_EUNSUPPORTED;
    }
    hs->lmax = std::max(hs->lmax, L);
    int c = 0;
    for (int i1 = 0; i1 <= L; ++i1)
      for (int i2 = 0; i2 <= L - i1; ++i2)
        for (int i3 = 0; i3 <= L - i1 - i2; ++i3) {
          const int p = a->p_shell[psh_index(n, s, i1, i2, i3)];
          if (p < 1 || p > a->npgs) {
            set_error("P_SHELL refers to a missing primitive: the shell is not cumulative");
            return PFE_EINVAL;
          }
          hs->prim[(size_t)s * MAXCOMP + c++] = p - 1;
        }
    const int h = hs->prim[(size_t)s * MAXCOMP];
    hs->head[s] = h;
    hs->x[s] = a->pgsx[h];
    hs->y[s] = a->pgsy[h];
    hs->z[s] = a->pgsz[h];
    hs->zeta[s] = a->zt[h];
    hs->L[s] = L;
    if (!(a->zt[h] > 0.0) || !std::isfinite(a->zt[h])) { set_error("non-positive exponent"); return PFE_EINVAL; }
  }
  return PFE_OK;
}

static uint64_t static_key(const pfe_args* a, const HostShells& hs) {
  uint64_t h = 1469598103934665603ull;
  h = fnv(h, &a->npgs, sizeof(int) * 4);
  h = fnv(h, hs.x.data(), sizeof(double) * hs.x.size());
  h = fnv(h, hs.y.data(), sizeof(double) * hs.y.size());
  h = fnv(h, hs.z.data(), sizeof(double) * hs.z.size());
  h = fnv(h, hs.zeta.data(), sizeof(double) * hs.zeta.size());
  h = fnv(h, hs.prim.data(), sizeof(int) * hs.prim.size());
  h = fnv(h, a->cc, sizeof(double) * (size_t)a->ncgs * a->npgs);
  h = fnv(h, a->igamma, sizeof(double) * 64);
  h = fnv(h, a->cel1, sizeof(int) * 9);
  h = fnv(h, a->period, sizeof(double) * 5);
  h = fnv(h, &a->myid, sizeof(int) * 3);
  h = fnv(h, &a->mixed_cutoff, sizeof(double));
  // the s-s overlaps of the shell heads are the only part of S_P the kernels read
  const int n = a->npshell;
  const int n1x = 2 * a->cel1[0] + 1, n1y = 2 * a->cel1[1] + 1, n1z = 2 * a->cel1[2] + 1;
  const size_t pp = (size_t)a->npgs * a->npgs;
  std::vector<double> col(n);
  for (int c = 0; c < n1x * n1y * n1z; ++c)
    for (int j = 0; j < n; ++j) {
      const double* sc = a->s_p + (size_t)a->npgs * hs.head[j] + pp * c;
      for (int i = 0; i < n; ++i) col[i] = sc[hs.head[i]];
      h = fnv(h, col.data(), sizeof(double) * n);
    }
  if (a->helix != 0.0 && a->c2h) {
    const int nq = 2 * (a->cel2[0] + a->cel1[0]) + 1;
    h = fnv(h, a->c2h, sizeof(double) * (size_t)a->ncgs * a->ncgs * nq);
  }
  return h;
}

static void reset_context(pfe_context* ctx) {
  if (ctx->lattice) lattice_release(ctx);
  ctx->release_all();
  ctx->shells = DevShells{};
  ctx->pairs = PairArrays{};
  ctx->d_sss = ctx->d_boys = ctx->d_maxc = ctx->d_cc = ctx->d_c2h = nullptr;
  ctx->d_jp = ctx->d_kp = ctx->d_w1 = ctx->d_w2 = nullptr;
  ctx->d_tidx = nullptr;
  ctx->d_tcoef = nullptr;
  ctx->d_blk = nullptr;
  ctx->d_rep = nullptr;
  ctx->d_repc = nullptr;
  ctx->d_scoef = nullptr;
  ctx->d_stidx = nullptr;
  ctx->d_tblk = nullptr;
  ctx->d_bmax = nullptr;
  ctx->d_n32 = nullptr;
  ctx->d_pt = nullptr;
  ctx->d_flag = nullptr;
  ctx->d_gr_start = ctx->d_gr_n = ctx->d_bk_list = nullptr;
  ctx->d_gr_max = nullptr;
  ctx->d_prec = nullptr;
  ctx->ngroups = 0;
  ctx->d_pp = ctx->d_pph = ctx->d_out_c = ctx->d_out_x = nullptr;
  ctx->pp_bytes = ctx->pph_bytes = ctx->out_bytes = 0;
  ctx->nlaunch = 0;
  ctx->ready = false;
  ctx->tuned = false;
}

static int setup_impl(pfe_context* ctx, const pfe_args* a, const HostShells& hs, uint64_t key) {
  int rc;
  PFE_CUDA(cudaSetDevice(ctx->device));
  if ((rc = upload_constants(ctx->device)) != PFE_OK) return rc;
  reset_context(ctx);
  ctx->npgs = a->npgs;
  ctx->ncgs = a->ncgs;
  ctx->npshell = a->npshell;
  for (int k = 0; k < 3; ++k) {
    ctx->cel1[k] = a->cel1[k];
    ctx->cel2[k] = a->cel2[k];
    ctx->rc1[k] = a->reduced_cel1[k];
    ctx->period[k] = a->period[k];
  }
  ctx->ncell1 = (2 * a->cel1[0] + 1) * (2 * a->cel1[1] + 1) * (2 * a->cel1[2] + 1);
  ctx->helix = a->helix;
  ctx->inttol = a->inttol;
  ctx->myid = a->myid;
  ctx->numprocs = a->numprocs;
  ctx->precision = a->precision_mode;
  ctx->mixed_cutoff = a->mixed_cutoff;
  if (a->precision_mode != PFE_PREC_FP64 && a->precision_mode != PFE_PREC_MIXED) {
    set_error("precision_mode must be PFE_PREC_FP64 or PFE_PREC_MIXED");
    return PFE_EINVAL;
  }
  if (!(a->mixed_cutoff >= 0.0)) { set_error("mixed_cutoff must be >= 0"); return PFE_EINVAL; }
  ctx->mcut = a->precision_mode == PFE_PREC_MIXED ? a->mixed_cutoff : 0.0;
  ctx->dtol = 0.0;
  ctx->molecular = (ctx->ncell1 == 1 && a->cel2[0] == 0 && a->cel2[1] == 0 && a->cel2[2] == 0 && a->helix == 0.0);
  cudaStream_t s = ctx->stream;
  const int n = a->npshell;
  // shells
  DevShells& sh = ctx->shells;
  sh.n = n;
  PFE_CUDA(ctx->alloc((void**)&sh.x, sizeof(double) * n));
  PFE_CUDA(ctx->alloc((void**)&sh.y, sizeof(double) * n));
  PFE_CUDA(ctx->alloc((void**)&sh.z, sizeof(double) * n));
  PFE_CUDA(ctx->alloc((void**)&sh.zeta, sizeof(double) * n));
  PFE_CUDA(ctx->alloc((void**)&sh.L, sizeof(int) * n));
  PFE_CUDA(ctx->alloc((void**)&sh.prim, sizeof(int) * n * MAXCOMP));
  PFE_CUDA(cudaMemcpyAsync(sh.x, hs.x.data(), sizeof(double) * n, cudaMemcpyHostToDevice, s));
  PFE_CUDA(cudaMemcpyAsync(sh.y, hs.y.data(), sizeof(double) * n, cudaMemcpyHostToDevice, s));
  PFE_CUDA(cudaMemcpyAsync(sh.z, hs.z.data(), sizeof(double) * n, cudaMemcpyHostToDevice, s));
  PFE_CUDA(cudaMemcpyAsync(sh.zeta, hs.zeta.data(), sizeof(double) * n, cudaMemcpyHostToDevice, s));
  PFE_CUDA(cudaMemcpyAsync(sh.L, hs.L.data(), sizeof(int) * n, cudaMemcpyHostToDevice, s));
  PFE_CUDA(cudaMemcpyAsync(sh.prim, hs.prim.data(), sizeof(int) * n * MAXCOMP, cudaMemcpyHostToDevice, s));
  // s-s overlaps of the shell heads per cell, [cell][J][I]
  {
    std::vector<double> sss((size_t)n * n * ctx->ncell1);
    const size_t pp = (size_t)a->npgs * a->npgs;
    for (int c = 0; c < ctx->ncell1; ++c)
      for (int j = 0; j < n; ++j)
        for (int i = 0; i < n; ++i)
          sss[(size_t)i + (size_t)n * j + (size_t)n * n * c] = a->s_p[(size_t)hs.head[i] + (size_t)a->npgs * hs.head[j] + pp * c];
    PFE_CUDA(ctx->alloc((void**)&ctx->d_sss, sizeof(double) * sss.size()));
    PFE_CUDA(cudaMemcpyAsync(ctx->d_sss, sss.data(), sizeof(double) * sss.size(), cudaMemcpyHostToDevice, s));
    PFE_CUDA(cudaStreamSynchronize(s));
  }
  // Boys table, row-major [T][m]
  {
    std::vector<double> tab((size_t)NIG_T * NIG_M);
    for (int t = 0; t < NIG_T; ++t)
      for (int m = 0; m < NIG_M; ++m) tab[(size_t)t * NIG_M + m] = a->igamma[t + (size_t)NIG_T * m];
    PFE_CUDA(ctx->alloc((void**)&ctx->d_boys, sizeof(double) * tab.size()));
    PFE_CUDA(cudaMemcpyAsync(ctx->d_boys, tab.data(), sizeof(double) * tab.size(), cudaMemcpyHostToDevice, s));
    PFE_CUDA(cudaStreamSynchronize(s));
  }
  // MAXC and CC
  {
    std::vector<double> maxc(a->npgs, 0.0);
    for (int p = 0; p < a->npgs; ++p)
      for (int r = 0; r < a->ncgs; ++r) maxc[p] = std::max(maxc[p], std::fabs(a->cc[r + (size_t)a->ncgs * p]));
    PFE_CUDA(ctx->alloc((void**)&ctx->d_maxc, sizeof(double) * a->npgs));
    PFE_CUDA(cudaMemcpy(ctx->d_maxc, maxc.data(), sizeof(double) * a->npgs, cudaMemcpyHostToDevice));
    PFE_CUDA(ctx->alloc((void**)&ctx->d_cc, sizeof(double) * (size_t)a->ncgs * a->npgs));
    PFE_CUDA(cudaMemcpy(ctx->d_cc, a->cc, sizeof(double) * (size_t)a->ncgs * a->npgs, cudaMemcpyHostToDevice));
  }
  if (a->helix != 0.0) {
    const int nq = 2 * (a->cel2[0] + a->cel1[0]) + 1;
    PFE_CUDA(ctx->alloc((void**)&ctx->d_c2h, sizeof(double) * (size_t)a->ncgs * a->ncgs * nq));
    PFE_CUDA(cudaMemcpy(ctx->d_c2h, a->c2h, sizeof(double) * (size_t)a->ncgs * a->ncgs * nq, cudaMemcpyHostToDevice));
  }
  // digestion targets and contracted blocks
  {
    std::vector<int> tidx(a->npgs, -1);
    std::vector<double> tcoef(a->npgs, 0.0);
    bool single = true;
    for (int p = 0; p < a->npgs; ++p) {
      int nz = 0;
      for (int r = 0; r < a->ncgs; ++r) {
        const double v = a->cc[r + (size_t)a->ncgs * p];
        if (v != 0.0) {
          ++nz;
          tidx[p] = r;
          tcoef[p] = v;
        }
      }
      if (nz > 1) single = false;
    }
    ctx->contracted = single && ctx->molecular && !ctx->force_primitive;
    if (!ctx->contracted) {
      for (int p = 0; p < a->npgs; ++p) {
        const bool ghost = tidx[p] < 0;
        tidx[p] = ghost ? -1 : p;
        tcoef[p] = ghost ? 0.0 : 1.0;
      }
    }
    ctx->nt = ctx->contracted ? a->ncgs : a->npgs;
    // contracted block of a shell: the tuple of target rows of its components
    std::map<std::vector<int>, int> keys;
    std::vector<int> blk(a->npshell);
    for (int sh = 0; sh < a->npshell; ++sh) {
      std::vector<int> key;
      key.push_back(hs.L[sh]);
      for (int c = 0; c < ncum(hs.L[sh]); ++c) {
        const int p = hs.prim[(size_t)sh * MAXCOMP + c];
        key.push_back(ctx->contracted ? tidx[p] : p);
      }
      auto it = keys.emplace(key, (int)keys.size()).first;
      blk[sh] = it->second;
    }
    ctx->nblk = (int)keys.size();
    if ((long long)ctx->nblk * ctx->nblk > (1LL << 30)) {
      set_error("too many shells for the block-pair index (more than 32768 distinct shells)");
      return PFE_EINVAL;
    }
    {
      std::vector<double> scoef((size_t)a->npshell * MAXCOMP, 0.0);
      std::vector<int> stidx((size_t)a->npshell * MAXCOMP, -1);
      for (int sh = 0; sh < a->npshell; ++sh)
        for (int c = 0; c < ncum(hs.L[sh]); ++c) {
          const int p = hs.prim[(size_t)sh * MAXCOMP + c];
          scoef[(size_t)sh * MAXCOMP + c] = tcoef[p];
          stidx[(size_t)sh * MAXCOMP + c] = tidx[p];
        }
      for (int L = 0; L < 3; ++L) { ctx->kept_max[L] = 0; ctx->lower_kept[L] = false; }
      for (int sh = 0; sh < a->npshell; ++sh) {
        const int L = hs.L[sh];
        int kept = 0, c = 0;
        for (int i1 = 0; i1 <= L; ++i1)   // the components in P_SHELL order, with their total power
          for (int i2 = 0; i2 <= L - i1; ++i2)
            for (int i3 = 0; i3 <= L - i1 - i2; ++i3, ++c)
              if (stidx[(size_t)sh * MAXCOMP + c] >= 0) {
                ++kept;
                if (i1 + i2 + i3 < L) ctx->lower_kept[L] = true;
              }
        ctx->kept_max[L] = std::max(ctx->kept_max[L], kept);
      }
      PFE_CUDA(ctx->alloc((void**)&ctx->d_scoef, sizeof(double) * scoef.size()));
      PFE_CUDA(ctx->alloc((void**)&ctx->d_stidx, sizeof(int) * stidx.size()));
      PFE_CUDA(cudaMemcpy(ctx->d_scoef, scoef.data(), sizeof(double) * scoef.size(), cudaMemcpyHostToDevice));
      PFE_CUDA(cudaMemcpy(ctx->d_stidx, stidx.data(), sizeof(int) * stidx.size(), cudaMemcpyHostToDevice));
    }
    PFE_CUDA(ctx->alloc((void**)&ctx->d_tidx, sizeof(int) * a->npgs));
    PFE_CUDA(ctx->alloc((void**)&ctx->d_tcoef, sizeof(double) * a->npgs));
    PFE_CUDA(ctx->alloc((void**)&ctx->d_blk, sizeof(int) * a->npshell));
    PFE_CUDA(cudaMemcpy(ctx->d_tidx, tidx.data(), sizeof(int) * a->npgs, cudaMemcpyHostToDevice));
    PFE_CUDA(cudaMemcpy(ctx->d_tcoef, tcoef.data(), sizeof(double) * a->npgs, cudaMemcpyHostToDevice));
    PFE_CUDA(cudaMemcpy(ctx->d_blk, blk.data(), sizeof(int) * a->npshell, cudaMemcpyHostToDevice));
    // representative primitive of every target (largest |coefficient|): P_C(mu,nu) is read
    // off P_P at the representatives of mu and nu
    std::vector<int> rep(ctx->nt, -1);
    std::vector<double> repc(ctx->nt, 0.0);
    for (int p = 0; p < a->npgs; ++p) {
      const int r = tidx[p];
      if (r >= 0 && std::fabs(tcoef[p]) > std::fabs(repc[r])) { rep[r] = p; repc[r] = tcoef[p]; }
    }
    // block of every target, for the per-block density maxima
    std::vector<int> tblk(ctx->nt, -1);
    for (int sh = 0; sh < a->npshell; ++sh)
      for (int c = 0; c < ncum(hs.L[sh]); ++c) {
        const int t = tidx[hs.prim[(size_t)sh * MAXCOMP + c]];
        if (t >= 0) tblk[t] = blk[sh];
      }
    PFE_CUDA(ctx->alloc((void**)&ctx->d_tblk, sizeof(int) * ctx->nt));
    PFE_CUDA(cudaMemcpy(ctx->d_tblk, tblk.data(), sizeof(int) * ctx->nt, cudaMemcpyHostToDevice));
    PFE_CUDA(ctx->alloc((void**)&ctx->d_bmax, sizeof(double) * (size_t)ctx->nblk * ctx->nblk));
    PFE_CUDA(ctx->alloc((void**)&ctx->d_n32, sizeof(unsigned long long)));
    PFE_CUDA(cudaMemset(ctx->d_n32, 0, sizeof(unsigned long long)));
    PFE_CUDA(ctx->alloc((void**)&ctx->d_rep, sizeof(int) * ctx->nt));
    PFE_CUDA(ctx->alloc((void**)&ctx->d_repc, sizeof(double) * ctx->nt));
    PFE_CUDA(ctx->alloc((void**)&ctx->d_pt, sizeof(double) * (size_t)ctx->nt * ctx->nt));
    PFE_CUDA(ctx->alloc((void**)&ctx->d_flag, sizeof(unsigned int)));
    PFE_CUDA(cudaMemcpy(ctx->d_rep, rep.data(), sizeof(int) * ctx->nt, cudaMemcpyHostToDevice));
    PFE_CUDA(cudaMemcpy(ctx->d_repc, repc.data(), sizeof(double) * ctx->nt, cudaMemcpyHostToDevice));
  }
  // accumulators and GEMM scratch
  const size_t pp = (size_t)a->npgs * a->npgs * ctx->ncell1;
  PFE_CUDA(ctx->alloc((void**)&ctx->d_jp, sizeof(double) * pp));
  PFE_CUDA(ctx->alloc((void**)&ctx->d_kp, sizeof(double) * pp));
  PFE_CUDA(ctx->alloc((void**)&ctx->d_w1, sizeof(double) * (size_t)a->ncgs * a->npgs * ctx->ncell1));
  PFE_CUDA(ctx->alloc((void**)&ctx->d_w2, sizeof(double) * (size_t)a->ncgs * a->ncgs * ctx->ncell1));
  rc = ctx->molecular ? molecular_setup(ctx, a) : lattice_setup(ctx, a);
  if (rc != PFE_OK) return rc;
  ctx->key = key;
  ctx->ready = true;
  return PFE_OK;
}

static int check_density(const double* p, size_t n) {
  // x*0 is 0 for finite x and NaN otherwise: four independent sums, no branch
  // per element (a density of a million elements checks in a fraction of a ms)
  double a0 = 0.0, a1 = 0.0, a2 = 0.0, a3 = 0.0;
  size_t i = 0;
  for (; i + 4 <= n; i += 4) {
    a0 += p[i] * 0.0;
    a1 += p[i + 1] * 0.0;
    a2 += p[i + 2] * 0.0;
    a3 += p[i + 3] * 0.0;
  }
  for (; i < n; ++i) a0 += p[i] * 0.0;
  if (!(a0 + a1 + a2 + a3 == 0.0)) {
    set_error("non-finite density element in P_P");
    return PFE_ENAN;
  }
  return PFE_OK;
}

}  // namespace pfe

using namespace pfe;

extern "C" {

const char* pfe_version(void) { return "polymer_fock 0.1 (sm_100a, cumulative s/p/d shells)"; }

int32_t pfe_debug_fail_allocation(int32_t after) {
  pfe::g_fail_alloc_after.store(after < 0 ? -1 : (long long)after);
  return PFE_OK;
}

int32_t pfe_last_error(char* buf, int32_t len) {
  const char* m = last_error_cstr();
  const int32_t n = (int32_t)strlen(m);
  if (buf && len > 0) {
    const int32_t k = n < len - 1 ? n : len - 1;
    memcpy(buf, m, k);
    buf[k] = 0;
  }
  return n;
}

int32_t pfe_context_create(int32_t device, pfe_context** out) {
  if (!out) { set_error("null output handle"); return PFE_EINVAL; }
  int ndev = 0;
  PFE_CUDA(cudaGetDeviceCount(&ndev));
  if (device < 0 || device >= ndev) { set_error("no such CUDA device"); return PFE_EINVAL; }
  PFE_CUDA(cudaSetDevice(device));
  pfe_context* ctx = new pfe_context();
  ctx->device = device;
  PFE_CUDA(cudaDeviceGetAttribute(&ctx->num_sms, cudaDevAttrMultiProcessorCount, device));
  PFE_CUDA(cudaStreamCreateWithFlags(&ctx->stream, cudaStreamNonBlocking));
  PFE_CUDA(cudaStreamCreateWithFlags(&ctx->side, cudaStreamNonBlocking));
  PFE_CUDA(cudaEventCreateWithFlags(&ctx->ev_fork, cudaEventDisableTiming));
  PFE_CUDA(cudaEventCreateWithFlags(&ctx->ev_join, cudaEventDisableTiming));
  *out = ctx;   // the cuBLAS handle comes with the first call that needs it (ensure_blas)
  return PFE_OK;
}

int32_t pfe_context_destroy(pfe_context* ctx) {
  if (!ctx) return PFE_OK;
  cudaSetDevice(ctx->device);
  cudaStreamSynchronize(ctx->stream);
  reset_context(ctx);
  if (ctx->blas) cublasDestroy(ctx->blas);
  if (ctx->side) {
    cudaStreamSynchronize(ctx->side);
    cudaStreamDestroy(ctx->side);
  }
  if (ctx->ev_fork) cudaEventDestroy(ctx->ev_fork);
  if (ctx->ev_join) cudaEventDestroy(ctx->ev_join);
  if (ctx->stream) cudaStreamDestroy(ctx->stream);
  delete ctx;
  return PFE_OK;
}

int32_t pfe_context_setup(pfe_context* ctx, const pfe_args* a) {
  if (!ctx) { set_error("null context"); return PFE_EINVAL; }
  HostShells hs;
  int rc = build_host_shells(a, &hs);
  if (rc != PFE_OK) return rc;
  const uint64_t key = static_key(a, hs);
  if (ctx->ready && ctx->key == key) return PFE_OK;
  rc = setup_impl(ctx, a, hs, key);
  if (rc != PFE_OK) ctx->ready = false;
  return rc;
}

int32_t pfe_context_fock(pfe_context* ctx, const double* d_p_p, const double* d_p_p_helix, double* d_c_c, double* d_x_c,
                         void* stream) {
  if (!ctx || !ctx->ready) { set_error("context is not set up"); return PFE_EINVAL; }
  if (!d_p_p || !d_c_c || !d_x_c) { set_error("null device pointer"); return PFE_EINVAL; }
  if (ctx->helix != 0.0 && !d_p_p_helix) { set_error("helix != 0 needs P_P_HELIX"); return PFE_EINVAL; }
  PFE_CUDA(cudaSetDevice(ctx->device));
  cudaStream_t s = (cudaStream_t)stream;
  if (!ctx->molecular) return lattice_fock(ctx, d_p_p, d_p_p_helix, d_c_c, d_x_c, s);
  int rc = molecular_fock(ctx, d_p_p, d_c_c, d_x_c, s);
  if (rc != PFE_OK || !ctx->contracted) return rc;
  // contracted targets read P_C off P_P: confirm P_P = CC^T P_C CC (not possible
  // while the stream is being captured; pfe_context_fock_pc takes P_C itself)
  cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
  PFE_CUDA(cudaStreamIsCapturing(s, &cs));
  if (cs != cudaStreamCaptureStatusNone) return PFE_OK;
  bool ok = true;
  if ((rc = molecular_density_ok(ctx, s, &ok)) != PFE_OK) return rc;
  if (!ok) {
    set_error("P_P is not the decontraction CC^T P_C CC of a contracted density; set the context up with "
              "primitive targets (pfe_context_primitive_targets, then pfe_context_setup)");
    return PFE_EINVAL;
  }
  return PFE_OK;
}

int32_t pfe_context_fock_pc(pfe_context* ctx, const double* d_p_c, double* d_c_c, double* d_x_c, void* stream) {
  if (!ctx || !ctx->ready) { set_error("context is not set up"); return PFE_EINVAL; }
  if (!d_p_c || !d_c_c || !d_x_c) { set_error("null device pointer"); return PFE_EINVAL; }
  if (!ctx->molecular) { set_error("pfe_context_fock_pc: molecules only (lattices take P_P and P_P_HELIX)"); return PFE_EUNSUPPORTED; }
  PFE_CUDA(cudaSetDevice(ctx->device));
  return molecular_fock_pc(ctx, d_p_c, d_c_c, d_x_c, (cudaStream_t)stream);
}

int32_t pfe_context_set_screening(pfe_context* ctx, int32_t precision_mode, double mixed_cutoff, double density_tol) {
  if (!ctx || !ctx->ready) { set_error("context is not set up"); return PFE_EINVAL; }
  if (precision_mode != PFE_PREC_FP64 && precision_mode != PFE_PREC_MIXED) {
    set_error("precision_mode must be PFE_PREC_FP64 or PFE_PREC_MIXED");
    return PFE_EINVAL;
  }
  if (!(mixed_cutoff >= 0.0) || !(density_tol >= 0.0)) { set_error("cutoffs must be >= 0"); return PFE_EINVAL; }
  if (!ctx->molecular && density_tol != 0.0) {
    set_error("density screening is implemented for molecules only");
    return PFE_EUNSUPPORTED;
  }
  if (!ctx->molecular && precision_mode == PFE_PREC_MIXED && !(mixed_cutoff > 0.0)) {
    set_error("lattices: PFE_PREC_MIXED needs a positive mixed_cutoff (it switches the far cells to FP32)");
    return PFE_EINVAL;
  }
  ctx->mcut = precision_mode == PFE_PREC_MIXED ? mixed_cutoff : 0.0;
  ctx->dtol = density_tol;
  return PFE_OK;
}

int32_t pfe_batch_create(int32_t device, pfe_batch** out) {
  if (!out) { set_error("null output handle"); return PFE_EINVAL; }
  int ndev = 0;
  PFE_CUDA(cudaGetDeviceCount(&ndev));
  if (device < 0 || device >= ndev) { set_error("no such CUDA device"); return PFE_EINVAL; }
  pfe_batch* b = new pfe_batch();
  b->device = device;
  *out = b;
  return PFE_OK;
}

// Frees the instances and the joined launches: the batch is not set up.
static void batch_clear(pfe_batch* b) {
  cudaSetDevice(b->device);
  cudaDeviceSynchronize();
  for (pfe_context* c : b->inst) pfe_context_destroy(c);
  b->inst.clear();
  b->release_all();
  b->off.assign(1, 0);
}

int32_t pfe_batch_destroy(pfe_batch* b) {
  if (!b) return PFE_OK;
  batch_clear(b);
  delete b;
  return PFE_OK;
}

int32_t pfe_batch_setup(pfe_batch* b, const pfe_args* args, int32_t n) {
  if (!b || !args || n < 1) { set_error("pfe_batch_setup: bad argument"); return PFE_EINVAL; }
  PFE_CUDA(cudaSetDevice(b->device));
  batch_clear(b);
  int rc = PFE_OK;
  for (int k = 0; k < n && rc == PFE_OK; ++k) {
    pfe_context* c = nullptr;
    if ((rc = pfe_context_create(b->device, &c)) != PFE_OK) break;
    b->inst.push_back(c);
    if ((rc = pfe_context_setup(c, &args[k])) != PFE_OK) break;
    if (!c->molecular) {
      set_error("pfe_batch_setup: batches hold molecules only");
      rc = PFE_EUNSUPPORTED;
    } else if (c->numprocs != 1) {
      set_error("pfe_batch_setup: one rank per batch (numprocs 1)");
      rc = PFE_EUNSUPPORTED;
    } else {
      b->off.push_back(b->off.back() + (long long)c->ncgs * c->ncgs);
    }
  }
  if (rc == PFE_OK) rc = batch_setup(b);
  if (rc != PFE_OK) {   // keep the message; leave no half-built batch behind
    batch_clear(b);
    return rc;
  }
  b->ready = true;
  return PFE_OK;
}

int32_t pfe_batch_set_screening(pfe_batch* b, int32_t precision_mode, double mixed_cutoff, double density_tol) {
  if (!b || !b->ready) { set_error("batch is not set up"); return PFE_EINVAL; }
  for (pfe_context* c : b->inst) {
    int rc = pfe_context_set_screening(c, precision_mode, mixed_cutoff, density_tol);
    if (rc != PFE_OK) return rc;
  }
  b->insts_for = nullptr;   // the launch records carry the thresholds
  return PFE_OK;
}

int32_t pfe_batch_set_instance_screening(pfe_batch* b, int32_t k, int32_t precision_mode, double mixed_cutoff,
                                         double density_tol) {
  if (!b || !b->ready) { set_error("batch is not set up"); return PFE_EINVAL; }
  if (k < 0 || k >= (int)b->inst.size()) { set_error("no such instance in the batch"); return PFE_EINVAL; }
  pfe_context* c = b->inst[k];
  const double mc = c->mcut, dt = c->dtol;
  int rc = pfe_context_set_screening(c, precision_mode, mixed_cutoff, density_tol);
  if (rc != PFE_OK) return rc;
  if (c->mcut != mc || c->dtol != dt) b->insts_for = nullptr;
  return PFE_OK;
}

int32_t pfe_batch_refresh(pfe_batch* b, const double* d_p_c) {
  if (!b || !b->ready) { set_error("batch is not set up"); return PFE_EINVAL; }
  if (!d_p_c) { set_error("null device pointer"); return PFE_EINVAL; }
  PFE_CUDA(cudaSetDevice(b->device));
  return batch_refresh(b, d_p_c);
}

// (la lb lc ld) of a (bra class, ket class) pair as a four-digit code
static int class_code(int cb, int ck) {
  static const int t[6][2] = {{0, 0}, {1, 0}, {1, 1}, {2, 0}, {2, 1}, {2, 2}};
  return 1000 * t[cb][0] + 100 * t[cb][1] + 10 * t[ck][0] + t[ck][1];
}

int32_t pfe_batch_autotune(pfe_batch* b, const double* d_p_c, void* stream) {
  if (!b || !b->ready) { set_error("batch is not set up"); return PFE_EINVAL; }
  if (!d_p_c) { set_error("null device pointer"); return PFE_EINVAL; }
  PFE_CUDA(cudaSetDevice(b->device));
  return batch_autotune(b, d_p_c, (cudaStream_t)stream);
}

int32_t pfe_batch_schedule(pfe_batch* b, pfe_kernel_stat* out, int32_t cap) {
  if (!b || !out) { set_error("null argument"); return PFE_EINVAL; }
  int n = 0;
  for (int i = 0; i < b->nlaunch && n < cap; ++i, ++n) {
    const ClassLaunch& cl = b->launches[i];
    out[n].cls = class_code(cl.cb, cl.ck);
    out[n].variant = cl.variant;
    for (int v = 0; v < 4; ++v) out[n].tuned_ms[v] = cl.tuned_ms[v];
    out[n].ms = 0.f;
    out[n].quartets = cl.quartets;
    out[n].flops = cl.quartets * class_flops(cl.cb, cl.ck);
    out[n].grid_mult = cl.gmul;
    out[n].pad_ = 0;
  }
  return n;
}

int32_t pfe_batch_offsets(pfe_batch* b, int64_t* off) {
  if (!b || !off) { set_error("null argument"); return PFE_EINVAL; }
  for (size_t k = 0; k < b->off.size(); ++k) off[k] = b->off[k];
  return (int32_t)b->inst.size();
}

int32_t pfe_batch_fock_pc(pfe_batch* b, const double* d_p_c, double* d_c_c, double* d_x_c, void* stream) {
  if (!b || !b->ready) { set_error("batch is not set up"); return PFE_EINVAL; }
  if (!d_p_c || !d_c_c || !d_x_c) { set_error("null device pointer"); return PFE_EINVAL; }
  PFE_CUDA(cudaSetDevice(b->device));
  return batch_fock_pc(b, d_p_c, d_c_c, d_x_c, (cudaStream_t)stream);
}

int32_t pfe_batch_census(pfe_batch* b, pfe_census* out) {
  if (!b || !out) { set_error("null argument"); return PFE_EINVAL; }
  pfe_census tot{};
  for (pfe_context* c : b->inst) {
    pfe_census ci{};
    int rc = pfe_context_census(c, &ci);
    if (rc != PFE_OK) return rc;
    tot.quartets += ci.quartets;
    tot.quartets_ref += ci.quartets_ref;
    tot.quartets_fp32 += ci.quartets_fp32;
    tot.flops += ci.flops;
    tot.pairs += ci.pairs;
  }
  int n = 0;
  for (int i = 0; i < b->nlaunch; ++i)
    n += (b->launches[i].variant == 0 && b->launches[i].has_straight) ? b->launches[i].npass_live : 1;
  tot.kernel_launches = n;
  *out = tot;
  return PFE_OK;
}

int32_t pfe_context_primitive_targets(pfe_context* ctx, int32_t enable) {
  if (!ctx) { set_error("null context"); return PFE_EINVAL; }
  if (ctx->force_primitive != (enable != 0)) {
    ctx->force_primitive = enable != 0;
    ctx->ready = false;  // the next set-up rebuilds the schedule
    ctx->key = 0;
  }
  return PFE_OK;
}

int32_t pfe_context_census(pfe_context* ctx, pfe_census* out) {
  if (!ctx || !out) { set_error("null argument"); return PFE_EINVAL; }
  out->quartets = ctx->census_quartets;
  out->quartets_ref = ctx->census_ref;
  out->flops = ctx->census_flops;
  out->quartets_fp32 = 0.0;
  if (ctx->d_n32) {
    unsigned long long n32 = 0;
    PFE_CUDA(cudaMemcpy(&n32, ctx->d_n32, sizeof(n32), cudaMemcpyDeviceToHost));
    out->quartets_fp32 = (double)n32;
  }
  out->pairs = ctx->npairs;
  if (ctx->molecular) {
    // class kernels (straight-line passes), the target-space density and its check,
    // the two symmetrisations (primitive targets: the contraction is cuBLAS), the block
    // maxima under density screening or mixed precision
    int n = 0;
    for (int i = 0; i < ctx->nlaunch; ++i)
      n += (ctx->launches[i].variant == 0 && ctx->launches[i].has_straight) ? ctx->launches[i].npass_live : 1;
    n += (ctx->contracted ? 2 : 0) + 2 + ((ctx->dtol > 0.0 || ctx->mcut > 0.0) ? 1 : 0);
    out->kernel_launches = n;
  } else {
    out->kernel_launches = lattice_class_launches(ctx) + 3;
  }
  return PFE_OK;
}

int32_t pfe_context_profile(pfe_context* ctx, int32_t enable) {
  if (!ctx) { set_error("null context"); return PFE_EINVAL; }
  ctx->profile = enable != 0;
  return PFE_OK;
}

int32_t pfe_context_kernel_stats(pfe_context* ctx, pfe_kernel_stat* out, int32_t cap) {
  if (!ctx || !out) { set_error("null argument"); return PFE_EINVAL; }
  if (!ctx->profile) { set_error("profiling is off"); return PFE_EINVAL; }
  int n = 0;
  for (int i = 0; i < ctx->nprof && n < cap; ++i, ++n) {
    float ms = 0.f;
    PFE_CUDA(cudaEventElapsedTime(&ms, ctx->ev[i], ctx->ev[i + 1]));
    out[n].cls = ctx->ev_cls[i];
    out[n].variant = ctx->ev_variant[i];
    for (int v = 0; v < 4; ++v) out[n].tuned_ms[v] = ctx->ev_tuned[i][v];
    out[n].ms = ms;
    out[n].quartets = ctx->ev_quartets[i];
    out[n].flops = ctx->ev_flops[i];
    out[n].grid_mult = ctx->ev_gmul[i];
    out[n].pad_ = 0;
  }
  return n;
}

int32_t pfe_context_autotune(pfe_context* ctx, const double* d_p_p, const double* d_p_p_helix, void* stream) {
  if (!ctx || !ctx->ready) { set_error("context is not set up"); return PFE_EINVAL; }
  if (!d_p_p) { set_error("null density"); return PFE_EINVAL; }
  (void)d_p_p_helix;
  PFE_CUDA(cudaSetDevice(ctx->device));
  if (!ctx->molecular) return PFE_OK;  // the lattice path has a single schedule
  return autotune(ctx, d_p_p, (cudaStream_t)stream);
}

int32_t pfe_context_force_variant(pfe_context* ctx, int32_t variant) {
  if (!ctx || !ctx->ready) { set_error("context is not set up"); return PFE_EINVAL; }
  if (variant < 0 || variant > 3) { set_error("variant must be 0, 1, 2 or 3"); return PFE_EINVAL; }
  if (!ctx->molecular) {   // lattices: straight-line kernels where a class has them (0) or the interpreter
    lattice_force_interpreter(ctx, variant != 0);
    return PFE_OK;
  }
  for (int i = 0; i < ctx->nlaunch; ++i) {
    ClassLaunch& cl = ctx->launches[i];
    if (variant == 0 && cl.has_straight) cl.variant = 0;
    if (variant == 1 && cl.has_table && sizeof(double) * (size_t)cl.per_warp <= 200 * 1024) cl.variant = 1;
    if (variant == 2 && cl.has_table) cl.variant = 2;
    if (variant == 3 && cl.has_wide) cl.variant = 3;
  }
  ctx->tuned = true;
  return PFE_OK;
}

int32_t pfe_measure_fp64_peak(int32_t device, double* tflops) {
  if (!tflops) { set_error("null output"); return PFE_EINVAL; }
  return measure_fp64_peak(device, tflops);
}

static std::mutex g_default_mu;
static pfe_context* g_default[64] = {nullptr};
static pfe_context* g_default_prim[64] = {nullptr};  // primitive targets, for P_P that is not decontracted

int32_t pfe_fourindex_eri(const pfe_args* a, double* c_c, double* x_c) {
  std::lock_guard<std::mutex> lock(g_default_mu);
  if (!c_c || !x_c) { set_error("null output array"); return PFE_EINVAL; }
  int dev = 0;
  PFE_CUDA(cudaGetDevice(&dev));
  if (dev < 0 || dev >= 64) { set_error("device index out of range"); return PFE_EINVAL; }
  if (!g_default[dev]) {
    int rc = pfe_context_create(dev, &g_default[dev]);
    if (rc != PFE_OK) return rc;
  }
  pfe_context* ctx = g_default[dev];
  HostShells hs;
  int rc = build_host_shells(a, &hs);
  if (rc != PFE_OK) return rc;
  if (!a->p_p) { set_error("P_P is null"); return PFE_EINVAL; }
  const size_t ncell1 = (size_t)(2 * a->cel1[0] + 1) * (2 * a->cel1[1] + 1) * (2 * a->cel1[2] + 1);
  const size_t npp = (size_t)a->npgs * a->npgs * ncell1;
  if ((rc = check_density(a->p_p, npp)) != PFE_OK) return rc;
  const uint64_t key = static_key(a, hs);
  if (!(ctx->ready && ctx->key == key)) {
    if ((rc = setup_impl(ctx, a, hs, key)) != PFE_OK) { ctx->ready = false; return rc; }
  }
  cudaStream_t s = ctx->stream;
  const size_t out_bytes = sizeof(double) * (size_t)a->ncgs * a->ncgs * ncell1;
  if (ctx->pp_bytes < npp * sizeof(double)) {
    ctx->free_now(ctx->d_pp);
    PFE_CUDA(ctx->alloc((void**)&ctx->d_pp, npp * sizeof(double)));
    ctx->pp_bytes = npp * sizeof(double);
  }
  if (ctx->out_bytes < out_bytes) {
    ctx->free_now(ctx->d_out_c);
    ctx->free_now(ctx->d_out_x);
    PFE_CUDA(ctx->alloc((void**)&ctx->d_out_c, out_bytes));
    PFE_CUDA(ctx->alloc((void**)&ctx->d_out_x, out_bytes));
    ctx->out_bytes = out_bytes;
  }
  PFE_CUDA(cudaMemcpyAsync(ctx->d_pp, a->p_p, npp * sizeof(double), cudaMemcpyHostToDevice, s));
  const double* d_pph = nullptr;
  if (a->helix != 0.0) {
    if (!a->p_p_helix) { set_error("helix != 0 needs P_P_HELIX"); return PFE_EINVAL; }
    const size_t nh = (size_t)a->npgs * a->npgs * (2 * a->cel2[0] + 1) * (2 * (a->cel2[0] + a->cel1[0]) + 1);
    if ((rc = check_density(a->p_p_helix, nh)) != PFE_OK) return rc;
    if (ctx->pph_bytes < nh * sizeof(double)) {
      ctx->free_now(ctx->d_pph);
      PFE_CUDA(ctx->alloc((void**)&ctx->d_pph, nh * sizeof(double)));
      ctx->pph_bytes = nh * sizeof(double);
    }
    PFE_CUDA(cudaMemcpyAsync(ctx->d_pph, a->p_p_helix, nh * sizeof(double), cudaMemcpyHostToDevice, s));
    d_pph = ctx->d_pph;
  }
  rc = ctx->molecular ? molecular_fock(ctx, ctx->d_pp, ctx->d_out_c, ctx->d_out_x, s)
                      : lattice_fock(ctx, ctx->d_pp, d_pph, ctx->d_out_c, ctx->d_out_x, s);
  if (rc != PFE_OK) return rc;
  bool ok = true;
  if ((rc = molecular_density_ok(ctx, s, &ok)) != PFE_OK) return rc;
  if (!ok) {
    // P_P is not CC^T P_C CC: build with primitive targets, as the reference does
    if (!g_default_prim[dev]) {
      if ((rc = pfe_context_create(dev, &g_default_prim[dev])) != PFE_OK) return rc;
      g_default_prim[dev]->force_primitive = true;
    }
    pfe_context* pc = g_default_prim[dev];
    if (!(pc->ready && pc->key == key)) {
      if ((rc = setup_impl(pc, a, hs, key)) != PFE_OK) { pc->ready = false; return rc; }
    }
    PFE_CUDA(cudaStreamSynchronize(s));
    if ((rc = molecular_fock(pc, ctx->d_pp, ctx->d_out_c, ctx->d_out_x, pc->stream)) != PFE_OK) return rc;
    PFE_CUDA(cudaStreamSynchronize(pc->stream));
  }
  PFE_CUDA(cudaMemcpyAsync(c_c, ctx->d_out_c, out_bytes, cudaMemcpyDeviceToHost, s));
  PFE_CUDA(cudaMemcpyAsync(x_c, ctx->d_out_x, out_bytes, cudaMemcpyDeviceToHost, s));
  PFE_CUDA(cudaStreamSynchronize(s));
  return PFE_OK;
}

int32_t pfe_fourindex_eri_gradient(const pfe_args* a, const int32_t* pgs_atom, int32_t natom, double* grad_j,
                                   double* grad_k) {
  std::lock_guard<std::mutex> lock(g_default_mu);
  if (!grad_j || !grad_k || !pgs_atom || natom <= 0) { set_error("invalid gradient arguments"); return PFE_EINVAL; }
  int dev = 0;
  PFE_CUDA(cudaGetDevice(&dev));
  if (dev < 0 || dev >= 64) { set_error("device index out of range"); return PFE_EINVAL; }
  if (!g_default[dev]) {
    int rc = pfe_context_create(dev, &g_default[dev]);
    if (rc != PFE_OK) return rc;
  }
  pfe_context* ctx = g_default[dev];
  HostShells hs;
  int rc = build_host_shells(a, &hs);
  if (rc != PFE_OK) return rc;
  if (!a->p_p) { set_error("P_P is null"); return PFE_EINVAL; }
  const bool molecule = a->cel1[0] == 0 && a->cel1[1] == 0 && a->cel1[2] == 0 && a->cel2[0] == 0 &&
                        a->cel2[1] == 0 && a->cel2[2] == 0 && a->helix == 0.0;
  if (!molecule) {
    set_error("the two-electron gradient is implemented for molecules (no lattice, no helix)");
    return PFE_EUNSUPPORTED;
  }
  std::vector<int> satom(a->npshell);
  for (int sh = 0; sh < a->npshell; ++sh) {
    const int at = pgs_atom[hs.head[sh]] - 1;
    if (at < 0 || at >= natom) { set_error("PGS_ATOM outside 1..natom"); return PFE_EINVAL; }
    satom[sh] = at;
  }
  const size_t npp = (size_t)a->npgs * a->npgs;
  if ((rc = check_density(a->p_p, npp)) != PFE_OK) return rc;
  const uint64_t key = static_key(a, hs);
  if (!(ctx->ready && ctx->key == key)) {
    if ((rc = setup_impl(ctx, a, hs, key)) != PFE_OK) { ctx->ready = false; return rc; }
  }
  cudaStream_t s = ctx->stream;
  if (ctx->pp_bytes < npp * sizeof(double)) {
    ctx->free_now(ctx->d_pp);
    PFE_CUDA(ctx->alloc((void**)&ctx->d_pp, npp * sizeof(double)));
    ctx->pp_bytes = npp * sizeof(double);
  }
  PFE_CUDA(cudaMemcpyAsync(ctx->d_pp, a->p_p, npp * sizeof(double), cudaMemcpyHostToDevice, s));
  int* d_satom = nullptr;
  double* d_g = nullptr;
  PFE_CUDA(ctx->alloc((void**)&d_satom, sizeof(int) * a->npshell));
  PFE_CUDA(ctx->alloc((void**)&d_g, sizeof(double) * 6 * (size_t)natom));
  PFE_CUDA(cudaMemcpyAsync(d_satom, satom.data(), sizeof(int) * a->npshell, cudaMemcpyHostToDevice, s));
  rc = molecular_gradient_pp(ctx, ctx->d_pp, d_satom, natom, d_g, d_g + 3 * (size_t)natom, s);
  bool ok = true;
  if (rc == PFE_OK) rc = molecular_density_ok(ctx, s, &ok);
  if (rc == PFE_OK && !ok) {
    set_error("pfe_fourindex_eri_gradient: P_P is not CC^T P_C CC (the gradient reads contracted targets)");
    rc = PFE_EINVAL;
  }
  if (rc == PFE_OK) {
    PFE_CUDA(cudaMemcpyAsync(grad_j, d_g, sizeof(double) * 3 * (size_t)natom, cudaMemcpyDeviceToHost, s));
    PFE_CUDA(cudaMemcpyAsync(grad_k, d_g + 3 * (size_t)natom, sizeof(double) * 3 * (size_t)natom,
                             cudaMemcpyDeviceToHost, s));
    PFE_CUDA(cudaStreamSynchronize(s));
  }
  PFE_CUDA(cudaStreamSynchronize(s));
  ctx->free_now(d_satom);
  ctx->free_now(d_g);
  return rc;
}


}  // extern "C"
