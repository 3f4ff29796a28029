// Molecular path of the Fock build (all cells 0, HELIX 0).
//
// Work is organised by contracted shell quartets.  A "group" is the run of
// primitive-shell pairs of one ordered contracted block pair (the primitive
// shells of one contracted shell share centre, angular type and target rows);
// a "group quartet" (G|H) holds every primitive quartet of a bra group and a
// ket group.
//
// Set-up (device):
//   * every unordered primitive-shell pair, oriented higher L first, then
//     higher block, then higher shell index, with the reference's Schwarz bound
//     (component 1 excluded, src/pfourindexdirect.f90:326-363);
//   * pairs sorted by (class, group maximum desc, group, bound desc): groups are
//     contiguous runs, each sorted by bound, and within a class the groups a
//     bra can reach form a prefix;
//   * ket groups of every class listed by size bucket (similar primitive counts
//     side by side); per (bra class, ket class) chunks of one bra group and up
//     to 32 ket groups of one bucket, cut by the group maxima (the reference's
//     screen IJIJ*KLKL < INTTOL, src/pfourindexdirect.f90:529, can only pass
//     inside that prefix).
// Build:
//   * the density in target space: contracted P_C read off P_P at one primitive
//     per contracted function (checked against every element of P_P), or P_P
//     itself when CC is a general contraction;
//   * per class one kernel: every primitive quartet of a group quartet passing
//     the reference's screen is evaluated (tabulated Boys function, generated
//     HGP recursion) and contracted, with its coefficients and its 8-fold
//     symmetry weight, into X(abcd) of the group quartet; X is then digested
//     once against the target-space density into J'/K' (FP64 atomics; the
//     bra's J' warp-reduced first).  Straight-line code with one group quartet
//     per lane, or the op-table interpreter with one (warp) or all (block)
//     threads per primitive quartet and X in shared memory;
//   * C_C = J' + J'^T and X_C = K' + K'^T (contracted targets), or the cuBLAS
//     contraction CC (J'+J'^T) CC^T for primitive targets.

#include <cublas_v2.h>
#include <cub/cub.cuh>

#include <algorithm>
#include <vector>

#include "pfe_common.cuh"
#include "pfe_context.cuh"
#include "pfe_interp.cuh"
#include "generated/eri_classes.cuh"
#include "pfe_mol_kernels.cuh"
#include "pfe_mol_wide.cuh"

namespace pfe {

constexpr int NBUCKET = 6;   // ket-group size buckets: 1, 2-3, 4-7, 8-15, 16-31, 32+

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

__global__ void k_pack_pairs(PairArrays pr, PairRec* __restrict__ rec, long long n) {
  const long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (t >= n) return;
  PairRec r;
  for (int k = 0; k < 3; ++k) { r.P[k] = pr.P[k][t]; r.PA[k] = pr.PA[k][t]; r.AB[k] = pr.AB[k][t]; }
  r.zeta = pr.zeta[t];
  r.S = pr.S[t];
  r.schwarz = pr.schwarz[t];
  r.si = pr.si[t];
  r.sj = pr.sj[t];
  r.oz = 0.5 / r.zeta;
  r.pad[0] = r.pad[1] = 0.0;
  rec[t] = r;
}

// ------------------------------------------------------------------ groups and chunks

__global__ void k_group_heads(const int* __restrict__ gid, int* __restrict__ head, long long n) {
  const long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (t < n) head[t] = (t == 0 || gid[t] != gid[t - 1]) ? 1 : 0;
}

__global__ void k_group_fill(const int* __restrict__ head, const int* __restrict__ gix, const double* __restrict__ sch,
                             const unsigned char* __restrict__ cls, int* __restrict__ gr_start,
                             double* __restrict__ gr_max, unsigned char* __restrict__ gr_cls, long long n) {
  const long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (t >= n || !head[t]) return;
  const int g = gix[t];
  gr_start[g] = (int)t;
  gr_max[g] = sch[t];   // a group is sorted by bound, descending
  gr_cls[g] = cls[t];
}

__device__ __forceinline__ int size_bucket(int n) { return min(NBUCKET - 1, 31 - __clz(max(n, 1))); }

__global__ void k_group_size(const int* __restrict__ gr_start, const unsigned char* __restrict__ gr_cls, int ngroups,
                             long long npairs, int* __restrict__ gr_n, unsigned char* __restrict__ bkey) {
  const int g = blockIdx.x * blockDim.x + threadIdx.x;
  if (g >= ngroups) return;
  const int n = (int)((g + 1 < ngroups ? (long long)gr_start[g + 1] : npairs) - gr_start[g]);
  gr_n[g] = n;
  bkey[g] = (unsigned char)(gr_cls[g] * 8 + size_bucket(n));
}

struct Segs {
  int s0[NBUCKET], s1[NBUCKET];
};

// End (exclusive list position) of the ket groups of bucket segment [s0, s1)
// that bra group G can reach: group maxima are non-increasing along a segment;
// for one class only groups up to G itself (the triangle).
__device__ __forceinline__ int reach_end(const double* __restrict__ gr_max, const int* __restrict__ bk_list, int s0,
                                         int s1, double gmx, int G, bool same, double inttol) {
  int lo = s0, hi = s1;
  while (lo < hi) {
    const int mid = (lo + hi) >> 1;
    if (gmx * gr_max[bk_list[mid]] < inttol) hi = mid; else lo = mid + 1;
  }
  int e = lo;
  if (same) {
    int l2 = s0, h2 = e;
    while (l2 < h2) {
      const int mid = (l2 + h2) >> 1;
      if (bk_list[mid] <= G) l2 = mid + 1; else h2 = mid;
    }
    e = l2;
  }
  return e;
}

__global__ void k_chunk_count(const double* __restrict__ gr_max, const int* __restrict__ bk_list, int g0, int ng,
                              Segs sg, bool same, double inttol, int* __restrict__ nchunk) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= ng) return;
  const int G = g0 + i;
  const double gmx = gr_max[G];
  int n = 0;
  for (int b = 0; b < NBUCKET; ++b) {
    if (sg.s0[b] >= sg.s1[b]) continue;
    const int e = reach_end(gr_max, bk_list, sg.s0[b], sg.s1[b], gmx, G, same, inttol);
    n += (e - sg.s0[b] + 31) >> 5;
  }
  nchunk[i] = n;
}

__global__ void k_chunk_fill(const double* __restrict__ gr_max, const int* __restrict__ bk_list, int g0, int ng,
                             Segs sg, bool same, double inttol, const int* __restrict__ off, int4* __restrict__ chunks) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= ng) return;
  const int G = g0 + i;
  const double gmx = gr_max[G];
  int o = off[i];
  for (int b = 0; b < NBUCKET; ++b) {
    if (sg.s0[b] >= sg.s1[b]) continue;
    const int e = reach_end(gr_max, bk_list, sg.s0[b], sg.s1[b], gmx, G, same, inttol);
    for (int k = sg.s0[b]; k < e; k += 32) chunks[o++] = make_int4(G, k, min(k + 32, e), 0);
  }
}

// Primitive quartets of every chunk that pass the screen (the census): lane per
// ket group, binary search over each ket group's bound-sorted pairs.
// Screened primitive quartets of every chunk (its cost, also the sort key of
// the work queue) and their total.
__global__ void k_chunk_census(const int4* __restrict__ chunks, int nchunks, const int* __restrict__ bk_list,
                               const int* __restrict__ gr_start, const int* __restrict__ gr_n,
                               const double* __restrict__ sch, double inttol, unsigned long long* __restrict__ total,
                               unsigned int* __restrict__ cost) {
  const int c = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
  const int lane = threadIdx.x & 31;
  if (c >= nchunks) return;
  const int4 ch = chunks[c];
  unsigned long long n = 0;
  const int li = ch.y + lane;
  if (li < ch.z) {
    const int G = ch.x, H = bk_list[li];
    const int g0 = gr_start[G], gn = gr_n[G], h0 = gr_start[H], hn = gr_n[H];
    for (int p = g0; p < g0 + gn; ++p) {
      const double sp = sch[p];
      const int qe = (G == H) ? p + 1 : h0 + hn;
      int lo = h0, hi = qe;
      while (lo < hi) {
        const int mid = (lo + hi) >> 1;
        if (sp * sch[mid] < inttol) hi = mid; else lo = mid + 1;
      }
      n += (unsigned long long)(lo - h0);
    }
  }
  for (int o = 16; o > 0; o >>= 1) n += __shfl_xor_sync(0xffffffffu, n, o);
  if (lane == 0) {
    if (n) atomicAdd(total, n);
    cost[c] = (unsigned int)min(n, 0xffffffffull);
  }
}

// ------------------------------------------------------------------ density in target space

// P_T(mu, nu) = P_P(r_mu, r_nu) / (c_mu c_nu) at the representative primitives.
__global__ void k_target_density(const double* __restrict__ pp, int npgs, const int* __restrict__ rep,
                                 const double* __restrict__ repc, int nt, double* __restrict__ pt) {
  const long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (t >= (long long)nt * nt) return;
  const int mu = (int)(t % nt), nu = (int)(t / nt);
  const int a = rep[mu], b = rep[nu];
  pt[t] = (a >= 0 && b >= 0) ? pp[a + (size_t)npgs * b] / (repc[mu] * repc[nu]) : 0.0;
}

// Every P_P(a,b) must equal c_a c_b P_T(t_a, t_b) (zero for primitives without a
// coefficient) to rounding; otherwise the flag is raised.
__global__ void k_check_density(const double* __restrict__ pp, int npgs, const int* __restrict__ tidx,
                                const double* __restrict__ tcoef, const double* __restrict__ pt, int nt,
                                unsigned int* __restrict__ flag) {
  const long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (t >= (long long)npgs * npgs) return;
  const int a = (int)(t % npgs), b = (int)(t / npgs);
  const int ta = tidx[a], tb = tidx[b];
  const double want = (ta >= 0 && tb >= 0) ? tcoef[a] * tcoef[b] * pt[ta + (size_t)nt * tb] : 0.0;
  const double got = pp[t];
  if (!(fabs(got - want) <= 1e-12 * fmax(fabs(got), fabs(want)))) atomicOr(flag, 1u);
}

// Block-pair maxima of |P_T|, as the bit patterns of non-negative doubles.
__global__ void k_block_dmax(const double* __restrict__ D, int nt, const int* __restrict__ tblk, int nblk,
                             unsigned long long* __restrict__ bmax) {
  const long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (t >= (long long)nt * nt) return;
  const int b1 = tblk[t % nt], b2 = tblk[t / nt];
  if (b1 < 0 || b2 < 0) return;
  const double v = fabs(D[t]);
  if (v > 0.0) atomicMax(bmax + (size_t)b1 * nblk + b2, (unsigned long long)__double_as_longlong(v));
}

// ------------------------------------------------------------------ interpreted classes

// Digestion of a contracted X(abcd) into the targets of one group quartet,
// target t in [0, NT): J'(ab), J'(cd), K'(ad), K'(bd), K'(ac), K'(bc).
template <int NA, int NB, int NC, int ND>
struct Digest {
  static constexpr int NT = NA * NB + NC * ND + (NA + NB) * (NC + ND);
  static constexpr int SB = NA, SC = NA + NB, SD = NA + NB + NC;
  static constexpr int NP = NA * NB + NC * ND + NA * NC + NA * ND + NB * NC + NB * ND;
  // density blocks in shared memory: Pab | Pcd | Pac | Pad | Pbc | Pbd
  static constexpr int OAB = 0, OCD = NA * NB, OAC = OCD + NC * ND, OAD = OAC + NA * NC, OBC = OAD + NA * ND,
                       OBD = OBC + NB * NC;
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
  __device__ static double value(int t, const double* __restrict__ X, const double* __restrict__ P) {
    double acc = 0.0;
    int r = t;
    if (r < NA * NB) {
      const int a = r / NB, b = r % NB;
      for (int cd = 0; cd < NC * ND; ++cd) acc = fma(P[OCD + cd], X[(a * NB + b) * NC * ND + cd], acc);
      return 0.25 * acc;
    }
    r -= NA * NB;
    if (r < NC * ND) {
      for (int ab = 0; ab < NA * NB; ++ab) acc = fma(P[OAB + ab], X[ab * NC * ND + r], acc);
      return 0.25 * acc;
    }
    r -= NC * ND;
    if (r < NA * ND) {
      const int a = r / ND, d = r % ND;
      for (int b = 0; b < NB; ++b)
        for (int cc = 0; cc < NC; ++cc) acc = fma(P[OBC + b * NC + cc], X[((a * NB + b) * NC + cc) * ND + d], acc);
      return 0.125 * acc;
    }
    r -= NA * ND;
    if (r < NB * ND) {
      const int b = r / ND, d = r % ND;
      for (int a = 0; a < NA; ++a)
        for (int cc = 0; cc < NC; ++cc) acc = fma(P[OAC + a * NC + cc], X[((a * NB + b) * NC + cc) * ND + d], acc);
      return 0.125 * acc;
    }
    r -= NB * ND;
    if (r < NA * NC) {
      const int a = r / NC, cc = r % NC;
      for (int b = 0; b < NB; ++b)
        for (int d = 0; d < ND; ++d) acc = fma(P[OBD + b * ND + d], X[((a * NB + b) * NC + cc) * ND + d], acc);
      return 0.125 * acc;
    }
    r -= NA * NC;
    const int b = r / NC, cc = r % NC;
    for (int a = 0; a < NA; ++a)
      for (int d = 0; d < ND; ++d) acc = fma(P[OAD + a * ND + d], X[((a * NB + b) * NC + cc) * ND + d], acc);
    return 0.125 * acc;
  }
};

// Shared-memory layout of one interpreter team (a warp or a block), in doubles:
// v[nslots] | P blocks[NP] | cab[NA*NB] | ccd[NC*ND] | X[NI] (X only when it is
// not in global scratch: the (22|22) working set exceeds shared memory)
template <int LA, int LB, int LC, int LD>
struct TeamLayout {
  static constexpr int NA = ncum(LA), NB = ncum(LB), NC = ncum(LC), ND = ncum(LD);
  static constexpr int NI = NA * NB * NC * ND;
  static __host__ __device__ int doubles(int nslots, bool x_in_smem) {
    return nslots + Digest<NA, NB, NC, ND>::NP + NA * NB + NC * ND + (x_in_smem ? NI : 0);
  }
};

// Team-cooperative evaluation of the group quartets of one chunk: all threads
// of the team (a warp, or the block) share one primitive quartet at a time and
// run the op table level by level; X accumulates in shared (or global) memory.
template <int LA, int LB, int LC, int LD, bool BLOCK>
__device__ __forceinline__ void gq_team(const MolLaunch& ql, const OpTableDev& tab, const int4 ch, double* sm,
                                        double* xg, OpGeom& geo, int* prm, double* sw, int tid, int team) {
  constexpr int NA = ncum(LA), NB = ncum(LB), NC = ncum(LC), ND = ncum(LD);
  constexpr int NI = NA * NB * NC * ND;
  constexpr int NCD = NC * ND;
  constexpr int LT = LA + LB + LC + LD;
  using DG = Digest<NA, NB, NC, ND>;
  auto sync = [&]() { if constexpr (BLOCK) __syncthreads(); else __syncwarp(); };
  double* v = sm;
  double* P = v + tab.nslots;
  double* cab = P + DG::NP;
  double* ccd = cab + NA * NB;
  double* X = xg ? xg : ccd + NCD;
  const PairArrays pr = ql.pairs;
  const int nt = ql.nt;
  const double* __restrict__ D = ql.dt;
  const double* __restrict__ scoef = ql.scoef;   // held in registers (ql may live in global memory)
  const double* __restrict__ boys = ql.boys;
  const double c2pi = 2.0 / sqrt(REF_PI);
  const int G = ch.x;
  const int g0 = ql.gr_start[G], gn = ql.gr_n[G];
  {
    const int I0 = pr.si[g0], J0 = pr.sj[g0];
    for (int x = tid; x < NA; x += team) prm[x] = ql.stidx[I0 * MAXCOMP + x];
    for (int x = tid; x < NB; x += team) prm[DG::SB + x] = ql.stidx[J0 * MAXCOMP + x];
  }
  sync();
  // bra shells whose lower components carry no coefficient (pure p or d) take
  // the pure-bra table: the outputs it drops would be weighted by zero
  bool pure = tab.ops_p != nullptr;
  for (int x = 0; pure && x < NA; ++x)
    if (comp_tot(LA, x) < LA && prm[x] >= 0) pure = false;
  for (int x = 0; pure && x < NB; ++x)
    if (comp_tot(LB, x) < LB && prm[DG::SB + x] >= 0) pure = false;
  const unsigned short* __restrict__ b_ops = pure ? tab.ops_p : tab.ops;
  const int* __restrict__ b_levels = pure ? tab.levels_p : tab.levels;
  const unsigned short* __restrict__ b_out = pure ? tab.out_p : tab.out;
  const int b_nlevels = pure ? tab.nlevels_p : tab.nlevels;
  pure = pure && tab.ops_p2 != nullptr;   // from here: the bra-and-ket table may apply
  for (int t = tid; t < NA * NB; t += team)
    P[DG::OAB + t] = dt_at(D, nt, prm[t / NB], prm[DG::SB + t % NB]);
  for (int k = ch.y; k < ch.z; ++k) {
    const int H = ql.bk_list[k];
    const int h0 = ql.gr_start[H], hn = ql.gr_n[H];
    const double hmax = ql.gr_max[H];
    const double thr = quartet_threshold(
        ql, ql.dtol > 0.0 ? quartet_pmax(ql, pr.si[g0], pr.sj[g0], pr.si[h0], pr.sj[h0]) : 0.0);
    if (ql.gr_max[G] * hmax < thr) continue;   // no quartet of (G|H) passes (team-uniform)
    {
      const int K0 = pr.si[h0], L0 = pr.sj[h0];
      for (int x = tid; x < NC; x += team) prm[DG::SC + x] = ql.stidx[K0 * MAXCOMP + x];
      for (int x = tid; x < ND; x += team) prm[DG::SD + x] = ql.stidx[L0 * MAXCOMP + x];
    }
    for (int i = tid; i < NI; i += team) X[i] = 0.0;
    sync();
    {
      const int* pa = prm;
      const int* pb = prm + DG::SB;
      const int* pc = prm + DG::SC;
      const int* pd = prm + DG::SD;
      for (int t = tid; t < NC * ND; t += team) P[DG::OCD + t] = dt_at(D, nt, pc[t / ND], pd[t % ND]);
      for (int t = tid; t < NA * NC; t += team) P[DG::OAC + t] = dt_at(D, nt, pa[t / NC], pc[t % NC]);
      for (int t = tid; t < NA * ND; t += team) P[DG::OAD + t] = dt_at(D, nt, pa[t / ND], pd[t % ND]);
      for (int t = tid; t < NB * NC; t += team) P[DG::OBC + t] = dt_at(D, nt, pb[t / NC], pc[t % NC]);
      for (int t = tid; t < NB * ND; t += team) P[DG::OBD + t] = dt_at(D, nt, pb[t / ND], pd[t % ND]);
    }
    sync();   // the blocks are read by the digestion, which may follow with no quartet in between
    // pure bra and pure ket shells take the table that drops both sides' lower
    // components (team-uniform: prm is shared)
    bool pure2 = pure;
    for (int x = 0; pure2 && x < NC; ++x)
      if (comp_tot(LC, x) < LC && prm[DG::SC + x] >= 0) pure2 = false;
    for (int x = 0; pure2 && x < ND; ++x)
      if (comp_tot(LD, x) < LD && prm[DG::SD + x] >= 0) pure2 = false;
    const unsigned short* __restrict__ t_ops = pure2 ? tab.ops_p2 : b_ops;
    const int* __restrict__ t_levels = pure2 ? tab.levels_p2 : b_levels;
    const unsigned short* __restrict__ t_out = pure2 ? tab.out_p2 : b_out;
    const int t_nlevels = pure2 ? tab.nlevels_p2 : b_nlevels;
    bool any = false;   // team-uniform: every loop decision below is
    for (int p = g0; p < g0 + gn; ++p) {
      const double sp = pr.schwarz[p];
      if (sp * hmax < thr) break;
      const int I = pr.si[p], J = pr.sj[p];
      for (int t = tid; t < NA * NB; t += team)
        cab[t] = scoef[I * MAXCOMP + t / NB] * scoef[J * MAXCOMP + t % NB];
      const double zb = pr.zeta[p];
      const double Px = pr.P[0][p], Py = pr.P[1][p], Pz = pr.P[2][p];
      const int qe = (G == H) ? p + 1 : h0 + hn;
      for (int q = h0; q < qe; ++q) {
        if (sp * pr.schwarz[q] < thr) break;   // the reference's screen (thr = INTTOL; team-uniform)
        const int K = pr.si[q], L = pr.sj[q];
        const double ze = pr.zeta[q];
        const double Qx = pr.P[0][q], Qy = pr.P[1][q], Qz = pr.P[2][q];
        const double zz = zb + ze, rho = zb * ze / zz;
        if (tid == 0) {
          const double T = rho * ((Px - Qx) * (Px - Qx) + (Py - Qy) * (Py - Qy) + (Pz - Qz) * (Pz - Qz));
          const double pref = c2pi * pr.S[p] * pr.S[q] * sqrt(rho);
          double F[LT + 1];
          boys_tab<LT>(T, pref, boys, F);
          v[0] = 0.0;
#pragma unroll
          for (int m = 0; m <= LT; ++m) v[1 + m] = F[m];
          sw[0] = ((I != J) ? 2.0 : 1.0) * ((K != L) ? 2.0 : 1.0) * ((p != q) ? 2.0 : 1.0);
        } else if (tid == 1) {
          const double W[3] = {(zb * Px + ze * Qx) / zz, (zb * Py + ze * Qy) / zz, (zb * Pz + ze * Qz) / zz};
          const double Pv[3] = {Px, Py, Pz}, Qv[3] = {Qx, Qy, Qz};
          double PA[3], QC[3], AB[3], CD[3], WP[3], WQ[3];
          for (int k2 = 0; k2 < 3; ++k2) {
            PA[k2] = pr.PA[k2][p]; QC[k2] = pr.PA[k2][q]; AB[k2] = pr.AB[k2][p]; CD[k2] = pr.AB[k2][q];
            WP[k2] = W[k2] - Pv[k2]; WQ[k2] = W[k2] - Qv[k2];
          }
          set_geom(geo, PA, WP, QC, WQ, AB, CD, 0.5 / zb, 0.5 / ze, 0.5 / zz, rho / zb, rho / ze);
        }
        for (int t = tid; t < NCD; t += team)
          ccd[t] = scoef[K * MAXCOMP + t / ND] * scoef[L * MAXCOMP + t % ND];
        sync();
        for (int l = 0; l < t_nlevels; ++l) {
          const int o0 = t_levels[l], o1 = t_levels[l + 1];
          run_level(t_ops, o0, o1, v, geo, tid, team, EvalD{});
          sync();
        }
        const double w = sw[0];
        for (int i = tid; i < NI; i += team) X[i] = fma(w * cab[i / NCD] * ccd[i % NCD], v[t_out[i]], X[i]);
        any = true;
        sync();
      }
    }
    // digestion of the group quartet
    for (int t = tid; any && t < DG::NT; t += team) {
      int kind, s1, s2;
      DG::slots(t, &kind, &s1, &s2);
      add_target(kind == 0 ? ql.jt : ql.kt, nt, prm[s1], prm[s2], DG::value(t, X, P));
    }
    sync();
  }
}

template <int LA, int LB, int LC, int LD>
__global__ void __launch_bounds__(256) k_gq_warp(MolLaunch ql, OpTableDev tab, int per_warp) {
  constexpr int NPRM = ncum(LA) + ncum(LB) + ncum(LC) + ncum(LD);
  extern __shared__ double smem[];
  __shared__ OpGeom s_geo[8];
  __shared__ int s_prm[8][NPRM];
  __shared__ double s_w[8];
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, wpb = blockDim.x >> 5;
  const int nchunks = *ql.nchunks;
  const int stride = gridDim.x * wpb * ql.numprocs;
  for (int c = (blockIdx.x * wpb + wid) * ql.numprocs + ql.myid; c < nchunks; c += stride) {
    const int4 ch = ql.chunks[c];
    gq_team<LA, LB, LC, LD, false>(ql.insts ? ql.insts[ch.w] : ql, tab, ch, smem + (size_t)wid * per_warp, nullptr,
                                   s_geo[wid], s_prm[wid], s_w + wid, lane, 32);
  }
}

// xg: per-block X scratch in global memory (gridDim.x * NI doubles), or null
// for X in shared memory.
template <int LA, int LB, int LC, int LD>
__global__ void __launch_bounds__(256) k_gq_block(MolLaunch ql, OpTableDev tab, double* xg) {
  constexpr int NPRM = ncum(LA) + ncum(LB) + ncum(LC) + ncum(LD);
  extern __shared__ double smem[];
  __shared__ OpGeom s_geo;
  __shared__ int s_prm[NPRM];
  __shared__ double s_w[1];
  const int nchunks = *ql.nchunks;
  for (int c = blockIdx.x * ql.numprocs + ql.myid; c < nchunks; c += gridDim.x * ql.numprocs)
    gq_team<LA, LB, LC, LD, true>(ql.insts ? ql.insts[ql.chunks[c].w] : ql, tab, ql.chunks[c], smem,
                                  xg ? xg + (size_t)blockIdx.x * (ncum(LA) * ncum(LB) * ncum(LC) * ncum(LD)) : nullptr,
                                  s_geo, s_prm, s_w, threadIdx.x, blockDim.x);
}

// FP64 straight-line launchers here; the mixed-precision ones in pfe_mol_mixed.cu,
// those of batches (launch records per chunk) in pfe_mol_batch*.cu
LaunchFn straight_launcher_mixed(int cb, int ck);
LaunchFn straight_launcher_batch(int cb, int ck);
LaunchFn straight_launcher_batch_mixed(int cb, int ck);

// (classes without a mixed instantiation run their FP64 straight-line kernels)
static LaunchFn straight_launcher(int cb, int ck, bool mixed = false, bool batch = false) {
  LaunchFn f = nullptr;
  if (batch) {
    f = mixed ? straight_launcher_batch_mixed(cb, ck) : nullptr;
    if (!f) f = straight_launcher_batch(cb, ck);
    if (!f) f = straight_launcher_big(cb, ck, true);
    return f;
  }
  f = mixed ? straight_launcher_mixed(cb, ck) : nullptr;
  if (!f) f = straight_launcher_t<false>(cb, ck);
  if (!f) f = straight_launcher_big(cb, ck);
  return f;
}

using BigFn = void (*)(const MolLaunch&, const OpTableDev&, double* xg, int grid, size_t smem, cudaStream_t);
using WarpFn = void (*)(const MolLaunch&, const OpTableDev&, int grid, int wpb, int per_warp, size_t smem, cudaStream_t);

template <int LA, int LB, int LC, int LD>
static void launch_big(const MolLaunch& ql, const OpTableDev& t, double* xg, int grid, size_t smem, cudaStream_t s) {
  k_gq_block<LA, LB, LC, LD><<<grid, 256, smem, s>>>(ql, t, xg);
}

template <int LA, int LB, int LC, int LD>
static void launch_warp(const MolLaunch& ql, const OpTableDev& t, int grid, int wpb, int per_warp, size_t smem,
                        cudaStream_t s) {
  k_gq_warp<LA, LB, LC, LD><<<grid, 32 * wpb, smem, s>>>(ql, t, per_warp);
}

template <int LA, int LB, int LC, int LD>
static cudaError_t allow_smem_both(size_t big, size_t warp) {
  cudaError_t e = cudaFuncSetAttribute(k_gq_block<LA, LB, LC, LD>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)big);
  if (e != cudaSuccess) return e;
  return cudaFuncSetAttribute(k_gq_warp<LA, LB, LC, LD>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)warp);
}

template <int LA, int LB, int LC, int LD>
static int team_doubles(int nslots, bool x_in_smem) { return TeamLayout<LA, LB, LC, LD>::doubles(nslots, x_in_smem); }

struct Variants {
  BigFn big;
  WarpFn warp;
  cudaError_t (*allow)(size_t, size_t);
  int (*doubles)(int, bool);
};

static Variants variants(int cb, int ck) {
#define V(A, B, C, D) \
  Variants{&launch_big<A, B, C, D>, &launch_warp<A, B, C, D>, &allow_smem_both<A, B, C, D>, &team_doubles<A, B, C, D>}
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
    default: return Variants{nullptr, nullptr, nullptr, nullptr};
  }
#undef V
}

// ------------------------------------------------------------------ set-up

template <typename KeyT>
static int radix_sort_pairs(pfe_context* ctx, const KeyT* kin, KeyT* kout, const int* vin, int* vout, int n, int bits,
                            cudaStream_t s) {
  size_t tb = 0;
  cub::DeviceRadixSort::SortPairs(nullptr, tb, kin, kout, vin, vout, n, 0, bits, s);
  void* tmp = nullptr;
  PFE_CUDA(ctx->alloc(&tmp, tb + 16));
  PFE_CUDA(cub::DeviceRadixSort::SortPairs(tmp, tb, kin, kout, vin, vout, n, 0, bits, s));
  ctx->free_later(tmp);
  return PFE_OK;
}

static int exclusive_sum(pfe_context* ctx, const int* in, int* out, int n, cudaStream_t s) {
  size_t tb = 0;
  cub::DeviceScan::ExclusiveSum(nullptr, tb, in, out, n, s);
  void* tmp = nullptr;
  PFE_CUDA(ctx->alloc(&tmp, tb + 16));
  PFE_CUDA(cub::DeviceScan::ExclusiveSum(tmp, tb, in, out, n, s));
  ctx->free_later(tmp);
  return PFE_OK;
}

// Shared memory of the wide variant (pfe_mol_wide.cu) for this molecule's
// shells: the slots of the largest op table one of its group quartets can take
// (the pure-bra or bra-and-ket table when no shell of the bra or ket kind has a
// target on a lower component) and the kept outputs of its largest group
// quartet; warps per block chosen for the most resident warps per SM.
// bit L: some shell of top angular momentum L has a coefficient on a lower component
static int lower_kept_bits(const pfe_context* ctx) {
  int bits = 0;
  for (int L = 0; L < 3; ++L) bits |= ctx->lower_kept[L] ? (1 << L) : 0;
  return bits;
}

static int size_wide(ClassLaunch& cl, const int kept_max[3], const bool lower_kept[3]) {
  cl.has_wide = false;
  const WideVariant wv = wide_variant(cl.cb, cl.ck);
  if (!wv.launch || !cl.has_table) return PFE_OK;
  const int la = kCL[cl.cb][0], lb = kCL[cl.cb][1], lc = kCL[cl.ck][0], ld = kCL[cl.ck][1];
  const bool bra_full = !cl.ops_p || lower_kept[la] || lower_kept[lb];
  const bool ket_full = lower_kept[lc] || lower_kept[ld] || !cl.ops_p2;
  const int vmax = bra_full ? cl.nslots : (ket_full ? cl.nslots_p : cl.nslots_p2);
  auto km = [&](int L) { return std::max(kept_max[L], 1); };
  const int xmax = km(la) * km(lb) * km(lc) * km(ld);
  const size_t pw = sizeof(double) * (size_t)wv.doubles(vmax, xmax);
  // at most 160 KB of shared memory per SM: the rest of the SM's 256 KB stays
  // L1, which then holds the op table the warps read their op records from
  // (61 KB for the pure-bra (dd|dp) table)
  const size_t cap = 160 * 1024;
  int best = 0, best_w = 0;
  for (int w = 1; w <= 8; ++w) {
    if (w * pw > cap) break;
    const int resident = w * (int)(cap / (w * pw));
    if (resident > best_w) { best_w = resident; best = w; }
  }
  if (best == 0 && pw <= 227 * 1024) best = 1;   // one warp per block where 160 KB is too little
  if (best == 0) return PFE_OK;   // does not fit: the class keeps its other variants
  cl.wide_vmax = vmax;
  cl.wide_xmax = xmax;
  cl.wide_per_warp = (int)(pw / sizeof(double));
  cl.wide_wpb = best;
  cl.smem_wide = pw * best;
  PFE_CUDA(wv.allow(cl.smem_wide));
  cl.has_wide = true;
  return PFE_OK;
}

int molecular_setup(pfe_context* ctx, const pfe_args* a) {
  (void)a;
  cudaStream_t s = ctx->stream;
  const int nsh = ctx->npshell;
  const long long npairs = (long long)nsh * (nsh + 1) / 2;
  if (npairs >= (1LL << 31)) { set_error("too many shell pairs for 32-bit pair indices"); return PFE_EINVAL; }
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
  // sort by (class, group maximum desc, group, bound desc): four stable radix passes
  const long long ngid = (long long)ctx->nblk * ctx->nblk;
  unsigned long long *gbits = nullptr, *k_sch = nullptr, *k_gmax = nullptr, *k64 = nullptr;
  int *perm_a = nullptr, *perm_b = nullptr, *k32 = nullptr, *k32b = nullptr;
  unsigned char *k8 = nullptr, *k8b = nullptr;
  PFE_CUDA(ctx->alloc((void**)&gbits, sizeof(unsigned long long) * ngid));
  PFE_CUDA(ctx->alloc((void**)&k_sch, sizeof(unsigned long long) * npairs));
  PFE_CUDA(ctx->alloc((void**)&k_gmax, sizeof(unsigned long long) * npairs));
  PFE_CUDA(ctx->alloc((void**)&k64, sizeof(unsigned long long) * npairs));
  PFE_CUDA(ctx->alloc((void**)&perm_a, sizeof(int) * npairs));
  PFE_CUDA(ctx->alloc((void**)&perm_b, sizeof(int) * npairs));
  PFE_CUDA(ctx->alloc((void**)&k32, sizeof(int) * npairs));
  PFE_CUDA(ctx->alloc((void**)&k32b, sizeof(int) * npairs));
  PFE_CUDA(ctx->alloc((void**)&k8, npairs));
  PFE_CUDA(ctx->alloc((void**)&k8b, npairs));
  PFE_CUDA(cudaMemsetAsync(gbits, 0, sizeof(unsigned long long) * ngid, s));
  k_mol_groupmax<<<nb256, 256, 0, s>>>(raw.schwarz, raw.gid, gbits, npairs);
  k_mol_keys<<<nb256, 256, 0, s>>>(raw.schwarz, raw.gid, gbits, k_sch, k_gmax, raw.gmax, npairs);
  k_mol_iota<<<nb256, 256, 0, s>>>(perm_a, npairs);
  PFE_CUDA(cudaGetLastError());
  {
    const int n = (int)npairs;
    if ((rc = radix_sort_pairs(ctx, k_sch, k64, perm_a, perm_b, n, 64, s)) != PFE_OK) return rc;
    k_gather_t<int><<<nb256, 256, 0, s>>>(raw.gid, perm_b, k32, npairs);
    if ((rc = radix_sort_pairs(ctx, k32, k32b, perm_b, perm_a, n, 32, s)) != PFE_OK) return rc;
    k_gather_t<unsigned long long><<<nb256, 256, 0, s>>>(k_gmax, perm_a, k_sch, npairs);
    if ((rc = radix_sort_pairs(ctx, k_sch, k64, perm_a, perm_b, n, 64, s)) != PFE_OK) return rc;
    k_gather_t<unsigned char><<<nb256, 256, 0, s>>>(raw.cls, perm_b, k8, npairs);
    if ((rc = radix_sort_pairs(ctx, k8, k8b, perm_b, perm_a, n, 8, s)) != PFE_OK) return rc;
    k_mol_gather<<<(unsigned)((npairs + 127) / 128), 128, 0, s>>>(raw, ctx->pairs, perm_a, npairs);
    PFE_CUDA(cudaGetLastError());
    PFE_CUDA(cudaStreamSynchronize(s));
  }
  PFE_CUDA(ctx->alloc((void**)&ctx->d_prec, sizeof(PairRec) * npairs));
  k_pack_pairs<<<nb256, 256, 0, s>>>(ctx->pairs, (PairRec*)ctx->d_prec, npairs);
  PFE_CUDA(cudaGetLastError());
  int hcount[8] = {0};
  PFE_CUDA(cudaMemcpy(hcount, d_count, sizeof(int) * 8, cudaMemcpyDeviceToHost));
  int off = 0;
  for (int c = 0; c < 6; ++c) {
    ctx->class_off[c] = off;
    ctx->class_n[c] = hcount[c];
    off += hcount[c];
  }
  // groups: runs of one gid in the sorted pairs
  int *head = nullptr, *gix = nullptr;
  PFE_CUDA(ctx->alloc((void**)&head, sizeof(int) * npairs));
  PFE_CUDA(ctx->alloc((void**)&gix, sizeof(int) * npairs));
  k_group_heads<<<nb256, 256, 0, s>>>(ctx->pairs.gid, head, npairs);
  if ((rc = exclusive_sum(ctx, head, gix, (int)npairs, s)) != PFE_OK) return rc;
  int last_gix = 0, last_head = 0;
  PFE_CUDA(cudaMemcpyAsync(&last_gix, gix + npairs - 1, sizeof(int), cudaMemcpyDeviceToHost, s));
  PFE_CUDA(cudaMemcpyAsync(&last_head, head + npairs - 1, sizeof(int), cudaMemcpyDeviceToHost, s));
  PFE_CUDA(cudaStreamSynchronize(s));
  const int ng = last_gix + last_head;
  ctx->ngroups = ng;
  unsigned char *gr_cls = nullptr, *bkey = nullptr, *bkey_sorted = nullptr;
  int* giota = nullptr;
  PFE_CUDA(ctx->alloc((void**)&ctx->d_gr_start, sizeof(int) * ng));
  PFE_CUDA(ctx->alloc((void**)&ctx->d_gr_n, sizeof(int) * ng));
  PFE_CUDA(ctx->alloc((void**)&ctx->d_gr_max, sizeof(double) * ng));
  PFE_CUDA(ctx->alloc((void**)&ctx->d_bk_list, sizeof(int) * ng));
  PFE_CUDA(ctx->alloc((void**)&gr_cls, ng));
  PFE_CUDA(ctx->alloc((void**)&bkey, ng));
  PFE_CUDA(ctx->alloc((void**)&bkey_sorted, ng));
  PFE_CUDA(ctx->alloc((void**)&giota, sizeof(int) * ng));
  k_group_fill<<<nb256, 256, 0, s>>>(head, gix, ctx->pairs.schwarz, ctx->pairs.cls, ctx->d_gr_start, ctx->d_gr_max,
                                     gr_cls, npairs);
  k_group_size<<<(ng + 255) / 256, 256, 0, s>>>(ctx->d_gr_start, gr_cls, ng, npairs, ctx->d_gr_n, bkey);
  k_mol_iota<<<(ng + 255) / 256, 256, 0, s>>>(giota, ng);
  PFE_CUDA(cudaGetLastError());
  if ((rc = radix_sort_pairs(ctx, bkey, bkey_sorted, giota, ctx->d_bk_list, ng, 8, s)) != PFE_OK) return rc;
  std::vector<unsigned char> h_cls(ng), h_bkey(ng);
  PFE_CUDA(cudaMemcpyAsync(h_cls.data(), gr_cls, ng, cudaMemcpyDeviceToHost, s));
  PFE_CUDA(cudaMemcpyAsync(h_bkey.data(), bkey_sorted, ng, cudaMemcpyDeviceToHost, s));
  PFE_CUDA(cudaStreamSynchronize(s));
  int cg0[6], cgn[6];
  for (int c = 0; c < 6; ++c) { cg0[c] = 0; cgn[c] = 0; }
  for (int g = ng - 1; g >= 0; --g) { cg0[h_cls[g]] = g; ++cgn[h_cls[g]]; }
  Segs seg[6];
  for (int c = 0; c < 6; ++c)
    for (int b = 0; b < NBUCKET; ++b) seg[c].s0[b] = seg[c].s1[b] = 0;
  for (int i = 0; i < ng; ++i) {
    const int c = h_bkey[i] >> 3, b = h_bkey[i] & 7;
    if (seg[c].s1[b] == 0) seg[c].s0[b] = i;
    seg[c].s1[b] = i + 1;
  }
  // chunk lists for every class pair cb >= ck
  ctx->nlaunch = 0;
  ctx->census_quartets = ctx->census_flops = ctx->census_ref = 0.0;
  PFE_CUDA(ctx->alloc((void**)&ctx->d_queue, sizeof(int) * 64 * 64));
  PFE_CUDA(cudaMemsetAsync(ctx->d_queue, 0, sizeof(int) * 64 * 64, s));
  int maxg = 1;
  for (int c = 0; c < 6; ++c) maxg = std::max(maxg, cgn[c]);
  int *nchunk = nullptr, *offs = nullptr;
  unsigned long long* d_total = nullptr;
  PFE_CUDA(ctx->alloc((void**)&nchunk, sizeof(int) * (maxg + 1)));
  PFE_CUDA(ctx->alloc((void**)&offs, sizeof(int) * (maxg + 1)));
  PFE_CUDA(ctx->alloc((void**)&d_total, sizeof(unsigned long long)));
  for (int cb = 0; cb < 6; ++cb)
    for (int ck = 0; ck <= cb; ++ck) {
      const int nbg = cgn[cb];
      bool any = false;
      for (int b = 0; b < NBUCKET; ++b) any = any || seg[ck].s1[b] > seg[ck].s0[b];
      if (nbg == 0 || !any) continue;
      k_chunk_count<<<(nbg + 127) / 128, 128, 0, s>>>(ctx->d_gr_max, ctx->d_bk_list, cg0[cb], nbg, seg[ck], cb == ck,
                                                      ctx->inttol, nchunk);
      PFE_CUDA(cudaMemsetAsync(nchunk + nbg, 0, sizeof(int), s));
      if ((rc = exclusive_sum(ctx, nchunk, offs, nbg + 1, s)) != PFE_OK) return rc;
      int total = 0;
      PFE_CUDA(cudaMemcpyAsync(&total, offs + nbg, sizeof(int), cudaMemcpyDeviceToHost, s));
      PFE_CUDA(cudaStreamSynchronize(s));
      if (total == 0) continue;
      ClassLaunch cl{};
      cl.gmul = 32;   // what the autotuner picks for most classes on C20H42 and the water batch
      cl.cb = cb;
      cl.ck = ck;
      cl.nchunks_host = total;
      PFE_CUDA(ctx->alloc((void**)&cl.chunks, sizeof(int4) * total));
      PFE_CUDA(ctx->alloc((void**)&cl.d_nchunks, sizeof(int)));
      PFE_CUDA(cudaMemcpyAsync(cl.d_nchunks, &cl.nchunks_host, sizeof(int), cudaMemcpyHostToDevice, s));
      k_chunk_fill<<<(nbg + 127) / 128, 128, 0, s>>>(ctx->d_gr_max, ctx->d_bk_list, cg0[cb], nbg, seg[ck], cb == ck,
                                                     ctx->inttol, offs, cl.chunks);
      PFE_CUDA(cudaMemsetAsync(d_total, 0, sizeof(unsigned long long), s));
      unsigned int *cost = nullptr, *cost_sorted = nullptr;
      int4* sorted = nullptr;
      PFE_CUDA(ctx->alloc((void**)&cost, sizeof(unsigned int) * total));
      PFE_CUDA(ctx->alloc((void**)&cost_sorted, sizeof(unsigned int) * total));
      PFE_CUDA(ctx->alloc((void**)&sorted, sizeof(int4) * total));
      k_chunk_census<<<(total + 3) / 4, 128, 0, s>>>(cl.chunks, total, ctx->d_bk_list, ctx->d_gr_start, ctx->d_gr_n,
                                                     ctx->pairs.schwarz, ctx->inttol, d_total, cost);
      PFE_CUDA(cudaGetLastError());
      {  // the work queue hands out the costliest chunks first (stable: equal costs keep their order)
        size_t tb = 0;
        cub::DeviceRadixSort::SortPairsDescending(nullptr, tb, cost, cost_sorted, cl.chunks, sorted, total, 0, 32, s);
        void* tmp = nullptr;
        PFE_CUDA(ctx->alloc(&tmp, tb + 16));
        PFE_CUDA(cub::DeviceRadixSort::SortPairsDescending(tmp, tb, cost, cost_sorted, cl.chunks, sorted, total, 0, 32,
                                                           s));
        PFE_CUDA(cudaMemcpyAsync(cl.chunks, sorted, sizeof(int4) * total, cudaMemcpyDeviceToDevice, s));
        PFE_CUDA(cudaStreamSynchronize(s));
        for (void* p : {(void*)tmp, (void*)cost, (void*)sorted}) ctx->free_now(p);
        cl.cost = cost_sorted;   // kept: a batch sorts its joined chunk list by it
      }
      unsigned long long nq = 0;
      PFE_CUDA(cudaMemcpyAsync(&nq, d_total, sizeof(unsigned long long), cudaMemcpyDeviceToHost, s));
      PFE_CUDA(cudaStreamSynchronize(s));
      cl.quartets = (double)nq;
      cl.has_straight = straight_launcher(cb, ck) != nullptr;
      cl.npass = cl.has_straight ? straight_npass(cb, ck) : 0;
      cl.npass_live = 0;   // register passes actually launched (the rest keep no coefficient)
      for (int p = 0; p < cl.npass; ++p)
        cl.npass_live += (cl.npass == 1 || pass_live(kCL[cb][0], kCL[cb][1], kCL[ck][0], kCL[ck][1], cl.npass, p,
                                                     lower_kept_bits(ctx)))
                             ? 1
                             : 0;
      cl.has_table = false;
      cl.variant = 0;
      cl.xg = nullptr;
      if (const OpTableHost* h = host_optable(cb, ck)) {
        OpTableDev d{};
        if ((rc = upload_optable(ctx, h, &d)) != PFE_OK) return rc;
        const Variants vv = variants(cb, ck);
        cl.has_table = true;
        cl.ops = d.ops; cl.levels = d.levels; cl.out = d.out;
        cl.nlevels = d.nlevels; cl.nout = d.nout; cl.nslots = d.nslots;
        cl.ops_p = nullptr; cl.levels_p = nullptr; cl.out_p = nullptr; cl.nlevels_p = 0;
        cl.nslots_p = cl.nslots_p2 = 0;
        if (const OpTableHost* hp = host_optable_pure(cb, ck)) {
          OpTableDev dp{};
          if ((rc = upload_optable(ctx, hp, &dp)) != PFE_OK) return rc;
          if (dp.nslots <= d.nslots) {   // runs inside the full table's shared-memory layout
            cl.ops_p = dp.ops; cl.levels_p = dp.levels; cl.out_p = dp.out; cl.nlevels_p = dp.nlevels;
            cl.nslots_p = dp.nslots;
          }
        }
        cl.ops_p2 = nullptr; cl.levels_p2 = nullptr; cl.out_p2 = nullptr; cl.nlevels_p2 = 0;
        if (const OpTableHost* hp = host_optable_pure2(cb, ck)) {
          OpTableDev dp{};
          if ((rc = upload_optable(ctx, hp, &dp)) != PFE_OK) return rc;
          if (dp.nslots <= d.nslots && cl.ops_p) {   // taken only where the pure-bra table is
            cl.ops_p2 = dp.ops; cl.levels_p2 = dp.levels; cl.out_p2 = dp.out; cl.nlevels_p2 = dp.nlevels;
            cl.nslots_p2 = dp.nslots;
          }
        }
        cl.per_warp = vv.doubles(h->nslots, true);
        cl.smem_big = sizeof(double) * (size_t)cl.per_warp;
        {  // warps per block that fit the most warps per SM in shared memory (228 KB, ~3 KB static per block)
          const size_t pw = sizeof(double) * (size_t)cl.per_warp;
          int best = 1, best_w = 0;
          for (int w = 1; w <= 8; ++w) {
            if (w * pw > 200 * 1024) break;
            const int resident = w * (int)((228 * 1024) / (w * pw + 3 * 1024));
            if (resident >= best_w) { best_w = resident; best = w; }
          }
          cl.wpb = best;
        }
        cl.smem_warp = sizeof(double) * (size_t)cl.per_warp * cl.wpb;
        if (cl.smem_big > 220 * 1024) {   // X to global scratch, one slice per block of the block variant
          cl.smem_big = sizeof(double) * (size_t)vv.doubles(h->nslots, false);
          if (cl.smem_big > 220 * 1024) {
            set_error("op-table working set of a quartet class exceeds shared memory");
            return PFE_EUNSUPPORTED;
          }
          PFE_CUDA(ctx->alloc((void**)&cl.xg, sizeof(double) * (size_t)h->nout * 2 * ctx->num_sms));
        }
        PFE_CUDA(vv.allow(cl.smem_big, std::min<size_t>(cl.smem_warp, 220 * 1024)));
        if ((rc = size_wide(cl, ctx->kept_max, ctx->lower_kept)) != PFE_OK) return rc;
        // default schedule (measured on B200, C20H42 and the water batch): straight-line code
        // where a class has it; (dd|dp) on the wide warp variant (3.2 ms against 4.9 ms per
        // block on C20H42); (dd|dd) per block (1.2 ms against 2.2 ms wide)
        cl.variant = cl.has_straight ? 0
                                     : ((cl.has_wide && h->nout <= 4000)
                                            ? 3
                                            : ((h->nout <= 640 && cl.smem_warp <= 200 * 1024) ? 1 : 2));
      }
      if (!cl.has_straight && !cl.has_table) {
        set_error("no kernel for a quartet class");
        return PFE_EUNSUPPORTED;
      }
      for (int v = 0; v < 4; ++v) cl.tuned_ms[v] = 0.f;
      cl.queue = ctx->d_queue + 64 * ctx->nlaunch;
      ctx->launches[ctx->nlaunch++] = cl;
      ctx->census_quartets += (double)nq;
      ctx->census_flops += (double)nq * class_flops(cb, ck);
    }
  ctx->free_now(d_count);
  free_pairs(ctx, &raw);
  for (void* p : {(void*)gbits, (void*)k_sch, (void*)k_gmax, (void*)k64, (void*)perm_a, (void*)perm_b, (void*)k32,
                  (void*)k32b, (void*)k8, (void*)k8b, (void*)head, (void*)gix, (void*)gr_cls, (void*)bkey,
                  (void*)bkey_sorted, (void*)giota, (void*)nchunk, (void*)offs, (void*)d_total})
    ctx->free_now(p);
  ctx->free_pending();
  return PFE_OK;
}

// ------------------------------------------------------------------ build

static MolLaunch make_launch(pfe_context* ctx, const double* d_dt) {
  MolLaunch ql{};
  ql.lower_kept_bits = lower_kept_bits(ctx);
  ql.pairs = ctx->pairs;
  ql.rec = (const PairRec*)ctx->d_prec;
  ql.prim = ctx->shells.prim;
  ql.stidx = ctx->d_stidx;
  ql.scoef = ctx->d_scoef;
  ql.boys = ctx->d_boys;
  ql.dt = d_dt;
  ql.jt = ctx->d_jp;
  ql.kt = ctx->d_kp;
  ql.gr_start = ctx->d_gr_start;
  ql.gr_n = ctx->d_gr_n;
  ql.gr_max = ctx->d_gr_max;
  ql.bk_list = ctx->d_bk_list;
  ql.blk = ctx->d_blk;
  ql.tblk = ctx->d_tblk;
  ql.bmax = ctx->d_bmax;
  ql.nblk = ctx->nblk;
  ql.dtol = ctx->dtol;
  ql.mcut = ctx->mcut;
  ql.n32 = ctx->d_n32;
  ql.inttol = ctx->inttol;
  ql.nt = ctx->nt;
  ql.myid = ctx->myid;
  ql.numprocs = ctx->numprocs;
  return ql;
}

static void launch_class(pfe_context* ctx, const ClassLaunch& cl, MolLaunch ql, int variant, cudaStream_t s,
                         bool mixed) {
  ql.chunks = cl.chunks;
  ql.nchunks = cl.d_nchunks;
  ql.queue = cl.queue;
  cudaMemsetAsync(cl.queue, 0, sizeof(int) * 64, s);   // every launch (pass) of the class starts its queue at 0
  const int work = (cl.nchunks_host + ctx->numprocs - 1) / ctx->numprocs;
  if ((variant == 0 && cl.has_straight) || !cl.has_table) {
    const int grid = std::min((work + 3) / 4, ctx->num_sms * cl.gmul);
    straight_launcher(cl.cb, cl.ck, mixed, ql.insts != nullptr)(ql, std::max(grid, 1), s);
    return;
  }
  OpTableDev t{cl.ops,   cl.levels,   cl.out,     cl.nlevels,   cl.nout,   cl.nslots,     cl.ops_p,
               cl.levels_p, cl.out_p, cl.nlevels_p, cl.ops_p2, cl.levels_p2, cl.out_p2, cl.nlevels_p2,
               cl.nslots_p, cl.nslots_p2};
  if (variant == 3 && cl.has_wide) {
    const int per_sm = std::max(1, (int)((160 * 1024) / cl.smem_wide));   // resident blocks per SM
    const int grid = std::min((work + cl.wide_wpb - 1) / cl.wide_wpb, ctx->num_sms * per_sm);
    wide_variant(cl.cb, cl.ck).launch(ql, t, std::max(grid, 1), cl.wide_wpb, cl.wide_per_warp, cl.wide_vmax,
                                      cl.wide_xmax, cl.smem_wide, s);
    return;
  }
  if (variant == 1) {
    const int grid = std::min((work + cl.wpb - 1) / cl.wpb, ctx->num_sms * 8);
    variants(cl.cb, cl.ck).warp(ql, t, std::max(grid, 1), cl.wpb, cl.per_warp, cl.smem_warp, s);
  } else {
    const int grid = std::min(work, ctx->num_sms * 2);   // cl.xg holds 2 * num_sms slices
    variants(cl.cb, cl.ck).big(ql, t, cl.xg, std::max(grid, 1), cl.smem_big, s);
  }
}

static size_t target_bytes(const pfe_context* ctx) { return sizeof(double) * (size_t)ctx->nt * ctx->nt; }

// Density in target space: P_P itself (primitive targets) or P_C read off P_P
// and checked (contracted targets); returns the pointer the kernels read.
static const double* target_density(pfe_context* ctx, const double* d_pp, cudaStream_t s) {
  if (!ctx->contracted) return d_pp;
  const long long nt2 = (long long)ctx->nt * ctx->nt, np2 = (long long)ctx->npgs * ctx->npgs;
  k_target_density<<<(unsigned)((nt2 + 255) / 256), 256, 0, s>>>(d_pp, ctx->npgs, ctx->d_rep, ctx->d_repc, ctx->nt,
                                                                   ctx->d_pt);
  cudaMemsetAsync(ctx->d_flag, 0, sizeof(unsigned int), s);
  k_check_density<<<(unsigned)((np2 + 255) / 256), 256, 0, s>>>(d_pp, ctx->npgs, ctx->d_tidx, ctx->d_tcoef,
                                                                  ctx->d_pt, ctx->nt, ctx->d_flag);
  return ctx->d_pt;
}

static bool variant_ok(const ClassLaunch& cl, int v) {
  if (v == 0) return cl.has_straight;
  if (v == 1) return cl.has_table && cl.smem_warp <= 200 * 1024;
  if (v == 3) return cl.has_wide;
  return cl.has_table;
}

// Time every execution variant of one class -- and, for the straight-line
// variant, its persistent grid (4, 8, 16 or 32 blocks per SM) -- and keep the
// fastest (best of two launches after one warm-up each).
static int tune_class(pfe_context* ctx, ClassLaunch& cl, const MolLaunch& ql, cudaStream_t s, bool mixed,
                      cudaEvent_t e0, cudaEvent_t e1) {
  float best = 1e30f;
  int bestv = cl.variant, bestg = cl.gmul;
  for (int v = 0; v < 4; ++v) {
    if (!variant_ok(cl, v)) continue;
    // the one-quartet-per-warp/block interpreters lose to the straight-line code by
    // 5-300x on every class that has it (measured on C20H42 and the water batch):
    // not timed there, which keeps the autotuner to seconds
    if ((v == 1 || v == 2) && cl.has_straight) continue;
    static const int kGmul[4] = {4, 8, 16, 32};
    const int ng = v == 0 ? 4 : 1;
    float tv = 1e30f;
    for (int gi = 0; gi < ng; ++gi) {
      if (v == 0) cl.gmul = kGmul[gi];
      launch_class(ctx, cl, ql, v, s, mixed);
      float t = 1e30f;
      for (int r = 0; r < 2; ++r) {
        PFE_CUDA(cudaEventRecord(e0, s));
        launch_class(ctx, cl, ql, v, s, mixed);
        PFE_CUDA(cudaEventRecord(e1, s));
        PFE_CUDA(cudaEventSynchronize(e1));
        float ms = 0.f;
        PFE_CUDA(cudaEventElapsedTime(&ms, e0, e1));
        t = std::min(t, ms);
      }
      PFE_CUDA(cudaGetLastError());
      tv = std::min(tv, t);
      if (t < best) { best = t; bestv = v; bestg = cl.gmul; }
    }
    cl.tuned_ms[v] = tv;
  }
  cl.variant = bestv;
  cl.gmul = bestg;
  return PFE_OK;
}

int autotune(pfe_context* ctx, const double* d_pp, cudaStream_t s) {
  const MolLaunch ql = make_launch(ctx, target_density(ctx, d_pp, s));
  PFE_CUDA(cudaGetLastError());
  cudaEvent_t e0, e1;
  PFE_CUDA(cudaEventCreate(&e0));
  PFE_CUDA(cudaEventCreate(&e1));
  for (int i = 0; i < ctx->nlaunch; ++i) {
    ClassLaunch& cl = ctx->launches[i];
    const int rc = tune_class(ctx, cl, ql, s, ctx->mcut > 0.0, e0, e1);
    if (rc != PFE_OK) return rc;
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  PFE_CUDA(cudaMemsetAsync(ctx->d_jp, 0, target_bytes(ctx), s));
  PFE_CUDA(cudaMemsetAsync(ctx->d_kp, 0, target_bytes(ctx), s));
  PFE_CUDA(cudaStreamSynchronize(s));
  ctx->tuned = true;
  return PFE_OK;
}

// Zero the target-space J'/K' and the FP32 counter; block maxima of the density
// when screening or mixed precision is on.
static int prepare_build(pfe_context* ctx, const double* d_dt, cudaStream_t s, bool always_bmax = false) {
  PFE_CUDA(cudaMemsetAsync(ctx->d_jp, 0, target_bytes(ctx), s));
  PFE_CUDA(cudaMemsetAsync(ctx->d_kp, 0, target_bytes(ctx), s));
  PFE_CUDA(cudaMemsetAsync(ctx->d_n32, 0, sizeof(unsigned long long), s));
  if (always_bmax || ctx->dtol > 0.0 || ctx->mcut > 0.0) {
    const long long nt2 = (long long)ctx->nt * ctx->nt;
    PFE_CUDA(cudaMemsetAsync(ctx->d_bmax, 0, sizeof(double) * (size_t)ctx->nblk * ctx->nblk, s));
    k_block_dmax<<<(unsigned)((nt2 + 255) / 256), 256, 0, s>>>(d_dt, ctx->nt, ctx->d_tblk, ctx->nblk,
                                                               (unsigned long long*)ctx->d_bmax);
    PFE_CUDA(cudaGetLastError());
  }
  return PFE_OK;
}

// The class launches of one molecule's build: the interpreter classes (wide,
// warp and block variants: few resident warps, bound by shared memory or
// barriers) on the context's side stream, forked from s, and the straight-line
// classes on s, so that the two kinds share the SMs; s then waits for the side
// stream.  J' and K' take atomic adds only, so the order of the classes does not
// matter.  Measured: C20H42 34.0 -> 32.0 ms.  Batches keep one stream (the
// 32-cluster water batch was 2 % slower split: its interpreter classes are a
// small share, and they slowed the straight-line ones beside them).  Serial on
// s when `serial` (per-class timing).
static int launch_classes(pfe_context* cx, const ClassLaunch* launches, int nlaunch, const MolLaunch& ql,
                          cudaStream_t s, bool mixed, bool serial) {
  bool any_side = false;
  for (int i = 0; i < nlaunch && !serial; ++i)
    any_side = any_side || !((launches[i].variant == 0 && launches[i].has_straight) || !launches[i].has_table);
  const bool split = any_side && cx->side != nullptr;
  if (split) {
    PFE_CUDA(cudaEventRecord(cx->ev_fork, s));
    PFE_CUDA(cudaStreamWaitEvent(cx->side, cx->ev_fork, 0));
    for (int i = 0; i < nlaunch; ++i) {
      const ClassLaunch& cl = launches[i];
      if (!((cl.variant == 0 && cl.has_straight) || !cl.has_table)) launch_class(cx, cl, ql, cl.variant, cx->side, mixed);
    }
    PFE_CUDA(cudaGetLastError());
  }
  for (int i = 0; i < nlaunch; ++i) {
    const ClassLaunch& cl = launches[i];
    const bool straight = (cl.variant == 0 && cl.has_straight) || !cl.has_table;
    if (!split || straight) launch_class(cx, cl, ql, cl.variant, s, mixed);
  }
  PFE_CUDA(cudaGetLastError());
  if (split) {
    PFE_CUDA(cudaEventRecord(cx->ev_join, cx->side));
    PFE_CUDA(cudaStreamWaitEvent(s, cx->ev_join, 0));
  }
  return PFE_OK;
}

static int run_build(pfe_context* ctx, const double* d_dt, double* d_cc, double* d_xc, cudaStream_t s) {
  const int rc = prepare_build(ctx, d_dt, s);
  if (rc != PFE_OK) return rc;
  const MolLaunch ql = make_launch(ctx, d_dt);
  if (ctx->profile) {
    for (int i = 0; i <= ctx->nlaunch && i < 64; ++i)
      if (!ctx->ev[i]) PFE_CUDA(cudaEventCreate(&ctx->ev[i]));
    ctx->nprof = ctx->nlaunch;
    PFE_CUDA(cudaEventRecord(ctx->ev[0], s));
  }
  if (!ctx->profile) {
    const int rc2 = launch_classes(ctx, ctx->launches, ctx->nlaunch, ql, s, ctx->mcut > 0.0, false);
    if (rc2 != PFE_OK) return rc2;
  }
  for (int i = 0; i < ctx->nlaunch && ctx->profile; ++i) {
    const ClassLaunch& cl = ctx->launches[i];
    launch_class(ctx, cl, ql, cl.variant, s, ctx->mcut > 0.0);
    PFE_CUDA(cudaGetLastError());
    {
      PFE_CUDA(cudaEventRecord(ctx->ev[i + 1], s));
      ctx->ev_cls[i] = 1000 * kCL[cl.cb][0] + 100 * kCL[cl.cb][1] + 10 * kCL[cl.ck][0] + kCL[cl.ck][1];
      ctx->ev_quartets[i] = cl.quartets;
      ctx->ev_flops[i] = cl.quartets * class_flops(cl.cb, cl.ck);
      ctx->ev_gmul[i] = cl.gmul;
      ctx->ev_variant[i] = cl.variant;
      for (int v = 0; v < 4; ++v) ctx->ev_tuned[i][v] = cl.tuned_ms[v];
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

int molecular_fock(pfe_context* ctx, const double* d_pp, double* d_cc, double* d_xc, cudaStream_t s) {
  const double* d_dt = target_density(ctx, d_pp, s);
  PFE_CUDA(cudaGetLastError());
  return run_build(ctx, d_dt, d_cc, d_xc, s);
}

// Build from the contracted density P_C (ncgs x ncgs): read directly as the
// target-space density, or decontracted on the device (P_P = CC^T P_C CC,
// src/pdensitymatrix.f90:343-381) for primitive targets.
int molecular_fock_pc(pfe_context* ctx, const double* d_pc, double* d_cc, double* d_xc, cudaStream_t s) {
  if (ctx->contracted) return run_build(ctx, d_pc, d_cc, d_xc, s);
  const int np = ctx->npgs, nc = ctx->ncgs;
  const double one = 1.0, zero = 0.0;
  if (!ensure_blas(ctx)) { set_error("cublasCreate failed"); return PFE_ECUDA; }
  cublasSetStream(ctx->blas, s);
  // W1 = P_C . CC (nc x np); P_P = CC^T . W1 (np x np) into the target-density buffer
  cublasStatus_t st = cublasDgemm(ctx->blas, CUBLAS_OP_N, CUBLAS_OP_N, nc, np, nc, &one, d_pc, nc, ctx->d_cc, nc, &zero,
                                  ctx->d_w1, nc);
  if (st != CUBLAS_STATUS_SUCCESS) { set_error("cublasDgemm (P_C.CC) failed"); return PFE_ECUDA; }
  st = cublasDgemm(ctx->blas, CUBLAS_OP_T, CUBLAS_OP_N, np, np, nc, &one, ctx->d_cc, nc, ctx->d_w1, nc, &zero,
                   ctx->d_pt, np);
  if (st != CUBLAS_STATUS_SUCCESS) { set_error("cublasDgemm (CC^T.W) failed"); return PFE_ECUDA; }
  return run_build(ctx, ctx->d_pt, d_cc, d_xc, s);
}

MolLaunch molecular_launch(pfe_context* ctx, const double* d_dt) { return make_launch(ctx, d_dt); }

int molecular_gradient(pfe_context* ctx, const double* d_dt, const int* d_satom, int natom, double* d_gj,
                       double* d_gk, cudaStream_t s);

// The two-electron gradient (pfe_grad.cu) for P_P: read as the target-space density as the
// Fock build does (molecules only).
int molecular_gradient_pp(pfe_context* ctx, const double* d_pp, const int* d_satom, int natom, double* d_gj,
                          double* d_gk, cudaStream_t s) {
  const double* d_dt = target_density(ctx, d_pp, s);
  PFE_CUDA(cudaGetLastError());
  return molecular_gradient(ctx, d_dt, d_satom, natom, d_gj, d_gk, s);
}

// Whether the last build's P_P was the decontraction of a contracted density
// (always true for primitive targets).  Synchronises the stream.
int molecular_density_ok(pfe_context* ctx, cudaStream_t s, bool* ok) {
  *ok = true;
  if (!ctx->contracted || !ctx->molecular) return PFE_OK;
  unsigned int f = 0;
  PFE_CUDA(cudaMemcpyAsync(&f, ctx->d_flag, sizeof(unsigned int), cudaMemcpyDeviceToHost, s));
  PFE_CUDA(cudaStreamSynchronize(s));
  *ok = (f == 0);
  return PFE_OK;
}

}  // namespace pfe

// ------------------------------------------------------------------ batches

namespace pfe {

__global__ void k_tag_chunks(int4* __restrict__ chunks, int n, int instance) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t < n) chunks[t].w = instance;
}

// Join the instances' chunk lists per (bra class, ket class): device copies and
// tags queued on one stream, one synchronisation at the end.
int batch_setup(pfe_batch* b) {
  b->nlaunch = 0;
  PFE_CUDA(b->alloc((void**)&b->d_queue, sizeof(int) * 64 * 64));
  cudaStream_t st = nullptr;
  PFE_CUDA(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
  struct StreamGuard {
    cudaStream_t s;
    ~StreamGuard() { if (s) { cudaStreamSynchronize(s); cudaStreamDestroy(s); } }
  } guard{st};
  for (int cb = 0; cb < 6; ++cb)
    for (int ck = 0; ck <= cb; ++ck) {
      long long total = 0;
      const ClassLaunch* tmpl = nullptr;
      for (pfe_context* c : b->inst)
        for (int i = 0; i < c->nlaunch; ++i)
          if (c->launches[i].cb == cb && c->launches[i].ck == ck) {
            total += c->launches[i].nchunks_host;
            if (!tmpl) tmpl = &c->launches[i];
          }
      if (!tmpl || total == 0) continue;
      if (total >= (1LL << 31)) { set_error("batch: too many chunks in one quartet class"); return PFE_EINVAL; }
      ClassLaunch cl = *tmpl;
      {  // launched passes over the whole batch: a pass is skipped only if no instance needs it
        int bits = 0;
        for (pfe_context* c : b->inst) bits |= lower_kept_bits(c);
        cl.npass_live = 0;
        for (int p = 0; p < cl.npass; ++p)
          cl.npass_live +=
              (cl.npass == 1 || pass_live(kCL[cb][0], kCL[cb][1], kCL[ck][0], kCL[ck][1], cl.npass, p, bits)) ? 1 : 0;
      }
      if (cl.has_wide) {   // the wide variant's working set must cover every instance
        int km[3] = {1, 1, 1};
        bool lk[3] = {false, false, false};
        for (pfe_context* c : b->inst)
          for (int L = 0; L < 3; ++L) { km[L] = std::max(km[L], c->kept_max[L]); lk[L] = lk[L] || c->lower_kept[L]; }
        const int rc = size_wide(cl, km, lk);
        if (rc != PFE_OK) return rc;
        if (!cl.has_wide && cl.variant == 3) cl.variant = cl.has_straight ? 0 : 2;
      }
      cl.nchunks_host = (int)total;
      cl.quartets = 0.0;
      cl.queue = b->d_queue + 64 * b->nlaunch;
      PFE_CUDA(b->alloc((void**)&cl.chunks, sizeof(int4) * total));
      PFE_CUDA(b->alloc((void**)&cl.d_nchunks, sizeof(int)));
      unsigned int* jcost = nullptr;
      PFE_CUDA(b->alloc((void**)&jcost, sizeof(unsigned int) * total));
      PFE_CUDA(cudaMemcpy(cl.d_nchunks, &cl.nchunks_host, sizeof(int), cudaMemcpyHostToDevice));   // pageable: synchronous
      long long o = 0;
      for (size_t k = 0; k < b->inst.size(); ++k) {
        pfe_context* c = b->inst[k];
        for (int i = 0; i < c->nlaunch; ++i) {
          const ClassLaunch& li = c->launches[i];
          if (li.cb != cb || li.ck != ck) continue;
          PFE_CUDA(cudaMemcpyAsync(cl.chunks + o, li.chunks, sizeof(int4) * li.nchunks_host, cudaMemcpyDeviceToDevice,
                                   st));
          PFE_CUDA(cudaMemcpyAsync(jcost + o, li.cost, sizeof(unsigned int) * li.nchunks_host,
                                   cudaMemcpyDeviceToDevice, st));
          k_tag_chunks<<<(li.nchunks_host + 255) / 256, 256, 0, st>>>(cl.chunks + o, li.nchunks_host, (int)k);
          PFE_CUDA(cudaGetLastError());
          o += li.nchunks_host;
          cl.quartets += li.quartets;
        }
      }
      {  // one queue over the whole batch, costliest chunks first
        unsigned int* ks = nullptr;
        int4* vs = nullptr;
        PFE_CUDA(b->alloc((void**)&ks, sizeof(unsigned int) * total));
        PFE_CUDA(b->alloc((void**)&vs, sizeof(int4) * total));
        size_t tb = 0;
        cub::DeviceRadixSort::SortPairsDescending(nullptr, tb, jcost, ks, cl.chunks, vs, (int)total, 0, 32, st);
        void* tmp = nullptr;
        PFE_CUDA(b->alloc(&tmp, tb + 16));
        PFE_CUDA(cub::DeviceRadixSort::SortPairsDescending(tmp, tb, jcost, ks, cl.chunks, vs, (int)total, 0, 32, st));
        PFE_CUDA(cudaMemcpyAsync(cl.chunks, vs, sizeof(int4) * total, cudaMemcpyDeviceToDevice, st));
        cl.cost = ks;
      }
      b->launches[b->nlaunch++] = cl;
    }
  PFE_CUDA(b->alloc(&b->d_insts, sizeof(MolLaunch) * b->inst.size()));
  PFE_CUDA(b->alloc((void**)&b->d_off, sizeof(long long) * b->off.size()));
  PFE_CUDA(cudaMemcpy(b->d_off, b->off.data(), sizeof(long long) * b->off.size(), cudaMemcpyHostToDevice));
  b->all_contracted = true;
  for (pfe_context* c : b->inst) b->all_contracted = b->all_contracted && c->contracted;
  PFE_CUDA(cudaMallocHost(&b->h_insts, sizeof(MolLaunch) * b->inst.size()));
  PFE_CUDA(cudaEventCreateWithFlags(&b->ev_insts, cudaEventDisableTiming));
  b->insts_for = nullptr;
  b->mixed = false;
  for (pfe_context* c : b->inst) b->mixed = b->mixed || c->mcut > 0.0;
  PFE_CUDA(cudaStreamSynchronize(st));
  PFE_CUDA(cudaDeviceSynchronize());
  return PFE_OK;
}

// Rewrite the pinned launch records for densities packed at d_pc with the
// instances' current screening (waits for the previous upload to finish).
int batch_refresh(pfe_batch* b, const double* d_pc) {
  if (b->ev_pending) PFE_CUDA(cudaEventSynchronize(b->ev_insts));
  b->ev_pending = false;
  MolLaunch* h = static_cast<MolLaunch*>(b->h_insts);
  for (size_t k = 0; k < b->inst.size(); ++k) {
    pfe_context* c = b->inst[k];
    h[k] = make_launch(c, c->contracted ? d_pc + b->off[k] : c->d_pt);
    b->mixed = b->mixed || c->mcut > 0.0;
  }
  b->insts_for = d_pc;
  return PFE_OK;
}

// Target-space densities of the instances with primitive targets: P_P = CC^T P_C CC.
static int batch_decontract(pfe_batch* b, const double* d_pc, cudaStream_t s) {
  for (size_t k = 0; k < b->inst.size(); ++k) {
    pfe_context* c = b->inst[k];
    if (c->contracted) continue;
    const int np = c->npgs, nc = c->ncgs;
    const double one = 1.0, zero = 0.0;
    if (!ensure_blas(c)) { set_error("cublasCreate failed"); return PFE_ECUDA; }
    cublasSetStream(c->blas, s);
    if (cublasDgemm(c->blas, CUBLAS_OP_N, CUBLAS_OP_N, nc, np, nc, &one, d_pc + b->off[k], nc, c->d_cc, nc, &zero,
                    c->d_w1, nc) != CUBLAS_STATUS_SUCCESS ||
        cublasDgemm(c->blas, CUBLAS_OP_T, CUBLAS_OP_N, np, np, nc, &one, c->d_cc, nc, c->d_w1, nc, &zero, c->d_pt,
                    np) != CUBLAS_STATUS_SUCCESS) {
      set_error("batch: cublasDgemm (decontraction) failed");
      return PFE_ECUDA;
    }
  }
  return PFE_OK;
}

// The per-instance work around a batched build as three launches over every
// instance (blockIdx.y = instance, the threads of its blocks stride over its
// matrices) instead of seven small ones per instance: zero J'/K', the block
// maxima and the FP32 counter; the block maxima of |P_T|; after the class
// kernels, C_C = J' + J'^T and X_C = K' + K'^T at the packed offsets.
__global__ void k_batch_zero(const MolLaunch* __restrict__ insts) {
  const MolLaunch& q = insts[blockIdx.y];
  const long long nt2 = (long long)q.nt * q.nt, nb2 = (long long)q.nblk * q.nblk;
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < nt2; t += (long long)gridDim.x * blockDim.x) {
    q.jt[t] = 0.0;
    q.kt[t] = 0.0;
    if (t < nb2) const_cast<double*>(q.bmax)[t] = 0.0;
  }
  for (long long t = nt2 + blockIdx.x * (long long)blockDim.x + threadIdx.x; t < nb2;
       t += (long long)gridDim.x * blockDim.x)
    const_cast<double*>(q.bmax)[t] = 0.0;
  if (blockIdx.x == 0 && threadIdx.x == 0) *q.n32 = 0ull;
}

__global__ void k_batch_dmax(const MolLaunch* __restrict__ insts) {
  const MolLaunch& q = insts[blockIdx.y];
  const long long nt2 = (long long)q.nt * q.nt;
  unsigned long long* bm = reinterpret_cast<unsigned long long*>(const_cast<double*>(q.bmax));
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < nt2; t += (long long)gridDim.x * blockDim.x) {
    const int b1 = q.tblk[t % q.nt], b2 = q.tblk[t / q.nt];
    if (b1 < 0 || b2 < 0) continue;
    const double v = fabs(q.dt[t]);
    if (v > 0.0) atomicMax(bm + (size_t)b1 * q.nblk + b2, (unsigned long long)__double_as_longlong(v));
  }
}

__global__ void k_batch_symmetrize(const MolLaunch* __restrict__ insts, const long long* __restrict__ off,
                                   double* __restrict__ cc, double* __restrict__ xc) {
  const MolLaunch& q = insts[blockIdx.y];
  const int n = q.nt;
  const long long nt2 = (long long)n * n;
  double* c = cc + off[blockIdx.y];
  double* x = xc + off[blockIdx.y];
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < nt2; t += (long long)gridDim.x * blockDim.x) {
    const int i = (int)(t % n), j = (int)(t / n);
    const long long tt = i * (long long)n + j;   // (j, i)
    c[t] = q.jt[t] + q.jt[tt];
    x[t] = q.kt[t] + q.kt[tt];
  }
}

// One build of every instance from the packed contracted densities d_pc.
int batch_fock_pc(pfe_batch* b, const double* d_pc, double* d_cc, double* d_xc, cudaStream_t s) {
  const size_t n = b->inst.size();
  {
    const int rc = batch_decontract(b, d_pc, s);
    if (rc != PFE_OK) return rc;
  }
  cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
  PFE_CUDA(cudaStreamIsCapturing(s, &cap));
  const bool capturing = cap != cudaStreamCaptureStatusNone;
  if (b->insts_for != d_pc) {
    if (capturing) {
      set_error("batch: launch records are stale inside a stream capture (call pfe_batch_refresh first)");
      return PFE_EINVAL;
    }
    const int rc = batch_refresh(b, d_pc);
    if (rc != PFE_OK) return rc;
  }
  // the records travel with every build: a captured graph uploads what the host
  // last wrote into the pinned copy
  PFE_CUDA(cudaMemcpyAsync(b->d_insts, b->h_insts, sizeof(MolLaunch) * n, cudaMemcpyHostToDevice, s));
  if (!capturing) {
    PFE_CUDA(cudaEventRecord(b->ev_insts, s));
    b->ev_pending = true;
  }
  // zero J'/K' and take the block maxima of every instance (its screening may
  // change between graph replays), one launch each over the whole batch
  const MolLaunch* di = static_cast<const MolLaunch*>(b->d_insts);
  const dim3 gb(8, (unsigned)n);
  k_batch_zero<<<gb, 256, 0, s>>>(di);
  k_batch_dmax<<<gb, 256, 0, s>>>(di);
  PFE_CUDA(cudaGetLastError());
  pfe_context* c0 = b->inst[0];
  MolLaunch lq = make_launch(c0, c0->d_pt);
  lq.insts = di;
  for (pfe_context* c : b->inst) lq.lower_kept_bits |= lower_kept_bits(c);   // a pass is skipped only if dead everywhere
  for (int i = 0; i < b->nlaunch; ++i) {
    const ClassLaunch& cl = b->launches[i];
    launch_class(c0, cl, lq, cl.variant, s, b->mixed);
    PFE_CUDA(cudaGetLastError());
  }
  if (b->all_contracted) {
    k_batch_symmetrize<<<gb, 256, 0, s>>>(di, b->d_off, d_cc, d_xc);
  } else {
    for (size_t k = 0; k < n; ++k) {
      pfe_context* c = b->inst[k];
      if (c->contracted) {
        launch_symmetrize(c->d_jp, d_cc + b->off[k], c->ncgs, 1, s);
        launch_symmetrize(c->d_kp, d_xc + b->off[k], c->ncgs, 1, s);
      } else {
        int rc = contract_outputs(c, c->d_jp, c->d_kp, d_cc + b->off[k], d_xc + b->off[k], true, 1, s);
        if (rc != PFE_OK) return rc;
      }
    }
  }
  PFE_CUDA(cudaGetLastError());
  return PFE_OK;
}

// The schedule autotuner over a batch: every execution variant of every joined
// class is timed on the batch's densities d_pc and the fastest kept.
int batch_autotune(pfe_batch* b, const double* d_pc, cudaStream_t s) {
  int rc = batch_decontract(b, d_pc, s);
  if (rc != PFE_OK) return rc;
  if (b->insts_for != d_pc && (rc = batch_refresh(b, d_pc)) != PFE_OK) return rc;
  PFE_CUDA(cudaMemcpyAsync(b->d_insts, b->h_insts, sizeof(MolLaunch) * b->inst.size(), cudaMemcpyHostToDevice, s));
  PFE_CUDA(cudaEventRecord(b->ev_insts, s));
  b->ev_pending = true;
  for (size_t k = 0; k < b->inst.size(); ++k) {
    pfe_context* c = b->inst[k];
    if ((rc = prepare_build(c, c->contracted ? d_pc + b->off[k] : c->d_pt, s, true)) != PFE_OK) return rc;
  }
  pfe_context* c0 = b->inst[0];
  MolLaunch lq = make_launch(c0, c0->d_pt);
  lq.insts = static_cast<const MolLaunch*>(b->d_insts);
  for (pfe_context* c : b->inst) lq.lower_kept_bits |= lower_kept_bits(c);
  cudaEvent_t e0, e1;
  PFE_CUDA(cudaEventCreate(&e0));
  PFE_CUDA(cudaEventCreate(&e1));
  for (int i = 0; i < b->nlaunch; ++i) {
    ClassLaunch& cl = b->launches[i];
    const int rc = tune_class(c0, cl, lq, s, b->mixed, e0, e1);
    if (rc != PFE_OK) return rc;
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  PFE_CUDA(cudaStreamSynchronize(s));
  return PFE_OK;
}

}  // namespace pfe
