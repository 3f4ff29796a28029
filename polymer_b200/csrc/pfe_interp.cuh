// Level-scheduled op-table interpreter shared by the molecular and lattice
// kernels: device view of a generated op table, the per-quartet geometry
// multipliers of the four op kinds, and the block-wide executor.
#pragma once

#include "pfe_common.cuh"
#include "pfe_context.cuh"

namespace pfe {

struct OpTableDev {
  const unsigned short* ops;   // 8 uint16 per op, 16-byte aligned (see eval_op)
  const int* levels;
  const unsigned short* out;
  int nlevels, nout, nslots;
  // the class's pure-bra variant (only the top-level components of the bra
  // shells; at most nslots slots), or null: the molecular interpreter runs it
  // for chunks whose bra shells have coefficient-free lower components
  const unsigned short* ops_p;
  const int* levels_p;
  const unsigned short* out_p;
  int nlevels_p;
  // the variant with pure bra and pure ket shells, for (G|H) whose ket shells
  // are pure too, or null
  const unsigned short* ops_p2;
  const int* levels_p2;
  const unsigned short* out_p2;
  int nlevels_p2;
  int nslots_p, nslots_p2;   // slots of the two variants (0 where absent)
};

// Geometry multipliers of the four op kinds, in shared memory.
struct OpGeom {
  double G1[4][3], G2[4][3];
  double X[4], Y[4], Z;
};

// Value of an op of a table: each op is one 16-byte record of eight uint16,
// (kind<<12 | axis<<10 | cA<<5 | cB, s1, s2, s3, s4, s5, dest, 0), read with
// one vector load:  v[dest] = G1*v[s1] + G2*v[s2] + cA*X*(v[s3] - Y*v[s4]) +
// cB*Z*v[s5] (slots are reused once their value's last reader has run, so the
// destination is part of the record).
__device__ __forceinline__ double eval_rec(const uint4 r, const double* v, const OpGeom& geo) {
  const int h = r.x & 0xffff;
  const int kind = h >> 12, ax = (h >> 10) & 3, cA = (h >> 5) & 31, cB = h & 31;
  double val = geo.G1[kind][ax] * v[r.x >> 16] + geo.G2[kind][ax] * v[r.y & 0xffff];
  if (cA) val += (double)cA * geo.X[kind] * (v[r.y >> 16] - geo.Y[kind] * v[r.z & 0xffff]);
  if (cB) val += (double)cB * geo.Z * v[r.z >> 16];
  return val;
}

__device__ __forceinline__ double eval_op(const unsigned short* __restrict__ ops, int o, const double* v,
                                          const OpGeom& geo) {
  return eval_rec(__ldg(reinterpret_cast<const uint4*>(ops) + o), v, geo);
}

struct EvalD {
  __device__ __forceinline__ double operator()(const uint4 r, const double* v, const OpGeom& g) const {
    return eval_rec(r, v, g);
  }
};

// One level [o0, o1) of a table by a team of `team` threads (this one is tid):
// the ops of a level only read lower levels, so each thread loads four op
// records before evaluating any of them (four record loads in flight instead
// of one load-use chain per op).
template <typename T, typename Geo, typename Eval>
__device__ __forceinline__ void run_level(const unsigned short* __restrict__ ops, int o0, int o1, T* v, const Geo& geo,
                                          int tid, int team, Eval eval) {
  const uint4* rec = reinterpret_cast<const uint4*>(ops);
  int o = o0 + tid;
  for (; o + 3 * team < o1; o += 4 * team) {
    const uint4 r0 = __ldg(rec + o), r1 = __ldg(rec + o + team), r2 = __ldg(rec + o + 2 * team),
                r3 = __ldg(rec + o + 3 * team);
    const T a0 = eval(r0, v, geo), a1 = eval(r1, v, geo), a2 = eval(r2, v, geo), a3 = eval(r3, v, geo);
    v[r0.w & 0xffff] = a0;
    v[r1.w & 0xffff] = a1;
    v[r2.w & 0xffff] = a2;
    v[r3.w & 0xffff] = a3;
  }
  for (; o < o1; o += team) {
    const uint4 r = __ldg(rec + o);
    v[r.w & 0xffff] = eval(r, v, geo);
  }
}

// The same op in FP32 (the mixed-precision lattice path): slots hold F_m/pref
// and the recursion's geometry rounded to float.
struct OpGeomF {
  float G1[4][3], G2[4][3];
  float X[4], Y[4], Z;
};

__device__ __forceinline__ float eval_rec_f(const uint4 r, const float* v, const OpGeomF& geo) {
  const int h = r.x & 0xffff;
  const int kind = h >> 12, ax = (h >> 10) & 3, cA = (h >> 5) & 31, cB = h & 31;
  float val = geo.G1[kind][ax] * v[r.x >> 16] + geo.G2[kind][ax] * v[r.y & 0xffff];
  if (cA) val += (float)cA * geo.X[kind] * (v[r.y >> 16] - geo.Y[kind] * v[r.z & 0xffff]);
  if (cB) val += (float)cB * geo.Z * v[r.z >> 16];
  return val;
}

struct EvalF {
  __device__ __forceinline__ float operator()(const uint4 r, const float* v, const OpGeomF& g) const {
    return eval_rec_f(r, v, g);
  }
};

__device__ __forceinline__ void geom_to_float(const OpGeom& g, OpGeomF& f) {
  for (int k = 0; k < 4; ++k) {
    for (int a = 0; a < 3; ++a) {
      f.G1[k][a] = (float)g.G1[k][a];
      f.G2[k][a] = (float)g.G2[k][a];
    }
    f.X[k] = (float)g.X[k];
    f.Y[k] = (float)g.Y[k];
  }
  f.Z = (float)g.Z;
}

__device__ __forceinline__ void run_optable(const OpTableDev& t, double* __restrict__ v, const OpGeom& geo) {
  for (int l = 0; l < t.nlevels; ++l) {
    const int o0 = t.levels[l], o1 = t.levels[l + 1];
    run_level(t.ops, o0, o1, v, geo, (int)threadIdx.x, (int)blockDim.x, EvalD{});
    __syncthreads();
  }
}

__device__ inline void set_geom(OpGeom& g, const double PA[3], const double WP[3], const double QC[3],
                                const double WQ[3], const double AB[3], const double CD[3], double oz, double oe,
                                double oze, double roz, double roe) {
  for (int k = 0; k < 3; ++k) {
    g.G1[0][k] = PA[k]; g.G2[0][k] = WP[k];
    g.G1[1][k] = QC[k]; g.G2[1][k] = WQ[k];
    g.G1[2][k] = 1.0;   g.G2[2][k] = AB[k];
    g.G1[3][k] = 1.0;   g.G2[3][k] = CD[k];
  }
  g.X[0] = oz; g.Y[0] = roz; g.X[1] = oe; g.Y[1] = roe; g.X[2] = g.X[3] = 0.0; g.Y[2] = g.Y[3] = 0.0;
  g.Z = oze;
}


__device__ __forceinline__ double dens_at(const double* __restrict__ D, int npgs, int i, int j) {
  return (i >= 0 && j >= 0) ? __ldg(D + i + (size_t)npgs * j) : 0.0;
}

// class index of a canonical pair (LA >= LB): 00,10,11,20,21,22
__host__ __device__ inline int pair_class(int la, int lb) { return la * (la + 1) / 2 + lb; }

template <int LA, int LB>
__device__ double schwarz_pair(const double* __restrict__ tab, double zeta, double S, const double PA[3],
                               const double AB[3], const int* __restrict__ pa, const int* __restrict__ pb,
                               const double* __restrict__ maxc) {
  constexpr int NA = ncum(LA), NB = ncum(LB);
  // (ab|ab) at T = 0: F_m = C2/(2m+1), C2 = 2 sqrt(rho/PI) S^2, rho = zeta/2
  const double rho = 0.5 * zeta;
  const double c2 = 2.0 * sqrt(rho / REF_PI) * S * S;
  if (LA + LB == 0) return sqrt(c2 * maxc[pa[0]] * maxc[pb[0]]);
  double F[2 * (LA + LB) + 1];
#pragma unroll
  for (int m = 0; m <= 2 * (LA + LB); ++m) F[m] = c2 / (double)(2 * m + 1);
  EriGeom<double> g;
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    g.PA[k] = PA[k]; g.QC[k] = PA[k]; g.AB[k] = AB[k]; g.CD[k] = AB[k]; g.WP[k] = 0.0; g.WQ[k] = 0.0;
  }
  g.oz = 0.5 / zeta; g.oe = 0.5 / zeta; g.oze = 0.25 / zeta; g.roz = 0.5; g.roe = 0.5;
  double out[NA * NB * NA * NB];
  eri_dispatch<LA, LB, LA, LB>(F, g, out);
  double best = 0.0;
#pragma unroll 1
  for (int a = 0; a < NA; ++a)
    for (int b = 0; b < NB; ++b) {
      if (a == 0 && b == 0) continue;  // component 1 is excluded (src/pfourindexdirect.f90:356,455)
      const int ia = pa[a], ib = pb[b];
      const double ma = ia >= 0 ? maxc[ia] : 0.0, mb = ib >= 0 ? maxc[ib] : 0.0;
      const double v = sqrt(out[((a * NB + b) * NA + a) * NB + b] * ma * mb);
      if (v > best) best = v;
    }
  return best;
}


// Schwarz bound of the (21) and (22) pair classes on the interpreter: one block per pair.
template <int LA, int LB>
__global__ void __launch_bounds__(256) k_schwarz_big(PairArrays pr, const int* __restrict__ prim,
                                                     const double* __restrict__ maxc, const int* __restrict__ list,
                                                     int n, OpTableDev tab) {
  constexpr int NA = ncum(LA), NB = ncum(LB);
  extern __shared__ double smem[];
  double* v = smem;
  __shared__ OpGeom geo;
  __shared__ double best[256];
  for (int w = blockIdx.x; w < n; w += gridDim.x) {
    const int t = list[w];
    const double z = pr.zeta[t], S = pr.S[t];
    if (threadIdx.x == 0) {
      const double rho = 0.5 * z, c2 = 2.0 * sqrt(rho / REF_PI) * S * S;
      v[0] = 0.0;
      for (int m = 0; m <= 2 * (LA + LB); ++m) v[1 + m] = c2 / (double)(2 * m + 1);
      double PA[3], AB[3], Z0[3] = {0.0, 0.0, 0.0};
      for (int k = 0; k < 3; ++k) { PA[k] = pr.PA[k][t]; AB[k] = pr.AB[k][t]; }
      set_geom(geo, PA, Z0, PA, Z0, AB, AB, 0.5 / z, 0.5 / z, 0.25 / z, 0.5, 0.5);
    }
    __syncthreads();
    run_optable(tab, v, geo);
    const int I = pr.si[t], J = pr.sj[t];
    double b = 0.0;
    for (int x = threadIdx.x; x < NA * NB; x += blockDim.x) {
      const int a = x / NB, bb = x % NB;
      if (a == 0 && bb == 0) continue;
      const int ia = prim[I * MAXCOMP + a], ib = prim[J * MAXCOMP + bb];
      const double ma = ia >= 0 ? maxc[ia] : 0.0, mb = ib >= 0 ? maxc[ib] : 0.0;
      const double val = sqrt(v[tab.out[((a * NB + bb) * NA + a) * NB + bb]] * ma * mb);
      b = fmax(b, val);
    }
    best[threadIdx.x] = b;
    __syncthreads();
    if (threadIdx.x == 0) {
      double m = 0.0;
      for (int k = 0; k < (int)blockDim.x; ++k) m = fmax(m, best[k]);
      pr.schwarz[t] = m;
      pr.key[t] = ~(unsigned long long)__double_as_longlong(m);
    }
    __syncthreads();
  }
}

}  // namespace pfe
