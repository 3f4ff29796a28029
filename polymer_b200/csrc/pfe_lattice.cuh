// Lattice/helix path state shared by the interpreter (pfe_lattice.cu) and the
// straight-line kernels (pfe_lattice_sl.cu).
#pragma once

#include "pfe_common.cuh"
#include "pfe_context.cuh"

namespace pfe {

struct LatGeom {
  int c1[3], c2[3];
  int n1[3];
  double period[3];
  double helix;
};

__device__ __forceinline__ int cell1_index(const LatGeom& g, int qx, int qy, int qz) {
  return (qx + g.c1[0]) + g.n1[0] * ((qy + g.c1[1]) + g.n1[1] * (qz + g.c1[2]));
}

struct LatticeRun {
  PairArrays pairs;
  const unsigned char* swp;
  const int* prim;
  const double* boys;
  const double* pp;    // P_P (npgs,npgs,cells1)
  const double* pph;   // P_P_HELIX or null
  double* cp;          // C_P (npgs,npgs,cells1)
  double* xp;
  const int4* chunks;
  const int* nchunks;
  const int4* tickets;
  const int* qcell;
  LatGeom g;
  int npgs;
  // mixed precision: ket images Q3 outside the CUTOFF1 box (the far cells) run
  // the recursion in FP32, the rest in FP64; n32 counts the FP32 quartets
  int far32;
  unsigned long long* n32;
  int* queue;          // chunk counter of the straight-line kernels, zero at launch
};

// The straight-line kernel of evaluated class (e1|e2) (e1 >= e2, swap: the
// chunk's bra class is e2) on `grid` blocks of 128 threads, or null where the
// class has more than 64 integrals (it keeps the op-table interpreter).
// work-queue counters per lattice class launch (one per register pass)
constexpr int kLatQueueSlots = 4;
using LatSlFn = void (*)(const LatticeRun&, int grid, cudaStream_t);
LatSlFn lattice_sl_launcher(int e1, int e2, bool sw);
// launches (register passes) of a straight-line class, 0 where the class has none
int lattice_sl_passes(int e1, int e2);

}  // namespace pfe
