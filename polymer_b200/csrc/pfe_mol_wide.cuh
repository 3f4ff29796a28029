// The warp-per-primitive-quartet variant of the large molecular quartet
// classes (pfe_mol_wide.cu): launcher, shared-memory opt-in and per-warp size.
#pragma once

#include "pfe_interp.cuh"
#include "pfe_mol_kernels.cuh"

namespace pfe {

struct WideVariant {
  // grid blocks of wpb warps; per_warp doubles of shared memory per warp, of which
  // vmax hold the op-table slots and xmax the kept outputs of a group quartet
  void (*launch)(const MolLaunch&, const OpTableDev&, int grid, int wpb, int per_warp, int vmax, int xmax,
                 size_t smem, cudaStream_t);
  cudaError_t (*allow)(size_t smem);
  int (*doubles)(int vmax, int xmax);
};

// The classes that have the variant: (21|11), (21|20), (21|21), (22|10),
// (22|11), (22|20), (22|21), (22|22); null members otherwise.
WideVariant wide_variant(int cb, int ck);

}  // namespace pfe
