// FP64 instantiations of the straight-line molecular kernels for batches (each
// chunk reads its molecule's launch record), compiled apart so the build runs
// them in parallel with the single-molecule ones.

#include "pfe_mol_kernels.cuh"

namespace pfe {

LaunchFn straight_launcher_batch(int cb, int ck) { return straight_launcher_t<false, true>(cb, ck); }

}  // namespace pfe
