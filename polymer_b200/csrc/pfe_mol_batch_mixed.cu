// Mixed-precision (FP32 recursion) instantiations of the straight-line
// molecular kernels for batches.

#include "pfe_mol_kernels.cuh"

namespace pfe {

LaunchFn straight_launcher_batch_mixed(int cb, int ck) { return straight_launcher_t<true, true>(cb, ck); }

}  // namespace pfe
