// Mixed-precision (FP32 recursion) instantiations of the straight-line
// molecular kernels, compiled apart from the FP64 ones in pfe_mol.cu.

#include "pfe_mol_kernels.cuh"

namespace pfe {

LaunchFn straight_launcher_mixed(int cb, int ck) { return straight_launcher_t<true>(cb, ck); }

}  // namespace pfe
