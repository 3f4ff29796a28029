// Batch instantiation (launch record per chunk) of the large FP64 register-pass
// class (22|11); dispatch in pfe_mol_big1.cu.

#include "pfe_mol_kernels.cuh"

namespace pfe {

template void launch_q<2, 2, 1, 1, 50, false, true>(const MolLaunch&, int, cudaStream_t);

}  // namespace pfe
