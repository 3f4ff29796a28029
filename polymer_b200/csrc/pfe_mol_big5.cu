// Batch instantiations (launch record per chunk) of the large FP64 register-pass
// classes (21|11), (21|20), (22|10); dispatch in pfe_mol_big1.cu.

#include "pfe_mol_kernels.cuh"

namespace pfe {

template void launch_q<2, 1, 1, 1, 14, false, true>(const MolLaunch&, int, cudaStream_t);
template void launch_q<2, 1, 2, 0, 10, false, true>(const MolLaunch&, int, cudaStream_t);
template void launch_q<2, 2, 1, 0, 10, false, true>(const MolLaunch&, int, cudaStream_t);

}  // namespace pfe
