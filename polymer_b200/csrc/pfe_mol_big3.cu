// FP64 register-pass instantiations of large quartet classes ((22|20)),
// compiled apart so the build runs them in parallel; the dispatch is in
// pfe_mol_big1.cu.

#include "pfe_mol_kernels.cuh"

namespace pfe {

template void launch_q<2, 2, 2, 0, 25, false, false>(const MolLaunch&, int, cudaStream_t);

}  // namespace pfe
