// FP64 register-pass instantiations of large quartet classes ((21|11), (21|20), (22|10)),
// compiled apart so the build runs them in parallel; the dispatch is in
// pfe_mol_big1.cu.

#include "pfe_mol_kernels.cuh"

namespace pfe {

template void launch_q<2, 1, 1, 1, 14, false>(const MolLaunch&, int, cudaStream_t);
template void launch_q<2, 1, 2, 0, 10, false>(const MolLaunch&, int, cudaStream_t);
template void launch_q<2, 2, 1, 0, 10, false>(const MolLaunch&, int, cudaStream_t);

extern template void launch_q<2, 1, 2, 1, 40, false>(const MolLaunch&, int, cudaStream_t);
extern template void launch_q<2, 2, 2, 0, 25, false>(const MolLaunch&, int, cudaStream_t);
extern template void launch_q<2, 2, 1, 1, 50, false>(const MolLaunch&, int, cudaStream_t);

LaunchFn straight_launcher_big(int cb, int ck) {
  switch (cb * 8 + ck) {
    case 4 * 8 + 2: return &launch_q<2, 1, 1, 1, 14, false>;
    case 4 * 8 + 3: return &launch_q<2, 1, 2, 0, 10, false>;
    case 4 * 8 + 4: return &launch_q<2, 1, 2, 1, 40, false>;
    case 5 * 8 + 1: return &launch_q<2, 2, 1, 0, 10, false>;
    case 5 * 8 + 2: return &launch_q<2, 2, 1, 1, 50, false>;
    case 5 * 8 + 3: return &launch_q<2, 2, 2, 0, 25, false>;
    default: return nullptr;
  }
}

}  // namespace pfe
