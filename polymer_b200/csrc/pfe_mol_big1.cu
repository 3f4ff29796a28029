// FP64 register-pass instantiations of large quartet classes ((21|11), (21|20), (22|10)),
// compiled apart so the build runs them in parallel; the dispatch over all
// large classes (single molecules and batches) is here.

#include "pfe_mol_kernels.cuh"

namespace pfe {

template void launch_q<2, 1, 1, 1, 14, false, false>(const MolLaunch&, int, cudaStream_t);
template void launch_q<2, 1, 2, 0, 10, false, false>(const MolLaunch&, int, cudaStream_t);
template void launch_q<2, 2, 1, 0, 10, false, false>(const MolLaunch&, int, cudaStream_t);

extern template void launch_q<2, 1, 2, 1, 40, false, false>(const MolLaunch&, int, cudaStream_t);
extern template void launch_q<2, 2, 2, 0, 25, false, false>(const MolLaunch&, int, cudaStream_t);
extern template void launch_q<2, 2, 1, 1, 50, false, false>(const MolLaunch&, int, cudaStream_t);
extern template void launch_q<2, 1, 1, 1, 14, false, true>(const MolLaunch&, int, cudaStream_t);
extern template void launch_q<2, 1, 2, 0, 10, false, true>(const MolLaunch&, int, cudaStream_t);
extern template void launch_q<2, 2, 1, 0, 10, false, true>(const MolLaunch&, int, cudaStream_t);
extern template void launch_q<2, 1, 2, 1, 40, false, true>(const MolLaunch&, int, cudaStream_t);
extern template void launch_q<2, 2, 2, 0, 25, false, true>(const MolLaunch&, int, cudaStream_t);
extern template void launch_q<2, 2, 1, 1, 50, false, true>(const MolLaunch&, int, cudaStream_t);

template <bool BATCH>
static LaunchFn big_table(int cb, int ck) {
  switch (cb * 8 + ck) {
    case 4 * 8 + 2: return &launch_q<2, 1, 1, 1, 14, false, BATCH>;
    case 4 * 8 + 3: return &launch_q<2, 1, 2, 0, 10, false, BATCH>;
    case 4 * 8 + 4: return &launch_q<2, 1, 2, 1, 40, false, BATCH>;
    case 5 * 8 + 1: return &launch_q<2, 2, 1, 0, 10, false, BATCH>;
    case 5 * 8 + 2: return &launch_q<2, 2, 1, 1, 50, false, BATCH>;
    case 5 * 8 + 3: return &launch_q<2, 2, 2, 0, 25, false, BATCH>;
    default: return nullptr;
  }
}

LaunchFn straight_launcher_big(int cb, int ck, bool batch) { return batch ? big_table<true>(cb, ck) : big_table<false>(cb, ck); }

}  // namespace pfe
