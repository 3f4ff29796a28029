// General (lattice / helix) path of the Fock build -- placeholder until the
// cell-triple kernels land; molecules take pfe_eri.cu.
#include "pfe_common.cuh"
#include "pfe_context.cuh"

namespace pfe {
int lattice_setup(pfe_context* ctx, const pfe_args* a) {
  (void)ctx; (void)a;
  set_error("periodic / helical inputs are not implemented yet");
  return PFE_EUNSUPPORTED;
}
int lattice_fock(pfe_context*, const double*, const double*, double*, double*, cudaStream_t) {
  set_error("periodic / helical inputs are not implemented yet");
  return PFE_EUNSUPPORTED;
}
void lattice_release(pfe_context* ctx) { ctx->lattice = nullptr; }
}  // namespace pfe
