// Kernel instantiations: Euler2d with the llf flux on triangles P0-P4.
#include "dgp_ops.cuh"

namespace dgp {
void register_euler2d_llf_ops() {
  add_ops<DGP_LAW_EULER2D, DGP_FLUX_LLF, 2, 0>();
  add_ops<DGP_LAW_EULER2D, DGP_FLUX_LLF, 2, 1>();
  add_ops<DGP_LAW_EULER2D, DGP_FLUX_LLF, 2, 2>();
  add_ops<DGP_LAW_EULER2D, DGP_FLUX_LLF, 2, 3>();
  add_ops<DGP_LAW_EULER2D, DGP_FLUX_LLF, 2, 4>();
}
}  // namespace dgp
