// Kernel instantiations: Burgers2D (central and Lax-Friedrichs) on triangles P0-P4.
#include "dgp_ops.cuh"

namespace dgp {
void register_burgers_ops() {
  add_ops<DGP_LAW_BURGERS2D, DGP_FLUX_CENTRAL, 2, 0>();
  add_ops<DGP_LAW_BURGERS2D, DGP_FLUX_CENTRAL, 2, 1>();
  add_ops<DGP_LAW_BURGERS2D, DGP_FLUX_CENTRAL, 2, 2>();
  add_ops<DGP_LAW_BURGERS2D, DGP_FLUX_CENTRAL, 2, 3>();
  add_ops<DGP_LAW_BURGERS2D, DGP_FLUX_CENTRAL, 2, 4>();
  add_ops<DGP_LAW_BURGERS2D, DGP_FLUX_LLF, 2, 0>();
  add_ops<DGP_LAW_BURGERS2D, DGP_FLUX_LLF, 2, 1>();
  add_ops<DGP_LAW_BURGERS2D, DGP_FLUX_LLF, 2, 2>();
  add_ops<DGP_LAW_BURGERS2D, DGP_FLUX_LLF, 2, 3>();
  add_ops<DGP_LAW_BURGERS2D, DGP_FLUX_LLF, 2, 4>();
}
}  // namespace dgp
