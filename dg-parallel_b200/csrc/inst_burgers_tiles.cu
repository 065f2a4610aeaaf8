// Kernel instantiations: Burgers2D (central and Lax-Friedrichs) on triangles
// P1-P4 with 64- and 256-thread tiles (autotuner candidates).
#include "dgp_ops.cuh"

namespace dgp {
void register_burgers_tile_ops() {
  add_tile_ops<DGP_LAW_BURGERS2D, DGP_FLUX_CENTRAL, 2, 1>();
  add_tile_ops<DGP_LAW_BURGERS2D, DGP_FLUX_CENTRAL, 2, 2>();
  add_tile_ops<DGP_LAW_BURGERS2D, DGP_FLUX_CENTRAL, 2, 3>();
  add_tile_ops<DGP_LAW_BURGERS2D, DGP_FLUX_CENTRAL, 2, 4>();
  add_tile_ops<DGP_LAW_BURGERS2D, DGP_FLUX_LLF, 2, 1>();
  add_tile_ops<DGP_LAW_BURGERS2D, DGP_FLUX_LLF, 2, 2>();
  add_tile_ops<DGP_LAW_BURGERS2D, DGP_FLUX_LLF, 2, 3>();
  add_tile_ops<DGP_LAW_BURGERS2D, DGP_FLUX_LLF, 2, 4>();
}
}  // namespace dgp
