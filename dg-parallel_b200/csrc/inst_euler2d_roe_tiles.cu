// Kernel instantiations: Euler2d with the roe flux on triangles P1-P4 with 64-
// and 256-thread tiles (autotuner candidates).
#include "dgp_ops.cuh"

namespace dgp {
void register_euler2d_roe_tile_ops() {
  add_tile_ops<DGP_LAW_EULER2D, DGP_FLUX_ROE, 2, 1>();
  add_tile_ops<DGP_LAW_EULER2D, DGP_FLUX_ROE, 2, 2>();
  add_tile_ops<DGP_LAW_EULER2D, DGP_FLUX_ROE, 2, 3>();
  add_tile_ops<DGP_LAW_EULER2D, DGP_FLUX_ROE, 2, 4>();
}
}  // namespace dgp
