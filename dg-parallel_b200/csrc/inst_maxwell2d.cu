// Kernel instantiations: Maxwell2d (fields Hx, Hy, Ez) on triangles P0-P4.
#include "dgp_ops.cuh"

namespace dgp {
void register_maxwell2d_ops() {
  add_ops<DGP_LAW_MAXWELL2D, DGP_FLUX_UPWIND, 2, 0>();
  add_ops<DGP_LAW_MAXWELL2D, DGP_FLUX_UPWIND, 2, 1>();
  add_ops<DGP_LAW_MAXWELL2D, DGP_FLUX_UPWIND, 2, 2>();
  add_ops<DGP_LAW_MAXWELL2D, DGP_FLUX_UPWIND, 2, 3>();
  add_ops<DGP_LAW_MAXWELL2D, DGP_FLUX_UPWIND, 2, 4>();
}
}  // namespace dgp
