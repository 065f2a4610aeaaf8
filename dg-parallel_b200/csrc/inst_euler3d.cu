// Kernel instantiations: Euler3d (exact Riemann solver) on tets P0-P3.
#include "dgp_ops.cuh"

namespace dgp {
void register_euler3d_ops() {
  add_ops<DGP_LAW_EULER3D, DGP_FLUX_GODUNOV, 3, 0>();
  add_ops<DGP_LAW_EULER3D, DGP_FLUX_GODUNOV, 3, 1>();
  add_ops<DGP_LAW_EULER3D, DGP_FLUX_GODUNOV, 3, 2>();
  add_ops<DGP_LAW_EULER3D, DGP_FLUX_GODUNOV, 3, 3>();
}
}  // namespace dgp
