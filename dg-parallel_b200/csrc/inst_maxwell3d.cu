// Kernel instantiations: 3D Maxwell (upwind) on tets P0-P3; P2 also with the
// workloads' quadrature rule.
#include "dgp_ops.cuh"

namespace dgp {
void register_maxwell3d_ops() {
  add_ops<DGP_LAW_MAXWELL3D, DGP_FLUX_UPWIND, 3, 0>();
  add_ops<DGP_LAW_MAXWELL3D, DGP_FLUX_UPWIND, 3, 1>();
  add_ops<DGP_LAW_MAXWELL3D, DGP_FLUX_UPWIND, 3, 2>();
  add_ops<DGP_LAW_MAXWELL3D, DGP_FLUX_UPWIND, 3, 3>();
  // the workloads' quadrature point counts at P2 (DGP_RULE_WORKLOAD)
  add_ops<DGP_LAW_MAXWELL3D, DGP_FLUX_UPWIND, 3, 2, kDefaultBlock, DGP_RULE_WORKLOAD>();
}
}  // namespace dgp
