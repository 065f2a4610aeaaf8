// Kernel instantiations: ScalarLaw (upwind) on triangles P0-P4 and tets P0-P3;
// P2 also with the workloads' quadrature rule.
#include "dgp_ops.cuh"

namespace dgp {
void register_scalar_ops() {
  add_ops<DGP_LAW_SCALAR, DGP_FLUX_UPWIND, 2, 0>();
  add_ops<DGP_LAW_SCALAR, DGP_FLUX_UPWIND, 2, 1>();
  add_ops<DGP_LAW_SCALAR, DGP_FLUX_UPWIND, 2, 2>();
  add_ops<DGP_LAW_SCALAR, DGP_FLUX_UPWIND, 2, 3>();
  add_ops<DGP_LAW_SCALAR, DGP_FLUX_UPWIND, 2, 4>();
  add_ops<DGP_LAW_SCALAR, DGP_FLUX_UPWIND, 3, 0>();
  add_ops<DGP_LAW_SCALAR, DGP_FLUX_UPWIND, 3, 1>();
  add_ops<DGP_LAW_SCALAR, DGP_FLUX_UPWIND, 3, 2>();
  add_ops<DGP_LAW_SCALAR, DGP_FLUX_UPWIND, 3, 3>();
  // the workloads' quadrature point counts at P2 (DGP_RULE_WORKLOAD)
  add_ops<DGP_LAW_SCALAR, DGP_FLUX_UPWIND, 2, 2, kDefaultBlock, DGP_RULE_WORKLOAD>();
  add_ops<DGP_LAW_SCALAR, DGP_FLUX_UPWIND, 3, 2, kDefaultBlock, DGP_RULE_WORKLOAD>();
}
}  // namespace dgp
