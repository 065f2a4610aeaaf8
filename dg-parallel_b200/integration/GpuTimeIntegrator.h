// GpuTimeIntegrator: the reference-side shim that makes libdgp a drop-in for
// DG-Parallel's explicit integrator (RungeKuttaTVD3::advanceInTime,
// TimeIntegrator.h:28, created by DGAnalysis.cc:233-243).  Compiled with
// DG-Parallel's headers and linked against libdgp.so: the coefficients of the
// reference's DGCells go to the device before a step and come back after it,
// so the reference's own driver, CFL reduction, sensors and output keep
// working on host data.
#ifndef DGP_GPU_TIME_INTEGRATOR_H
#define DGP_GPU_TIME_INTEGRATOR_H

#include <vector>

#include "DGCell.h"
#include "TimeIntegrator.h"
#include "dgp.h"
#include "mException.h"

class GpuTimeIntegrator : public TimeIntegrator {
 public:
  // `msh` is the file DG-Parallel imported; `cells` lists the DGCells in the
  // order of the cell elements in that file (the shim's state layout).
  GpuTimeIntegrator(mDGMesh* m, ConservationLaw* law, int order, const char* msh,
                    const std::vector<DGCell*>& cells, int lawKind, int flux, int field,
                    const double* params /* DGP_NPARAMS */, int precision = DGP_PRECISION_FP64)
      : TimeIntegrator(m, 0, law->getNbFields(), 0), cells_(cells) {
    check(dgp_mesh_from_msh(msh, &mesh_));
    check(dgp_law_create(lawKind, flux, field, params, &law_));
    check(dgp_solver_create(mesh_, law_, order, precision, DGP_LIMITER_NONE, &s_));
    int nf, np, e, f;
    check(dgp_solver_info(s_, &nf, &np, &e, &f));
    dof_ = nf * np;
    buf_.resize((size_t)e * dof_);
  }
  ~GpuTimeIntegrator() {
    dgp_solver_destroy(s_);
    dgp_law_destroy(law_);
    dgp_mesh_destroy(mesh_);
  }

  // RungeKuttaTVD3::advanceInTime(t, dt): same arguments, same returned residual
  double advanceInTime(double t, double dt) {
    pushCoefficients();
    double resid = 0;
    check(dgp_step(s_, t, dt, &resid));
    pullCoefficients();
    return resid;
  }

 private:
  void pushCoefficients() {
    for (size_t e = 0; e < cells_.size(); ++e)
      for (int i = 0; i < dof_; ++i) buf_[e * dof_ + i] = cells_[e]->theFieldsCoefficients->get()[i];
    check(dgp_set_state(s_, buf_.data()));
  }
  void pullCoefficients() {
    check(dgp_get_state(s_, buf_.data()));
    for (size_t e = 0; e < cells_.size(); ++e) {
      for (int i = 0; i < dof_; ++i) cells_[e]->theFieldsCoefficients->get()[i] = buf_[e * dof_ + i];
      cells_[e]->computeMean();
    }
  }
  static void check(int rc) {
    if (rc != DGP_OK) throw new mException(__LINE__, __FILE__, (char*)dgp_last_error());
  }
  dgp_mesh mesh_ = 0;
  dgp_law law_ = 0;
  dgp_solver s_ = 0;
  int dof_ = 0;
  std::vector<DGCell*> cells_;
  std::vector<double> buf_;
};

#endif
