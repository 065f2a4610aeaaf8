// GpuTimeIntegrator: the reference-side shim that makes libdgp a drop-in for
// DG-Parallel's explicit integrator (RungeKuttaTVD3::advanceInTime,
// TimeIntegrator.h:28, created by DGAnalysis.cc:233-243).  Compiled with
// DG-Parallel's headers and linked against libdgp.so: the coefficients of the
// reference's DGCells go to the device before a step and come back after it,
// so the reference's own driver, CFL reduction, sensors and output keep
// working on host data.
#ifndef DGP_GPU_TIME_INTEGRATOR_H
#define DGP_GPU_TIME_INTEGRATOR_H

#include <typeinfo>
#include <vector>

#include "Burgers.h"
#include "DGCell.h"
#include "EulerLaw.h"
#include "MaxwellLaw.h"
#include "ScalarLaw.h"
#include "TimeIntegrator.h"
#include "dgp.h"
#include "mException.h"

// GpuConservationLaw: the library's law and numerical-flux ids of a
// DG-Parallel law object (ConservationLaw.h:12-60), by its dynamic type: each
// class whose riemannSolver the library has kernels for maps to one pair.
// Subclasses with other Riemann solvers (EulervanLeer, Euler2dHLLC,
// Euler2dExactRiemann, Euler3dRoe, ...) have none and are refused.
struct GpuConservationLaw {
  static bool map(const ConservationLaw* law, int* kind, int* flux) {
    const std::type_info& t = typeid(*law);
    if (t == typeid(Euler2dRoe)) return set(DGP_LAW_EULER2D, DGP_FLUX_ROE, kind, flux);
    if (t == typeid(Euler2d)) return set(DGP_LAW_EULER2D, DGP_FLUX_GODUNOV, kind, flux);
    if (t == typeid(Euler3d)) return set(DGP_LAW_EULER3D, DGP_FLUX_GODUNOV, kind, flux);
    if (t == typeid(ScalarLaw)) return set(DGP_LAW_SCALAR, DGP_FLUX_UPWIND, kind, flux);
    if (t == typeid(Burgers2D)) return set(DGP_LAW_BURGERS2D, DGP_FLUX_CENTRAL, kind, flux);
    if (t == typeid(Maxwell2d)) return set(DGP_LAW_MAXWELL2D, DGP_FLUX_UPWIND, kind, flux);
    return false;
  }
  static int kind(const ConservationLaw* law) {
    int k, f;
    if (!map(law, &k, &f)) throw new mException(__LINE__, __FILE__, (char*)"no GPU kernels for this ConservationLaw");
    return k;
  }
  static int flux(const ConservationLaw* law) {
    int k, f;
    if (!map(law, &k, &f)) throw new mException(__LINE__, __FILE__, (char*)"no GPU kernels for this ConservationLaw");
    return f;
  }

 private:
  static bool set(int k, int f, int* kind, int* flux) {
    *kind = k;
    *flux = f;
    return true;
  }
};

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
  // the same, with the law and flux ids read off the reference law object;
  // the field evaluator (a host callback) is named by id
  GpuTimeIntegrator(mDGMesh* m, ConservationLaw* law, int order, const char* msh,
                    const std::vector<DGCell*>& cells, int field, const double* params,
                    int precision = DGP_PRECISION_FP64)
      : GpuTimeIntegrator(m, law, order, msh, cells, GpuConservationLaw::kind(law), GpuConservationLaw::flux(law),
                          field, params, precision) {}
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
