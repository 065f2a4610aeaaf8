// Opaque handle types behind the C ABI (include/dgp.h) and the error helpers
// shared by the translation units that implement it.
#pragma once

#include <cuda_runtime.h>

#include <map>
#include <string>
#include <utility>
#include <vector>

#include "../../include/dgp.h"
#include "dgp_host.h"
#include "dgp_solver.h"

namespace dgp {
// records `msg` as the calling thread's dgp_last_error() and returns `code`
int fail(int code, const std::string& msg);
}  // namespace dgp

#define DGP_CUDA(call)                                                               \
  do {                                                                               \
    cudaError_t e_ = (call);                                                         \
    if (e_ != cudaSuccess)                                                           \
      return ::dgp::fail(DGP_ERR_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_)); \
  } while (0)

using dgp::fail;

struct dgp_mesh_s {
  dgp::HostMesh m;
};

struct dgp_law_s {
  int kind, flux, field;
  double p[DGP_NPARAMS];
  int nbc = 0;
  int bc_id[DGP_MAX_BC] = {};
  int bc_kind[DGP_MAX_BC] = {};
  // the device view of the law: parameters, field and boundary settings
  dgp::LawParams params() const {
    dgp::LawParams lp{};
    lp.field = field;
    for (int i = 0; i < DGP_NPARAMS; ++i) lp.p[i] = p[i];
    lp.nbc = nbc;
    for (int i = 0; i < nbc; ++i) {
      lp.bc_id[i] = bc_id[i];
      lp.bc_kind[i] = bc_kind[i];
    }
    return lp;
  }
};

// Discrete adjoint bookkeeping of a solver: checkpoints of the last
// dgp_forward_checkpointed, the stage states of one recomputed segment, the
// adjoint vectors and the receiver objective.
struct AdjointState {
  int nsteps = 0, every = 0, nseg = 0;
  double t0 = 0, dt = 0;
  double* ckpt = nullptr;   // (nseg + 1) states
  size_t ckpt_states = 0;
  double* store = nullptr;  // every x 3 stage states (u_n, u1, u2) of a segment
  size_t store_states = 0;
  double* lam = nullptr;    // lambda (input of the reversed step, output of it)
  double* lam2 = nullptr;
  double* lam1 = nullptr;
  double* acc = nullptr;
  double* t_seg = nullptr;  // device scalar
  // Barth limiter: its slope factors per (step, stage, cell, field) of the
  // steps whose stage states are kept (the frozen active set)
  double* slopes = nullptr;
  size_t slopes_n = 0;
  bool freeze = false;      // forward passes replay the recorded factors
  bool ready = false;       // a forward pass is recorded
  bool recorded = false;    // every stage state of the forward pass is kept (no recompute)
  // receivers: J = sum_r (rho(x_r) - obs_r)^2
  int nrec = 0;
  int* rcell = nullptr;
  double* rphi = nullptr;
  double* robs = nullptr;
  double* rrho = nullptr;
  double* rJ = nullptr;
};

struct dgp_probe_s;

// Local time stepping (RungeKuttaTVD2adaptive on the size bins of
// DGAnalysis::sortCellsBySize): bins and roles per internal cell, and device
// lists of the integrator's cell groups and face classes.  Group (g, b): g = 0
// inner cells of bin b, 1 large cells on interface b (bin b), 2 small cells on
// interface b (bin b + 1).  Face class c < nb: faces of bin c; nb + c: faces
// between bins c and c + 1.
struct LtsState {
  bool on = false;
  int nb = 0;
  std::vector<int> bin, role;        // internal cell order
  int* lists = nullptr;              // all lists below, concatenated
  int* fcls = nullptr;               // [F] class of each face
  int* cface = nullptr;              // [E][NLF] face of each local face
  double *c1 = nullptr, *save = nullptr, *racc = nullptr;  // copy slot, u_n, RHS accumulator
  std::vector<int> goff, gn;         // group (g, b) at 3 * b + g: offset and length
  std::vector<int> foff, fn;         // face class c: faces
  std::map<unsigned, std::pair<int, int>> lift;  // class set (bit c) -> offset, length of
                                                 // the cells touching its faces
};

struct dgp_solver_s {
  AdjointState adj;
  dgp::PointLocator locator;            // built on first use (receivers, probes)
  bool locator_ready = false;
  std::vector<dgp_probe_s*> probes;     // probes of this solver (recorders sample in every step)
  std::vector<dgp::HostMesh> meshes;  // one per instance (one for a single solver)
  std::vector<int> inst_off;          // first internal cell of each instance
  std::vector<int> inst_ufirst;       // first cell of each instance in the joined file order
  dgp::RefTables tab;
  dgp::Ops ops;
  dgp::DeviceBuffers b;
  int law = 0, flux = 0, order = 0, precision = 0, limiter = 0, device = 0;
  int rule = 0;  // quadrature rule option (DGP_RULE_*)
  cudaStream_t stream = nullptr;
  std::vector<int> i2f, f2i;  // internal <-> file cell order
  int* d_i2f = nullptr;
  int* d_f2i = nullptr;
  std::vector<void*> allocs;
  cudaGraphExec_t graph = nullptr;   // graph_steps SSP-RK3 steps
  cudaGraphExec_t graph1 = nullptr;  // one step (the tail of a run with a step limit)
  int graph_steps = 0;
  dgp::TimeCtl* h_ctl = nullptr;  // pinned, 2 entries
  LtsState lts;                    // local time stepping (off unless enabled)
  bool fused = false;              // stages run through the fused stage kernel
  bool fused_ok = false;           // the fused stage kernel is built for this solver
  bool tr_stale = false;           // the face-point traces (tr) lag the state (the fused
                                   // kernel keeps none; the local time stepping kernels read them)
  void drop_graphs() {
    if (graph) cudaGraphExecDestroy(graph);
    if (graph1) cudaGraphExecDestroy(graph1);
    graph = graph1 = nullptr;
  }
  ~dgp_solver_s();
  void destroy_resources() {
    drop_graphs();
    for (void* p : allocs) cudaFree(p);
    if (h_ctl) cudaFreeHost(h_ctl);
    if (stream) cudaStreamDestroy(stream);
  }
  template <typename U>
  int alloc(U** p, size_t count) {
    void* v = nullptr;
    if (count == 0) count = 1;
    cudaError_t e = cudaMalloc(&v, count * sizeof(U));
    if (e != cudaSuccess) return fail(DGP_ERR_NOMEM, std::string("cudaMalloc: ") + cudaGetErrorString(e));
    allocs.push_back(v);
    *p = static_cast<U*>(v);
    return DGP_OK;
  }
  // upload FP64 host data as the hot-path type
  int upload_t(void** dst, const std::vector<double>& src) {
    const size_t n = src.size();
    if (ops.tsize == 8) {
      double* d;
      if (int rc = alloc(&d, n)) return rc;
      DGP_CUDA(cudaMemcpy(d, src.data(), n * 8, cudaMemcpyHostToDevice));
      *dst = d;
    } else {
      std::vector<float> f(src.begin(), src.end());
      float* d;
      if (int rc = alloc(&d, n)) return rc;
      DGP_CUDA(cudaMemcpy(d, f.data(), n * 4, cudaMemcpyHostToDevice));
      *dst = d;
    }
    return DGP_OK;
  }
  template <typename U>
  int upload(U** dst, const std::vector<U>& src) {
    if (int rc = alloc(dst, src.size())) return rc;
    DGP_CUDA(cudaMemcpy(*dst, src.data(), src.size() * sizeof(U), cudaMemcpyHostToDevice));
    return DGP_OK;
  }
  size_t state_count() const { return static_cast<size_t>(b.E) * b.M * b.NP; }
};

// Point probes (DGPointSensor / DGLineSensor, DGSensor.cc:88-186): cells and
// basis values of the points, located once on the host; evaluated on the
// device, on demand or inside every step of a run (recorder).
struct dgp_probe_s {
  dgp_solver s = nullptr;  // cleared when the solver is destroyed first
  int n = 0, found = 0;
  int* cell = nullptr;     // [n] internal cell (-1: outside the mesh)
  double* phi = nullptr;   // [n][Np] basis values at the points
  double* vals = nullptr;  // [n][M]
  int every = 0, max_samples = 0;  // recorder: every `every` steps of a run
  double* rec = nullptr;           // [max_samples][n][M]
  double* rec_t = nullptr;         // [max_samples] times
  int* rec_n = nullptr;            // samples taken in the current run
  std::vector<void*> allocs;
  ~dgp_probe_s() {
    for (void* p : allocs) cudaFree(p);
  }
};

namespace dgp {
// point location on a single solver's mesh: internal cell (-1: outside) and
// basis values of each point (dgp_probe.cu)
int locate_points(dgp_solver s, int n, const double* points, std::vector<int>& cell, std::vector<double>& phi);
// probe recorders: launched at the end of every step; reset when a run starts
void launch_probe_recorders(dgp_solver s);
int reset_probe_recorders(dgp_solver s);
// local time stepping (dgp_lts.cu): one advanceInTime of the current ctl->dt,
// the step's end, and with next_dt the next step's CFL reduction; returns the
// number of kernels launched (dry: count only)
int launch_lts_step(dgp_solver s, bool next_dt, bool dry = false);
}  // namespace dgp

inline dgp_solver_s::~dgp_solver_s() {
  for (dgp_probe_s* p : probes) p->s = nullptr;
  destroy_resources();
}

struct dgp_ensemble_s {
  int n = 0;
  std::vector<dgp_solver> groups;       // one batched solver per (law, flux, element, order)
  std::vector<int> inst_group, inst_index;
};
