// Solver object behind the C ABI: device buffers in the internal (Morton)
// cell order and the kernel set of one (law, flux, dim, order, precision).
#pragma once

#include <cuda_runtime.h>

#include <map>
#include <string>
#include <tuple>
#include <vector>

#include "dgp_host.h"
#include "dgp_kernels.cuh"
#include "dgp_lts.cuh"

namespace dgp {

// Device buffers; pointers typed as void* hold the hot-path precision T.
struct DeviceBuffers {
  int E = 0, F = 0, NB = 0, order = 0, dim = 0, M = 0, NP = 0;
  void* jinv = nullptr;
  void* detj = nullptr;
  double* detjd = nullptr;
  double* csize = nullptr;
  double* x0 = nullptr;
  double* jac = nullptr;
  int* fel = nullptr;
  int* fcode = nullptr;
  void* fnrm = nullptr;
  void* fj = nullptr;
  double* bpts = nullptr;
  int* bbid = nullptr;
  int* bpart = nullptr;
  void* bpphi = nullptr;
  void* blob = nullptr;   // element-kernel tables in shared-memory layout
  void* fblob = nullptr;  // the fused stage kernel's tables (gradient rows in its G order)
  int blob_bytes = 0;
  void* phi = nullptr;
  void* dphi = nullptr;
  void* qw = nullptr;
  void* phif = nullptr;
  void* fqw = nullptr;
  int* qmap = nullptr;
  double* phiv = nullptr;
  void* phimax = nullptr;  // largest |phi_k| over volume and face points
  double* phiq = nullptr;
  double* qwd = nullptr;
  double* qpd = nullptr;
  int nqe = 0;
  double* eqp = nullptr;
  double* eqw = nullptr;
  double* ephi = nullptr;
  double phi0 = 0.0;
  void* C = nullptr;      // state [cell][field][mode], updated in place by the stages
  void* Cout = nullptr;   // when set, the stages write here instead of into C
  void* U0 = nullptr;     // u_n of the current step
  void* slots = nullptr;  // per-cell face slots
  void* tr = nullptr;     // face-point traces of C (slot layout)
  void* rhs = nullptr;    // assembled RHS for dgp_rhs
  void* scratch = nullptr;// state-sized staging for device-side set/get
  void* X1 = nullptr;     // stage states u1, u2 of the fused stage kernel (the state C holds u_n)
  void* X2 = nullptr;
  TileMesh tm{};          // per-tile face records and halos of the fused stage kernel
  int mbar_polls = 0;     // bound of the fused kernel's first bulk-copy wait (0: default)
  int tensor_cores = 0;   // mixed form: volume contraction on the tensor cores (tcgen05)
  int round_mask = 0;     // FP64 rounding probe of the fused kernel (error decomposition; 0: off)
  TimeCtl* ctl = nullptr;
  Status* status = nullptr;
  double* partials = nullptr;
  int npartials = 0;
  LawParams law{};
  // P0 fallback and triangle moment limiter
  int p0 = 0;                     // 1: DGCell::setToZero fallback on
  unsigned char* bad = nullptr;   // [E] P0 marks
  int limiter_kind = 0;           // DGP_LIMITER_* of the solver
  int* cface = nullptr;           // Barth: [E][NLF] face of each local face
  double* bphif = nullptr;        // Barth: FP64 face-point basis values [NLF * NQF][NP]
  unsigned char* trig = nullptr;  // [E * M] trigger degree of each row in the last limiter pass
  double* lim_slope = nullptr;    // Barth: [E][M] slope factors of the pass (written; read when replayed)
  int lim_replay = 0;             // Barth: 1 applies lim_slope instead of computing the factors
  unsigned char* lbig = nullptr;  // [E * M] degrees with a mode above the limiter's threshold
  double* lmo = nullptr;          // [E * M][NP] moments of every degree of each row
  int* nb = nullptr;              // [E][4] left, right, bottom, top
  double* lgeo = nullptr;         // [E][10] limiter geometry
  double* limD = nullptr;         // derivative tables per degree
  double* limDinv = nullptr;
  // ensembles (nullptr / 0 for a single solver; then gctl == ctl)
  TimeCtl* gctl = nullptr;
  int* cell_inst = nullptr;
  int* inst_end = nullptr;
  int* tile_first = nullptr;
  LawParams* laws = nullptr;
  int ninst = 0;
};

template <typename T>
inline StageArgs<T> make_args(const DeviceBuffers& b) {
  StageArgs<T> a{};
  a.mesh.E = b.E;
  a.mesh.F = b.F;
  a.mesh.NB = b.NB;
  a.mesh.jinv = static_cast<const T*>(b.jinv);
  a.mesh.detj = static_cast<const T*>(b.detj);
  a.mesh.detjd = b.detjd;
  a.mesh.csize = b.csize;
  a.mesh.x0 = b.x0;
  a.mesh.jac = b.jac;
  a.mesh.fel = b.fel;
  a.mesh.fcode = b.fcode;
  a.mesh.fnrm = static_cast<const T*>(b.fnrm);
  a.mesh.fj = static_cast<const T*>(b.fj);
  a.mesh.bpts = b.bpts;
  a.mesh.bbid = b.bbid;
  a.mesh.bpart = b.bpart;
  a.mesh.bpphi = static_cast<const T*>(b.bpphi);
  a.tab.blob = static_cast<const T*>(b.blob);
  a.tab.blob_bytes = b.blob_bytes;
  a.tab.phi = static_cast<const T*>(b.phi);
  a.tab.dphi = static_cast<const T*>(b.dphi);
  a.tab.qw = static_cast<const T*>(b.qw);
  a.tab.phif = static_cast<const T*>(b.phif);
  a.tab.fqw = static_cast<const T*>(b.fqw);
  a.tab.qmap = b.qmap;
  a.tab.phiv = b.phiv;
  a.tab.phimax = static_cast<const T*>(b.phimax);
  a.tab.phiq = b.phiq;
  a.tab.qwd = b.qwd;
  a.tab.qpd = b.qpd;
  a.tab.nqe = b.nqe;
  a.tab.eqp = b.eqp;
  a.tab.eqw = b.eqw;
  a.tab.ephi = b.ephi;
  a.tab.phi0 = b.phi0;
  a.law = b.law;
  a.tm = b.tm;
  a.mbar_polls = b.mbar_polls;
  a.round_mask = b.round_mask;
  a.C = static_cast<const double*>(b.C);
  a.U0 = static_cast<const double*>(b.U0);
  a.Cout = static_cast<double*>(b.Cout ? b.Cout : b.C);
  a.U0out = static_cast<double*>(b.U0);
  a.slots = static_cast<T*>(b.slots);
  a.tr = static_cast<T*>(b.tr);
  a.ctl = b.ctl;
  a.status = b.status;
  a.partials = b.partials;
  a.bad = b.bad;
  a.gctl = b.gctl ? b.gctl : b.ctl;
  a.cell_inst = b.cell_inst;
  a.inst_end = b.inst_end;
  a.tile_first = b.tile_first;
  a.laws = b.laws;
  a.ninst = b.ninst;
  a.order = b.order;
  return a;
}

// One reversed stage of the discrete adjoint: out = ca mu + cb dt w + cc acc,
// acc <- cd acc + ce mu, with w the transposed linearised L at the stage
// state (b.C) and the stage time *t_seg + t_factor * dt (t_seg: the step's
// start time, t_factor 0, 1, 0.5 as the forward stage).
struct AdjStage {
  const double* mu;
  double* out;
  double* acc;
  double ca, cb, cc, cd, ce, dt;
  const double* t_seg;
  double t_factor;
};

// Kernel set of one instantiation.
struct Ops {
  int M = 0, NP = 0, NQ = 0, NQF = 0, TE = 0, elem_block = 0, precision = 0;
  int fpb = 0;  // faces per face-kernel CTA
  size_t elem_smem = 0;
  size_t tsize = 8;
  size_t blob_elems = 0;
  // writes the element-kernel table blob (FP64) from dphi [KV][NP], phif [NS][NP],
  // phi [NQ][NP], qw [NQ]
  void (*fill_blob)(const double*, const double*, const double*, const double*, double*) = nullptr;
  void (*fill_fused_blob)(const double*, const double*, const double*, const double*, double*) = nullptr;
  size_t fused_blob_elems = 0;
  bool tensor_cores_ok = false;  // the fused kernel has a tensor-core contraction for this shape
  bool probe_ok = false;         // the fused kernel has the rounding probe for this configuration
  cudaError_t (*prepare)() = nullptr;
  // one SSP-RK3 stage (face kernel + element kernel); stage 0 writes the RHS
  void (*stage)(const DeviceBuffers&, int stage, double time_factor, int fuse_cfl, cudaStream_t) = nullptr;
  void (*face)(const DeviceBuffers&, int stage, double time_factor, cudaStream_t) = nullptr;
  void (*elem)(const DeviceBuffers&, int stage, int fuse_cfl, cudaStream_t) = nullptr;
  // fused stage kernel: reads the stage input `in` (this tile's and its halo's
  // rows) and u_n, writes `out` (stage 0: the RHS); u0copy, when set, receives
  // the input rows in stage 1
  void (*fused)(const DeviceBuffers&, const double* in, const double* u0, double* out, double* u0copy, int stage,
                double time_factor, int fuse_cfl, cudaStream_t) = nullptr;
  size_t (*fused_smem)(int nh_max) = nullptr;
  void (*cfl)(const DeviceBuffers&, cudaStream_t) = nullptr;
  void (*project)(const DeviceBuffers&, double t, cudaStream_t) = nullptr;
  // over cells [e_begin, e_end); lp: field parameters (nullptr: the solver's law)
  void (*norms)(const DeviceBuffers&, double t, int quantity, int rule, int e_begin, int e_end, const LawParams* lp,
                cudaStream_t);
  void (*l2err)(const DeviceBuffers&, double t, int field, int e_begin, int e_end, const LawParams* lp,
                cudaStream_t) = nullptr;
  void (*totals)(const DeviceBuffers&, double refm, int e_begin, int e_end, cudaStream_t) = nullptr;
  int (*grid_elem)(int E) = nullptr;
  // moment limiter pass (triangles, p >= 1; nullptr elsewhere)
  void (*limit)(const DeviceBuffers&, int check_done, cudaStream_t) = nullptr;
  // face-point traces of C (only: cells to refresh, nullptr for all)
  void (*trace)(const DeviceBuffers&, const unsigned char* only, cudaStream_t) = nullptr;
  // discrete adjoint stage (nullptr where the adjoint is not built)
  void (*adj_stage)(const DeviceBuffers&, const AdjStage&, cudaStream_t) = nullptr;
  // local time stepping (FP64, 128-thread tiles; nullptr elsewhere), over
  // segments of `lists` (LtsSegs): volume term of the cells into racc; face
  // kernel over face lists (boundary time t + fac * dt); lift of the face
  // classes in mask into racc over one cell list; coefficient operations
  // (LtsUpdateOp) with dt = ctl->dt * fac
  void (*lts_vol)(const DeviceBuffers&, const int* lists, const LtsSegs&, double* racc, cudaStream_t) = nullptr;
  void (*lts_face)(const DeviceBuffers&, const int* lists, const LtsSegs&, cudaStream_t) = nullptr;
  void (*lts_lift)(const DeviceBuffers&, const int* cells, int n, const int* cface, const int* fcls, unsigned mask,
                   double* racc, cudaStream_t) = nullptr;
  void (*lts_update)(const DeviceBuffers&, const int* lists, const LtsSegs&, double* c1, double* save,
                     double* racc, cudaStream_t) = nullptr;
  int lts_cpb = 0;  // cells per CTA of the cell kernels (LtsTile::CPB)
  int lts_fpb = 0;  // faces per CTA of the face kernel
};

// law, flux, dim, order, precision, block (tile variant: 64, 128 or 256 threads)
// (law, flux, dim, order, precision, block, quadrature rule)
using OpsKey = std::tuple<int, int, int, int, int, int, int>;
constexpr int kDefaultBlock = 128;
std::map<OpsKey, Ops>& ops_registry();
void register_scalar_ops();
void register_burgers_ops();
void register_euler2d_godunov_ops();
void register_euler2d_roe_ops();
void register_euler2d_llf_ops();
void register_euler3d_ops();
void register_maxwell3d_ops();
void register_maxwell2d_ops();
void register_burgers_tile_ops();
void register_euler2d_roe_tile_ops();

template <class K>
Ops make_ops();

}  // namespace dgp
