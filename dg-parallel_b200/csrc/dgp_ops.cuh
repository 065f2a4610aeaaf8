// Launchers of one kernel instantiation (included by the per-law
// instantiation units).
#pragma once

#include "dgp_adjoint.cuh"
#include "dgp_elem.cuh"
#include "dgp_limiter.cuh"
#include "dgp_lts.cuh"
#include "dgp_solver.h"
#include "dgp_stage.cuh"

namespace dgp {

// the discrete adjoint covers every law and flux (the exact Riemann solver is
// differentiated through its Newton iteration:
// dual numbers carry the derivative of every iterate, which converges with
// the iterate to the derivative of the solution)
template <class K>
constexpr bool adjoint_built() {
  return true;
}

constexpr size_t kSmemPerCta = 227 * 1024;

template <class K, bool ENS>
cudaError_t fused_prepare();

template <class K>
cudaError_t ops_prepare() {
  if (cudaError_t e = fused_prepare<K, false>()) return e;
  if (cudaError_t e = fused_prepare<K, true>()) return e;
  const size_t smem = elem_kernel_smem<K>();
  if (smem > 48 * 1024) {
    cudaError_t e = cudaFuncSetAttribute(elem_kernel<K>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         static_cast<int>(smem));
    if (e != cudaSuccess) return e;
  }

  if constexpr (adjoint_built<K>()) {
    const size_t as = adj_elem_smem<K>();
    if (as > 48 * 1024)
      return cudaFuncSetAttribute(adj_elem_kernel<K>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  static_cast<int>(as));
  }
  return cudaSuccess;
}

// dynamic shared memory of the fused stage kernel may use whatever the static
// part leaves of the 227 KB a CTA can hold
template <class K, bool ENS, bool TC>
cudaError_t fused_prepare_one() {
  cudaFuncAttributes fa;
  cudaError_t e = cudaFuncGetAttributes(&fa, stage_kernel<K, ENS, TC>);
  if (e != cudaSuccess) return e;
  return cudaFuncSetAttribute(stage_kernel<K, ENS, TC>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                              static_cast<int>(kSmemPerCta - fa.sharedSizeBytes));
}

template <class K, bool ENS>
cudaError_t fused_prepare() {
  if constexpr (FusedSmem<K>::UMMA_OK)
    if (cudaError_t e = fused_prepare_one<K, ENS, true>()) return e;
  if constexpr (probe_built<K>() && !ENS) {
    cudaFuncAttributes fa;
    cudaError_t e = cudaFuncGetAttributes(&fa, stage_kernel<K, false, false, true>);
    if (e != cudaSuccess) return e;
    e = cudaFuncSetAttribute(stage_kernel<K, false, false, true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             static_cast<int>(kSmemPerCta - fa.sharedSizeBytes));
    if (e != cudaSuccess) return e;
  }
  return fused_prepare_one<K, ENS, false>();
}

template <class K>
int ops_grid_elem(int E) {
  return (E + K::TE - 1) / K::TE;
}

template <class K>
StageArgs<typename K::T> stage_args(const DeviceBuffers& b, int stage, double time_factor, int fuse_cfl) {
  using T = typename K::T;
  StageArgs<T> a = make_args<T>(b);
  a.stage = stage;
  a.stage_time_factor = time_factor;
  a.fuse_cfl = fuse_cfl;
  a.p0 = b.p0;
  if (stage == 0) a.Cout = static_cast<double*>(b.rhs);
  return a;
}

template <class K>
void ops_face(const DeviceBuffers& b, int stage, double time_factor, cudaStream_t st) {
  auto a = stage_args<K>(b, stage, time_factor, 0);
  const int fgrid = (b.F + K::FPB - 1) / K::FPB;
  if (b.cell_inst)
    face_kernel<K, true><<<fgrid, K::FACE_BLOCK, 0, st>>>(a);
  else
    face_kernel<K, false><<<fgrid, K::FACE_BLOCK, 0, st>>>(a);
}

// second face pass of the P0 fallback (a no-op unless a cell was marked)
template <class K>
void ops_face_rerun(const DeviceBuffers& b, int stage, double time_factor, cudaStream_t st) {
  auto a = stage_args<K>(b, stage, time_factor, 0);
  const int fgrid = (b.F + K::FPB - 1) / K::FPB;
  const int g = fgrid < 296 ? fgrid : 296;
  if (b.cell_inst)
    face_rerun_kernel<K, true><<<g, K::FACE_BLOCK, 0, st>>>(a);
  else
    face_rerun_kernel<K, false><<<g, K::FACE_BLOCK, 0, st>>>(a);
}

// volume-point check of the P0 fallback (marks only)
template <class K>
void ops_p0_volume(const DeviceBuffers& b, int stage, cudaStream_t st) {
  auto a = stage_args<K>(b, stage, 0.0, 0);
  const long long n = (long long)b.E * K::NQ;
  const int g = (int)((n + 127) / 128);
  if (b.cell_inst)
    p0_volume_kernel<K, true><<<g, 128, 0, st>>>(a);
  else
    p0_volume_kernel<K, false><<<g, 128, 0, st>>>(a);
}

template <class K>
void ops_elem(const DeviceBuffers& b, int stage, int fuse_cfl, cudaStream_t st) {
  auto a = stage_args<K>(b, stage, 0.0, fuse_cfl);
  elem_kernel<K><<<ops_grid_elem<K>(b.E), K::BLOCK, elem_kernel_smem<K>(), st>>>(a);
}

template <class K>
void ops_stage(const DeviceBuffers& b, int stage, double time_factor, int fuse_cfl, cudaStream_t st) {
  if (b.p0) ops_p0_volume<K>(b, stage, st);
  ops_face<K>(b, stage, time_factor, st);
  if (b.p0) ops_face_rerun<K>(b, stage, time_factor, st);
  ops_elem<K>(b, stage, fuse_cfl, st);
}

template <class K>
size_t ops_fused_smem(int nh_max) {
  const size_t a = FusedSmem<K, false>::bytes(nh_max), b = FusedSmem<K, true>::bytes(nh_max);
  return a > b ? a : b;
}

template <class K>
void ops_fused(const DeviceBuffers& b, const double* in, const double* u0, double* out, double* u0copy, int stage,
               double time_factor, int fuse_cfl, cudaStream_t st) {
  auto a = stage_args<K>(b, stage, time_factor, fuse_cfl);
  a.C = in;
  a.U0 = u0;
  a.Cout = out;
  a.U0out = u0copy;
  a.tab.blob = static_cast<const typename K::T*>(b.fblob);
  const int grid = ops_grid_elem<K>(b.E);
  if constexpr (probe_built<K>()) {
    if (b.round_mask && !b.cell_inst) {
      stage_kernel<K, false, false, true><<<grid, K::BLOCK, FusedSmem<K, false>::bytes(b.tm.nh_max), st>>>(a);
      if (stage == 3) stage_finalize_kernel<K><<<1, kFinalizeThreads, 0, st>>>(a, grid);
      return;
    }
  }
  bool tc = false;
  if constexpr (FusedSmem<K>::UMMA_OK) tc = b.tensor_cores != 0;
  if (tc) {
    if constexpr (FusedSmem<K>::UMMA_OK) {
      const size_t smem = FusedSmem<K, true>::bytes(b.tm.nh_max);
      if (b.cell_inst)
        stage_kernel<K, true, true><<<grid, K::BLOCK, smem, st>>>(a);
      else
        stage_kernel<K, false, true><<<grid, K::BLOCK, smem, st>>>(a);
    }
  } else {
    const size_t smem = FusedSmem<K, false>::bytes(b.tm.nh_max);
    if (b.cell_inst)
      stage_kernel<K, true, false><<<grid, K::BLOCK, smem, st>>>(a);
    else
      stage_kernel<K, false, false><<<grid, K::BLOCK, smem, st>>>(a);
  }
  if (stage == 3) stage_finalize_kernel<K><<<1, kFinalizeThreads, 0, st>>>(a, ops_grid_elem<K>(b.E));
}

template <class K>
void ops_trace(const DeviceBuffers& b, const unsigned char* only, cudaStream_t st) {
  auto a = make_args<typename K::T>(b);
  trace_kernel<K><<<ops_grid_elem<K>(b.E), K::BLOCK, 0, st>>>(a, only);
}

// the solver's limiter on the current state.  Barth: one pass in place.
// Triangle moment limiter: moments of every row, then the limited rows (and
// their traces) in place.
template <class K>
void ops_limit(const DeviceBuffers& b, int check_done, cudaStream_t st) {
  if constexpr (K::ORDER >= 1) {
    if (b.limiter_kind == DGP_LIMITER_BARTH) {
      BarthArgs a;
      a.C = static_cast<double*>(b.C);
      a.trig = b.trig;
      a.cface = b.cface;
      a.fel = b.fel;
      a.fcode = b.fcode;
      a.phif = b.bphif;
      a.phi0 = b.phi0;
      a.tr = b.tr;
      a.phif_t = b.phif;
      a.ctl = check_done ? b.ctl : nullptr;
      a.gctl = b.gctl;
      a.cell_inst = b.cell_inst;
      a.E = b.E;
      a.slope = b.lim_slope;
      a.replay = b.lim_replay;
      barth_kernel<K><<<(b.E + 127) / 128, 128, 0, st>>>(a);
      return;
    }
  }
  if constexpr (K::DIM == 2 && K::ORDER >= 1) {
    LimArgs a;
    a.C = static_cast<double*>(b.C);
    a.Mo = b.lmo;
    a.big = b.lbig;
    a.trig = b.trig;
    a.nb = b.nb;
    a.geo = b.lgeo;
    a.Dn = b.limD;
    a.Dinv = b.limDinv;
    a.tr = b.tr;
    a.phif = b.phif;
    a.ctl = check_done ? b.ctl : nullptr;
    a.gctl = b.gctl;
    a.cell_inst = b.cell_inst;
    a.E = b.E;
    const long long rows = static_cast<long long>(b.E) * K::M;
    const int grid = static_cast<int>((rows + 127) / 128);
    limit_moments_kernel<K><<<grid, 128, 0, st>>>(a);
    limit_kernel<K><<<grid, 128, 0, st>>>(a);
  }
}

// one reversed stage of the discrete adjoint (face kernel, then element kernel)
template <class K>
void ops_adj_stage(const DeviceBuffers& b, const AdjStage& g, cudaStream_t st) {
  if constexpr (adjoint_built<K>()) {
    AdjArgs<typename K::T> a;
    a.s = make_args<typename K::T>(b);
    a.mu = g.mu;
    a.out = g.out;
    a.acc = g.acc;
    a.ca = g.ca;
    a.cb = g.cb;
    a.cc = g.cc;
    a.cd = g.cd;
    a.ce = g.ce;
    a.dt = g.dt;
    a.t_seg = g.t_seg;
    a.t_factor = g.t_factor;
    const int fgrid = (b.F + K::FPB - 1) / K::FPB;
    adj_face_kernel<K><<<fgrid, K::FACE_BLOCK, 0, st>>>(a);
    adj_elem_kernel<K><<<ops_grid_elem<K>(b.E), K::BLOCK, adj_elem_smem<K>(), st>>>(a);
  }
}

template <class K>
void ops_cfl(const DeviceBuffers& b, cudaStream_t st) {
  StageArgs<typename K::T> a = make_args<typename K::T>(b);
  // ensembles: one block per instance-pure tile
  const int grid = b.cell_inst ? ops_grid_elem<K>(b.E) : (b.E + 255) / 256;
  cfl_kernel<K><<<grid, 256, 0, st>>>(a);
}

template <class K>
void ops_project(const DeviceBuffers& b, double t, cudaStream_t st) {
  using T = typename K::T;
  StageArgs<T> a = make_args<T>(b);
  const long long n = static_cast<long long>(b.E) * K::NP;
  project_kernel<K><<<static_cast<int>((n + 127) / 128), 128, 0, st>>>(a, t, static_cast<double*>(b.C));
}

template <class K>
void ops_norms(const DeviceBuffers& b, double t, int quantity, int rule, int e_begin, int e_end,
               const LawParams* lp, cudaStream_t st) {
  auto a = make_args<typename K::T>(b);
  norms_kernel<K><<<(e_end - e_begin + 255) / 256, 256, 0, st>>>(a, t, quantity, rule, b.partials, e_begin, e_end,
                                                                 lp);
}

template <class K>
void ops_l2err(const DeviceBuffers& b, double t, int field, int e_begin, int e_end, const LawParams* lp,
               cudaStream_t st) {
  StageArgs<typename K::T> a = make_args<typename K::T>(b);
  l2err_kernel<K><<<(e_end - e_begin + 255) / 256, 256, 0, st>>>(a, t, field, b.partials, e_begin, e_end, lp);
}

template <class K>
void ops_totals(const DeviceBuffers& b, double refm, int e_begin, int e_end, cudaStream_t st) {
  StageArgs<typename K::T> a = make_args<typename K::T>(b);
  totals_kernel<K><<<(e_end - e_begin + 255) / 256, 256, 0, st>>>(a, refm, b.partials, e_begin, e_end);
}

// local time stepping launches over segment tables; S.block0 is filled here
// from the segments' lengths and the kernels' cells (faces) per CTA
inline int lts_fill_blocks(LtsSegs& S, int per_cta) {
  int nb = 0;
  for (int i = 0; i < S.nseg; ++i) {
    S.block0[i] = nb;
    nb += (S.cnt[i] + per_cta - 1) / per_cta;
  }
  S.block0[S.nseg] = nb;
  return nb;
}

template <class K>
void ops_lts_vol(const DeviceBuffers& b, const int* lists, const LtsSegs& segs, double* racc, cudaStream_t st) {
  const StageArgs<double> a = make_args<double>(b);
  LtsSegs S = segs;
  const int grid = lts_fill_blocks(S, LtsTile<K>::CPB);
  lts_vol_kernel<K><<<grid, 128, 0, st>>>(a, lists, S, racc);
}

template <class K>
void ops_lts_face(const DeviceBuffers& b, const int* lists, const LtsSegs& segs, cudaStream_t st) {
  const StageArgs<double> a = make_args<double>(b);
  LtsSegs S = segs;
  const int grid = lts_fill_blocks(S, K::FPB);
  lts_face_kernel<K><<<grid, K::FACE_BLOCK, 0, st>>>(a, lists, S);
}

template <class K>
void ops_lts_lift(const DeviceBuffers& b, const int* cells, int n, const int* cface, const int* fcls, unsigned mask,
                  double* racc, cudaStream_t st) {
  const StageArgs<double> a = make_args<double>(b);
  lts_lift_kernel<K><<<LtsTile<K>::grid(n), 128, 0, st>>>(a, cells, n, cface, fcls, mask, racc);
}

template <class K>
void ops_lts_update(const DeviceBuffers& b, const int* lists, const LtsSegs& segs, double* c1, double* save,
                    double* racc, cudaStream_t st) {
  const StageArgs<double> a = make_args<double>(b);
  LtsSegs S = segs;
  const int grid = lts_fill_blocks(S, LtsTile<K>::CPB);
  lts_update_kernel<K><<<grid, 128, 0, st>>>(a, lists, S, c1, save, racc);
}

template <class K>
Ops make_ops() {
  Ops o;
  o.M = K::M;
  o.NP = K::NP;
  o.NQ = K::NQ;
  o.NQF = K::NQF;
  o.TE = K::TE;
  o.elem_block = K::BLOCK;
  o.fpb = K::FPB;
  o.elem_smem = elem_kernel_smem<K>();
  o.tsize = sizeof(typename K::T);
  o.blob_elems = ElemSmem<K>::blob_elems;
  o.fill_blob = &fill_table_blob<K>;
  o.fill_fused_blob = &fill_fused_blob<K>;
  o.fused_blob_elems = FusedSmem<K>::fblob_elems;
  o.tensor_cores_ok = FusedSmem<K>::UMMA_OK;
  o.probe_ok = probe_built<K>();
  o.precision = sizeof(typename K::T) == 8 ? DGP_PRECISION_FP64 : DGP_PRECISION_MIXED;
  o.prepare = &ops_prepare<K>;
  o.stage = &ops_stage<K>;
  o.face = &ops_face<K>;
  o.elem = &ops_elem<K>;
  o.fused = &ops_fused<K>;
  o.fused_smem = &ops_fused_smem<K>;
  o.cfl = &ops_cfl<K>;
  o.project = &ops_project<K>;
  o.l2err = &ops_l2err<K>;
  o.norms = &ops_norms<K>;
  o.totals = &ops_totals<K>;
  o.grid_elem = &ops_grid_elem<K>;
  o.limit = K::ORDER >= 1 ? &ops_limit<K> : nullptr;
  // the adjoint and local time stepping are built for the reference rule
  if constexpr (K::RULE == 0) o.adj_stage = adjoint_built<K>() ? &ops_adj_stage<K> : nullptr;
  o.trace = &ops_trace<K>;
  if constexpr (sizeof(typename K::T) == 8 && K::BLOCK == kDefaultBlock && K::RULE == 0) {
    o.lts_vol = &ops_lts_vol<K>;
    o.lts_face = &ops_lts_face<K>;
    o.lts_lift = &ops_lts_lift<K>;
    o.lts_update = &ops_lts_update<K>;
    o.lts_cpb = LtsTile<K>::CPB;
    o.lts_fpb = K::FPB;
  }
  return o;
}

template <int LAW, int FLUX, int DIM, int ORDER, int BLOCK = kDefaultBlock, int RULE = 0>
void add_ops() {
  ops_registry()[OpsKey(LAW, FLUX, DIM, ORDER, DGP_PRECISION_FP64, BLOCK, RULE)] =
      make_ops<Cfg<LAW, FLUX, DIM, ORDER, double, BLOCK, RULE>>();
  ops_registry()[OpsKey(LAW, FLUX, DIM, ORDER, DGP_PRECISION_MIXED, BLOCK, RULE)] =
      make_ops<Cfg<LAW, FLUX, DIM, ORDER, float, BLOCK, RULE>>();
}

// the other tile shapes the autotuner chooses among
template <int LAW, int FLUX, int DIM, int ORDER>
void add_tile_ops() {
  add_ops<LAW, FLUX, DIM, ORDER, 64>();
  add_ops<LAW, FLUX, DIM, ORDER, 256>();
}

}  // namespace dgp
