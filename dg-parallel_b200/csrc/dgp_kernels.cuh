// CUDA kernels of one explicit DG stage on sm_100a.
//
//   face_kernel  one thread per (face, face point): gathers the left and right
//                traces from [cell][field][mode] coefficients, evaluates the
//                law's numerical (or boundary) flux and writes -F|J|w into the
//                left cell's face slot and +F|J|w into the right cell's slot
//                (per-cell slots [cell][local face][point][field]; no atomics).
//                Replaces DGBoundaryCell::computeBoundaryContributions
//                (DGCell.cc:639-732).
//   elem_kernel  one CTA per tile of TE cells staged in shared memory: volume
//                term (DGCell::computeVolumeContribution, DGCell.cc:184-249) as
//                interpolate -> flux -> contraction with the reference gradient
//                table, plus the lift of the face slots, the diagonal inverse
//                mass 1/|J| and the SSP-RK3 stage combination
//                (RungeKuttaTVD3::advanceInTime, TimeIntegrator.cc:838-990).  The
//                last stage also reduces the CFL time step of the next step
//                (DGCell::adaptTimeStep, DGCell.cc:1155-1207) and the residual.
//   cfl_kernel   the same CFL reduction for the first step.
#pragma once

#include <cstdint>

#include "dgp_laws.cuh"

namespace dgp {

// ---- compile-time shape of one (law, flux, dim, order, precision) ----------
// Quadrature points.  Rule 0: DG-Parallel's rules (volume degree 2p, tet faces
// 2p+1, edges p+1 Gauss points).  Rule 1 (DGP_RULE_WORKLOAD): the point counts
// the workloads state at P2 -- triangles the 7-point volume rule of degree 5,
// tets the 11-point volume rule and the 6-point face rule of degree 4; every
// other order as rule 0.
constexpr int tri_vol_points(int p, int rule = 0) {
  return rule == 1 && p == 2 ? 7 : p == 0 ? 1 : p == 1 ? 3 : p == 2 ? 6 : p == 3 ? 12 : 16;
}
constexpr int tet_vol_points(int p, int rule = 0) {
  return rule == 1 && p == 2 ? 11 : p == 0 ? 1 : p == 1 ? 4 : p == 2 ? 14 : 24;
}
constexpr int tet_face_points(int p, int rule = 0) {
  return rule == 1 && p == 2 ? 6 : p == 0 ? 1 : p == 1 ? 4 : p == 2 ? 7 : 13;
}

// BLOCK_: threads of the element and face kernels; it sets the cells per
// element-kernel tile (TE) and the faces per face-kernel CTA, the shapes the
// autotuner chooses among (64, 128, 256).
// RULE_: the quadrature rule option (see tri_vol_points).
template <int LAW_, int FLUX_, int DIM_, int ORDER_, typename T_, int BLOCK_ = 128, int RULE_ = 0>
struct Cfg {
  using T = T_;
  static constexpr int LAW = LAW_, FLUX = FLUX_, DIM = DIM_, ORDER = ORDER_, RULE = RULE_;
  static constexpr int M = LawTraits<LAW>::M;
  static constexpr int NP = DIM == 2 ? (ORDER + 1) * (ORDER + 2) / 2
                                     : (ORDER + 1) * (ORDER + 2) * (ORDER + 3) / 6;
  static constexpr int NQ = DIM == 2 ? tri_vol_points(ORDER, RULE) : tet_vol_points(ORDER, RULE);
  static constexpr int NQF = DIM == 2 ? ORDER + 1 : tet_face_points(ORDER, RULE);
  static constexpr int NLF = DIM + 1;
  static constexpr int NPERM = DIM == 2 ? 2 : 6;
  static constexpr int MNP = M * NP;
  static constexpr int NS = NLF * NQF;   // face points of a cell (lift length)
  static constexpr int KV = NQ * DIM;    // volume contraction length
  // element kernel: one thread per (cell, field) row of the tile, all modes of
  // the row in registers; TE cells per CTA, capped by a shared-memory budget
  static constexpr int BLOCK = BLOCK_;
  static constexpr int NV = DIM == 2 ? 4 : 1;  // states of the CFL (mean + vertices)
  static constexpr int LDK = KV | 1;           // row stride of G (odd: conflict-free)
  // shared memory per cell of a tile: FP64 state and u_n, G rows, face slots,
  // geometry, CFL eigenvalues
  static constexpr int CELL_BYTES = 16 * MNP + (int)sizeof(T) * (M * LDK + NS * M) + 8 * (NV + DIM * DIM + 1);
  // shared-memory budget of a tile: 768 bytes per thread, at most 64 KB so
  // that three tiles (with the table blob) share an SM whatever the order
  static constexpr int SMEM_BUDGET = BLOCK * 768 < 64 * 1024 ? BLOCK * 768 : 64 * 1024;
  static constexpr int TE_SMEM = SMEM_BUDGET / CELL_BYTES;
  static constexpr int TE_ROWS = BLOCK / M;
  static constexpr int TE = TE_SMEM < TE_ROWS ? (TE_SMEM < 1 ? 1 : TE_SMEM) : TE_ROWS;
  static constexpr int ROWS = TE * M;
  static constexpr int EG = BLOCK / NQ;   // cells processed concurrently in the volume phase
  // face slots live tile-transposed, [tile][face point][row], so that the
  // element kernel reads them row-coalesced: slot(e, s, j) =
  // ((e / TE) * NS + s) * ROWS + (e % TE) * M + j
  // the face kernel's CTA does not depend on the tile shape (the slots are
  // addressed per cell): 128 threads keep its register budget at the size
  // that measured fastest
  static constexpr int FACE_BLOCK = 128;
  static constexpr int FPB = FACE_BLOCK / NQF;  // faces per face-kernel CTA
  static constexpr int LDM = MNP | 1;           // staged coefficient row stride
};

template <class K>
__device__ __forceinline__ size_t slot_index(int e, int s, int j) {
  return ((size_t)(e / K::TE) * K::NS + s) * K::ROWS + (size_t)(e % K::TE) * K::M + j;
}

// time-step control that lives in device memory so that a whole run can be
// captured in a CUDA graph without host round trips
struct TimeCtl {
  double t;          // time at the start of the current step
  double dt;         // current step
  double tend;       // <= 0: no end time
  double cfl;
  double resid;      // sum (u_new - u_n)^2 of the last step
  int steps;         // steps completed
  int max_steps;     // <= 0: unbounded
  int done;          // set when tend or max_steps is reached
  int lts_shift;     // local time stepping: the step is the CFL minimum times 2^lts_shift
  unsigned long long dtmin_bits;  // atomicMin accumulator (positive double bits)
  unsigned int blocks_done;       // completion counter of the reducing kernel
  unsigned int pad2;
  unsigned long long t_mark_ns;   // device clock: run start (whole-launch entry) or
                                  // the moment the instance finished (ensembles)
};

struct Status {
  int nonphysical;
  int first_bad;  // internal cell index, INT_MAX when none
  int timeouts;   // bounded waits on bulk copies that gave up (never expected)
  int stage_bad;  // cells marked for the P0 fallback in the current stage
};

// device views (internal cell order); T = arithmetic type of the hot path
template <typename T>
struct DevMesh {
  int E, F, NB;
  const T* jinv;      // E x DIM*DIM, [i][r] = d xi_r / d x_i
  const T* detj;      // E, |det J| (arithmetic type)
  const double* detjd;// E, |det J| in FP64 (inverse mass of the stage update)
  const double* csize;// E, DGCell::computeCellSize
  const double* x0;   // E x 3 affine origin (FP64)
  const double* jac;  // E x 9 rows d x / d xi_r (FP64)
  const int* fel;     // F x 2: eL, eR (eR < 0: boundary face -eR-1)
  const int* fcode;   // F: lfL | lfR << 4 | perm << 8
  const T* fnrm;      // F x DIM
  const T* fj;        // F: |J_f|
  const double* bpts; // NB x NQF x 3 physical points of boundary faces
  const int* bbid;    // NB classification ids
  const int* bpart;   // NB periodic partner cell (-1: none)
  const T* bpphi;     // NB x NQF x NP partner basis at the mirrored points
};

template <typename T>
struct DevTables {
  const T* blob;    // element-kernel tables in their shared-memory layout (bulk copied)
  int blob_bytes;
  const T* phi;     // NQ x NP
  const T* dphi;    // NQ x DIM x NP
  const T* qw;      // NQ
  const T* phif;    // NLF x NQF x NP
  const T* fqw;     // NQF
  const int* qmap;  // NPERM x NQF
  const double* phiv;  // (DIM+1) x NP  (FP64, CFL)
  const T* phimax;     // NP: largest |phi_k| over the volume and face points (P0 check)
  const double* phiq;  // NQ x NP (FP64, projection)
  const double* qwd;   // NQ (FP64)
  const double* qpd;   // NQ x 3 (FP64)
  int nqe;             // error rule
  const double* eqp;   // nqe x 3
  const double* eqw;   // nqe
  const double* ephi;  // nqe x NP
  double phi0;
};

// Per-tile face records and halo lists of the fused stage kernel.  Tile t
// owns cells [t TE, (t + 1) TE); its faces are every face with a side in the
// tile (a face between two tiles appears in both lists and is evaluated by
// both, identically); a local row index l < TE is the own cell e0 + l, l >= TE
// the halo cell th_cell[th_off[t] + l - TE].
struct TileMesh {
  const int* tf_off;     // [ntiles + 1] face records of each tile
  const int* tf_side;    // lL | (lR + 1) << 16 (interior) or (partner + 1) << 16 (periodic), 0 above
  const int* tf_code;    // lfL | lfR << 4 | perm << 8 | ownL << 12 | ownR << 13 | kind << 14
                         // (kind 0 interior, 1 boundary, 2 periodic)
  const int* tf_bnd;     // boundary face index of kinds 1 and 2
  const double* tf_nrm;  // [NTF][DIM] unit normal out of the left cell (FP64)
  const double* tf_fj;   // [NTF] |J_f| (FP64)
  const int* th_off;     // [ntiles + 1] halo cells of each tile
  const int* th_cell;    // internal cell index of each halo row
  int nh_max;            // largest halo of a tile
};

template <typename T>
struct StageArgs {
  DevMesh<T> mesh;
  DevTables<T> tab;
  TileMesh tm;
  int mbar_polls;  // bound of the first bulk-copy wait of the fused stage kernel (0: default)
  int round_mask;  // rounding probe of the fused stage kernel (0: off)
  LawParams law;
  // the state is FP64 in both forms; T is the arithmetic of the RHS
  const double* C;   // state the stage reads
  const double* U0;  // u_n (stages 2 and 3)
  double* Cout;      // state the stage writes (or the RHS when stage == 0)
  double* U0out;     // stage 1 copies u_n here
  T* slots;        // E x NLF x NQF x M
  T* tr;           // face-point traces of the state C, slot layout (kept current by the
                   // element kernel and by trace_kernel after any other change of C)
  TimeCtl* ctl;
  Status* status;
  double* partials;  // per-block residual partials (stage 3)
  double stage_time_factor;  // 0, 1, 0.5: boundary time = t + factor * dt
  unsigned char* bad;  // [E] P0-fallback marks (DGCell::setToZero)
  // ensembles: a batch of independent instances in one cell/face index space,
  // each instance's cells contiguous from a tile boundary, with its own time
  // control ctl[i]; gctl carries the launch-wide counters and the all-done
  // flag.  A single solver has cell_inst == nullptr and gctl == ctl.
  TimeCtl* gctl;
  const int* cell_inst;    // [E] instance of each cell (-1: padding)
  const int* inst_end;     // [ninst] one past the last cell of each instance
  const int* tile_first;   // [ninst + 1] first element-kernel tile of each instance
  const LawParams* laws;   // [ninst] field parameters of each instance
  int ninst;
  int stage;       // 0: RHS only, 1..3: SSP-RK3 stages
  int fuse_cfl;    // stage 3 reduces the next step's dt
  int order;
  int p0;          // 1: P0 fallback on (face kernel marks, element kernel consumes marks)
};

__device__ __forceinline__ void flag_nonphysical(Status* st, int cell) {
  atomicAdd(&st->nonphysical, 1);
  atomicMin(&st->first_bad, cell);
}

template <typename T>
__device__ __forceinline__ void mark_p0(const StageArgs<T>& a, int cell) {
  if (!a.bad[cell]) {
    a.bad[cell] = 1;
    atomicAdd(&a.status->stage_bad, 1);
  }
}

// -----------------------------------------------------------------------------
// largest power of two (<= 16) dividing n
constexpr int pow2_div(int n) { return (n % 16 == 0) ? 16 : (n % 8 == 0) ? 8 : (n % 4 == 0) ? 4 : 1; }

// N values through the read-only path with loads of ALIGN bytes (p is
// ALIGN-aligned)
// N values to memory with stores of ALIGN bytes (p is ALIGN-aligned)
template <typename T, int N, int ALIGN>
__device__ __forceinline__ void st_vec(T* p, const T (&v)[N]) {
  if constexpr (ALIGN == 16 && sizeof(T) == 8 && N % 2 == 0) {
#pragma unroll
    for (int i = 0; i < N / 2; ++i) reinterpret_cast<double2*>(p)[i] = make_double2(v[2 * i], v[2 * i + 1]);
  } else if constexpr (ALIGN == 16 && sizeof(T) == 4 && N % 4 == 0) {
#pragma unroll
    for (int i = 0; i < N / 4; ++i)
      reinterpret_cast<float4*>(p)[i] = make_float4(v[4 * i], v[4 * i + 1], v[4 * i + 2], v[4 * i + 3]);
  } else if constexpr (ALIGN >= 8 && sizeof(T) == 4 && N % 2 == 0) {
#pragma unroll
    for (int i = 0; i < N / 2; ++i) reinterpret_cast<float2*>(p)[i] = make_float2(v[2 * i], v[2 * i + 1]);
  } else {
#pragma unroll
    for (int i = 0; i < N; ++i) p[i] = v[i];
  }
}

template <typename T, int N, int ALIGN>
__device__ __forceinline__ void ldg_vec(const T* __restrict__ p, T (&out)[N]) {
  if constexpr (ALIGN == 16 && sizeof(T) == 8 && N % 2 == 0) {
#pragma unroll
    for (int i = 0; i < N / 2; ++i) {
      const double2 v = __ldg(reinterpret_cast<const double2*>(p) + i);
      out[2 * i] = v.x;
      out[2 * i + 1] = v.y;
    }
  } else if constexpr (ALIGN == 16 && sizeof(T) == 4 && N % 4 == 0) {
#pragma unroll
    for (int i = 0; i < N / 4; ++i) {
      const float4 v = __ldg(reinterpret_cast<const float4*>(p) + i);
      out[4 * i] = v.x;
      out[4 * i + 1] = v.y;
      out[4 * i + 2] = v.z;
      out[4 * i + 3] = v.w;
    }
  } else if constexpr (ALIGN >= 8 && sizeof(T) == 4 && N % 2 == 0) {
#pragma unroll
    for (int i = 0; i < N / 2; ++i) {
      const float2 v = __ldg(reinterpret_cast<const float2*>(p) + i);
      out[2 * i] = v.x;
      out[2 * i + 1] = v.y;
    }
  } else {
#pragma unroll
    for (int i = 0; i < N; ++i) out[i] = __ldg(p + i);
  }
}

// trace of a cell's state at one face point: U[j] = sum_k phi[k] C[j][k],
// streamed field by field (FP64 state converted to the arithmetic type)
template <class K>
__device__ __forceinline__ void cell_trace(const double* __restrict__ c, const typename K::T* phi,
                                           typename K::T* U, bool p0 = false) {
  using T = typename K::T;
  constexpr int NP = K::NP;
  constexpr int ALIGN = pow2_div(NP * 8) < pow2_div(K::MNP * 8) ? pow2_div(NP * 8) : pow2_div(K::MNP * 8);
  if (p0) {  // cell dropped to P0: its trace is the mean
#pragma unroll
    for (int j = 0; j < K::M; ++j) U[j] = phi[0] * (T)__ldg(c + j * NP);
    return;
  }
#pragma unroll
  for (int j = 0; j < K::M; ++j) {
    double cj[NP];
    ldg_vec<double, NP, ALIGN>(c + j * NP, cj);
    T acc = 0;
#pragma unroll
    for (int k = 0; k < NP; ++k) acc += phi[k] * (T)cj[k];
    U[j] = acc;
  }
}

// the M field values of a cell's trace at face point s (slot layout, M
// contiguous values)
template <class K>
__device__ __forceinline__ void load_trace(const typename K::T* __restrict__ tr, int e, int s,
                                           typename K::T* U) {
  using T = typename K::T;
  constexpr int B = (int)(K::M * sizeof(T));
  constexpr int ALIGN = pow2_div(B) < 16 ? pow2_div(B) : 16;
  T v[K::M];
  ldg_vec<T, K::M, ALIGN>(tr + slot_index<K>(e, s, 0), v);
#pragma unroll
  for (int j = 0; j < K::M; ++j) U[j] = v[j];
}

// Face-point traces of the state, for every cell (only == nullptr) or the
// cells with only[e] != 0: one CTA per tile, one thread per (cell, field)
// row, in the order the element kernel uses for its fresh state.
template <class K>
__global__ void __launch_bounds__(K::BLOCK) trace_kernel(const __grid_constant__ StageArgs<typename K::T> a,
                                                          const unsigned char* only) {
  using T = typename K::T;
  constexpr int M = K::M, NP = K::NP, NS = K::NS, ROWS = K::ROWS;
  const int e0 = blockIdx.x * K::TE, row = threadIdx.x;
  const int e = e0 + row / M;
  if (row >= ROWS || e >= a.mesh.E) return;
  if (only && !only[e]) return;
  T c[NP];
#pragma unroll
  for (int k = 0; k < NP; ++k) c[k] = (T)a.C[((size_t)e0 * M + row) * NP + k];
  T* out = a.tr + (size_t)blockIdx.x * NS * ROWS + row;
  for (int s = 0; s < NS; ++s) {
    T acc = 0;
#pragma unroll
    for (int k = 0; k < NP; ++k) acc += __ldg(a.tab.phif + s * NP + k) * c[k];
    out[(size_t)s * ROWS] = acc;
  }
}

// One face point once its traces are in registers: non-physical checks (P0
// marks), numerical, periodic or boundary flux, the two face slots.  UR holds
// the right cell's trace at its point qR for interior faces.  RERUN: second
// pass of the P0 fallback (no checks; a periodic partner marked bad gives its
// mean).
template <class K, bool RERUN, bool ENS>
__device__ __forceinline__ void face_finish(const StageArgs<typename K::T>& a, int f, int q, int eL, int eR,
                                            int inst, int lfL, int lfR, int qR, const typename K::T (&n)[K::DIM],
                                            typename K::T jw, const typename K::T (&UL)[K::M],
                                            const typename K::T (&UR)[K::M], double tfac = -1.0) {
  using T = typename K::T;
  constexpr int M = K::M, NP = K::NP, NQF = K::NQF, DIM = K::DIM, MNP = K::MNP;
  T flux[M];
  if (!RERUN && !is_physical<K::LAW, T>(a.law, UL)) {
    flag_nonphysical(a.status, eL);
    if (a.p0) mark_p0(a, eL);
  }
  if (eR >= 0) {
    if (!RERUN && !is_physical<K::LAW, T>(a.law, UR)) {
      flag_nonphysical(a.status, eR);
      if (a.p0) mark_p0(a, eR);
    }
    numerical_flux<K::LAW, K::FLUX, DIM, T>(a.law, n, UL, UR, flux);
  } else if (a.mesh.bpart[-eR - 1] >= 0) {
    // periodic edge (DGCell.cc:687-705): the partner cell's trace at the
    // mirrored point through the numerical flux; only the left cell gets it
    const int b = -eR - 1, pe = a.mesh.bpart[b];
    T UP[M];
    cell_trace<K>(a.C + (size_t)pe * MNP, a.mesh.bpphi + ((size_t)b * NQF + q) * NP, UP, RERUN && a.bad[pe]);
    numerical_flux<K::LAW, K::FLUX, DIM, T>(a.law, n, UL, UP, flux);
  } else {
    const int b = -eR - 1;
    const double* x = a.mesh.bpts + ((size_t)b * NQF + q) * 3;
    if constexpr (ENS) {  // the instance's own clock and far-field parameters
      const TimeCtl* c = a.ctl + inst;
      const double time = __fma_rn(a.stage_time_factor, c->dt, c->t);
      boundary_flux<K::LAW, K::FLUX, DIM, T>(a.laws[inst], a.mesh.bbid[b], n, x, time, UL, flux);
    } else {
      // tfac >= 0: the caller's time factor (local time stepping's 2^-k)
      const double time = __fma_rn(tfac < 0.0 ? a.stage_time_factor : tfac, a.ctl->dt, a.ctl->t);
      boundary_flux<K::LAW, K::FLUX, DIM, T>(a.law, a.mesh.bbid[b], n, x, time, UL, flux);
    }
  }
  // the M values of a face point are contiguous in the slot layout: vector stores
  constexpr int B = (int)(M * sizeof(T));
  constexpr int ALIGN = pow2_div(B) < 16 ? pow2_div(B) : 16;
  T v[M];
#pragma unroll
  for (int j = 0; j < M; ++j) v[j] = -flux[j] * jw;
  st_vec<T, M, ALIGN>(a.slots + slot_index<K>(eL, lfL * NQF + q, 0), v);
  if (eR >= 0) {
#pragma unroll
    for (int j = 0; j < M; ++j) v[j] = flux[j] * jw;
    st_vec<T, M, ALIGN>(a.slots + slot_index<K>(eR, lfR * NQF + qR, 0), v);
  }
}

// One face point: traces of both sides (precomputed, or for RERUN evaluated
// from the coefficients with marked cells at their means), then face_finish.
template <class K, bool RERUN, bool ENS>
__device__ __forceinline__ void face_point(const StageArgs<typename K::T>& a, int f, int q,
                                           const typename K::T* s_phif, const typename K::T* s_fqw,
                                           const int* s_qmap, double tfac = -1.0) {
  using T = typename K::T;
  constexpr int M = K::M, NP = K::NP, NQF = K::NQF, DIM = K::DIM, MNP = K::MNP;
  const int eL = a.mesh.fel[2 * f], eR = a.mesh.fel[2 * f + 1];
  int inst = 0;
  if constexpr (ENS) {
    inst = a.cell_inst[eL];
    if (a.ctl[inst].done) return;
  }
  const int code = a.mesh.fcode[f];
  const int lfL = code & 15, lfR = (code >> 4) & 15, perm = code >> 8;
  T n[DIM];
#pragma unroll
  for (int i = 0; i < DIM; ++i) n[i] = a.mesh.fnrm[f * DIM + i];
  const T jw = a.mesh.fj[f] * s_fqw[q];
  T UL[M], UR[M];
  if constexpr (RERUN)
    cell_trace<K>(a.C + (size_t)eL * MNP, s_phif + (lfL * NQF + q) * NP, UL, a.bad[eL]);
  else
    load_trace<K>(a.tr, eL, lfL * NQF + q, UL);
  int qR = 0;
  if (eR >= 0) {
    qR = s_qmap[perm * NQF + q];
    if constexpr (RERUN)
      cell_trace<K>(a.C + (size_t)eR * MNP, s_phif + (lfR * NQF + qR) * NP, UR, a.bad[eR]);
    else
      load_trace<K>(a.tr, eR, lfR * NQF + qR, UR);
  }
  face_finish<K, RERUN, ENS>(a, f, q, eL, eR, inst, lfL, lfR, qR, n, jw, UL, UR, tfac);
}

template <class K>
__device__ __forceinline__ void face_tables(const StageArgs<typename K::T>& a, typename K::T* s_phif,
                                            typename K::T* s_fqw, int* s_qmap) {
  constexpr int NQF = K::NQF, NP = K::NP;
  const int tid = threadIdx.x;
  for (int i = tid; i < K::NLF * NQF * NP; i += blockDim.x) s_phif[i] = a.tab.phif[i];
  for (int i = tid; i < NQF; i += blockDim.x) s_fqw[i] = a.tab.fqw[i];
  for (int i = tid; i < K::NPERM * NQF; i += blockDim.x) s_qmap[i] = a.tab.qmap[i];
  __syncthreads();
}

// P0 fallback (DGAnalysis.cc:392-417, DGCell::setToZero DGCell.cc:785-811): with
// a.p0 set the face kernel marks every cell with a non-physical trace at a face
// point; face_rerun_kernel then recomputes every face with the marked cells'
// traces taken as their means and drops their modes k >= 1.
// ENS: ensemble batch (per-instance done flags, clocks and far fields)
template <class K, bool ENS>
__global__ void __launch_bounds__(K::FACE_BLOCK) face_kernel(const __grid_constant__ StageArgs<typename K::T> a) {
  using T = typename K::T;
  if (a.gctl->done) return;
  // the traces come precomputed: only the weights and orientation maps
  __shared__ T s_fqw[K::NQF];
  __shared__ int s_qmap[K::NPERM * K::NQF];
  const int tid = threadIdx.x;
  for (int i = tid; i < K::NQF; i += blockDim.x) s_fqw[i] = a.tab.fqw[i];
  for (int i = tid; i < K::NPERM * K::NQF; i += blockDim.x) s_qmap[i] = a.tab.qmap[i];
  __syncthreads();
  const int fl = tid / K::NQF, q = tid - (tid / K::NQF) * K::NQF;
  const int f = blockIdx.x * K::FPB + fl;
  if (fl >= K::FPB || f >= a.mesh.F) return;
  face_point<K, false, ENS>(a, f, q, nullptr, s_fqw, s_qmap);
}

// Second pass of the P0 fallback on a small grid: returns at once unless a
// cell was marked in this stage (the common case costs one tiny launch).  The
// faces read only the means of marked cells while the modes k >= 1 of those
// cells are zeroed, so both run in the same pass.
template <class K, bool ENS>
__global__ void __launch_bounds__(K::FACE_BLOCK) face_rerun_kernel(const __grid_constant__ StageArgs<typename K::T> a) {
  using T = typename K::T;
  if (a.gctl->done) return;
  if (*(volatile int*)&a.status->stage_bad == 0) return;
  __shared__ T s_phif[K::NLF * K::NQF * K::NP];
  __shared__ T s_fqw[K::NQF];
  __shared__ int s_qmap[K::NPERM * K::NQF];
  face_tables<K>(a, s_phif, s_fqw, s_qmap);
  const int tid = threadIdx.x;
  for (int e = blockIdx.x * blockDim.x + tid; e < a.mesh.E; e += gridDim.x * blockDim.x)
    if (a.bad[e])
      for (int r = 0; r < K::M; ++r)
        for (int k = 1; k < K::NP; ++k) const_cast<double*>(a.C)[((size_t)e * K::M + r) * K::NP + k] = 0.0;
  const int fl = tid / K::NQF, q = tid - (tid / K::NQF) * K::NQF;
  if (fl >= K::FPB) return;
  for (int vb = blockIdx.x; vb * K::FPB < a.mesh.F; vb += gridDim.x) {
    const int f = vb * K::FPB + fl;
    if (f < a.mesh.F) face_point<K, true, ENS>(a, f, q, s_phif, s_fqw, s_qmap);
  }
}

// First check of the P0 fallback, thread per (cell, volume quadrature point):
// a cell with a non-physical value at one of its volume points is marked (the
// correction inside DGCell::computeVolumeContribution, DGCell.cc:197-221);
// the face kernel marks the cells with a non-physical face-point trace, and
// face_rerun_kernel drops every marked cell to its mean.
template <class K, bool ENS>
__global__ void __launch_bounds__(128) p0_volume_kernel(const __grid_constant__ StageArgs<typename K::T> a) {
  using T = typename K::T;
  if (a.gctl->done) return;
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= (long long)a.mesh.E * K::NQ) return;
  const int e = (int)(i / K::NQ), q = (int)(i - (long long)e * K::NQ);
  const LawParams* lp = &a.law;
  if constexpr (ENS) {
    const int inst = a.cell_inst[e];
    if (inst < 0 || a.ctl[inst].done) return;
    lp = a.laws + inst;
  }
  T U[K::M];
  cell_trace<K>(a.C + (size_t)e * K::MNP, a.tab.phi + q * K::NP, U);
  if (!is_physical<K::LAW, T>(*lp, U)) {
    flag_nonphysical(a.status, e);
    mark_p0(a, e);
  }
}

// -----------------------------------------------------------------------------
// CFL time step of one cell: |cell| * cfl / (a (2p+1)), a = max eigenvalue at
// the mean and (triangles) at the three reference vertices; FP64 in both forms.
template <class K>
__device__ __forceinline__ double cell_dt(const StageArgs<typename K::T>& a, const double* c, int e,
                                          double cfl) {
  constexpr int M = K::M, NP = K::NP;
  double mean[M];
#pragma unroll
  for (int j = 0; j < M; ++j) mean[j] = c[j * NP] * a.tab.phi0;
  double am = max_eigen<K::LAW, double>(a.law, mean);
  if constexpr (K::DIM == 2) {
#pragma unroll
    for (int v = 0; v < 3; ++v) {
      double val[M];
#pragma unroll
      for (int j = 0; j < M; ++j) {
        double acc = 0;
#pragma unroll
        for (int k = 0; k < NP; ++k) acc += a.tab.phiv[v * NP + k] * c[j * NP + k];
        val[j] = acc;
      }
      double b = max_eigen<K::LAW, double>(a.law, val);
      am = (b > am ? b : am);
    }
  }
  return a.mesh.csize[e] * cfl / (am * (2. * K::ORDER + 1.0));
}

__device__ __forceinline__ double ctl_finalize(TimeCtl* c, double dtmin) {
  bool done = (c->max_steps > 0 && c->steps >= c->max_steps) || (c->tend > 0 && c->t >= c->tend);
  double dt = dtmin * (double)(1 << c->lts_shift);  // DGAnalysis.cc:590 (exact)
  if (c->tend > 0 && !done) {
    int N = (int)ceil((c->tend - c->t) / dt);
    dt = (c->tend - c->t) / N;
  }
  c->dt = dt;
  c->done = done ? 1 : 0;
  return dt;
}

// block-wide min of a double; thread 0 gets the result
template <int BLOCK>
__device__ __forceinline__ double block_min(double v, double* red) {
  for (int o = 16; o > 0; o >>= 1) v = fmin(v, __shfl_xor_sync(0xffffffffu, v, o));
  const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
  if (l == 0) red[w] = v;
  __syncthreads();
  if (w == 0) {
    v = (l < BLOCK / 32) ? red[l] : 1e300;
    for (int o = 16; o > 0; o >>= 1) v = fmin(v, __shfl_xor_sync(0xffffffffu, v, o));
  }
  __syncthreads();
  return v;
}

template <int BLOCK>
__device__ __forceinline__ double block_sum(double v, double* red) {
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
  if (l == 0) red[w] = v;
  __syncthreads();
  if (w == 0) {
    v = (l < BLOCK / 32) ? red[l] : 0.0;
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  }
  __syncthreads();
  return v;
}

// -----------------------------------------------------------------------------
// -----------------------------------------------------------------------------
__device__ __forceinline__ unsigned long long device_clock_ns() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

// Ensembles: the last CTA of a reducing kernel finalizes every instance that
// was running (time step from its dtmin accumulator, done flag, finish time)
// and sets the launch-wide done flag once all instances are done.
template <int BLOCK, typename T>
__device__ __forceinline__ void finalize_instances(const StageArgs<T>& a, bool advance, bool with_dt) {
  for (int i = threadIdx.x; i < a.ninst; i += BLOCK) {
    TimeCtl* c = a.ctl + i;
    if (c->done) continue;
    if (advance) {
      double r = 0.0;  // residual of the instance's tiles in a fixed order
      for (int b = a.tile_first[i]; b < a.tile_first[i + 1]; ++b) r += ((volatile double*)a.partials)[b];
      c->resid = r;
      c->t = c->t + c->dt;
      c->steps += 1;
    }
    if (with_dt) {
      const unsigned long long bits = atomicExch(&c->dtmin_bits, 0x7FF0000000000000ull);
      ctl_finalize(c, __longlong_as_double((long long)bits));
      if (c->done) c->t_mark_ns = device_clock_ns();
    }
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    int all = 1;
    for (int i = 0; i < a.ninst; ++i) all &= (*(volatile int*)&a.ctl[i].done) != 0;
    a.gctl->blocks_done = 0;
    a.gctl->done = all;
  }
}

// CFL reduction of the first step (and, with the limiter, after the last
// stage's limiter pass).  Ensembles reduce per instance over instance-pure
// tiles of TE cells, one tile per block.
template <class K>
__global__ void __launch_bounds__(256) cfl_kernel(const __grid_constant__ StageArgs<typename K::T> a) {
  __shared__ double red[256 / 32];
  __shared__ bool amLast;
  if (a.gctl->done) return;
  TimeCtl* c = a.ctl;
  int e = blockIdx.x * 256 + threadIdx.x, eend = a.mesh.E;
  bool active = true;
  if (a.cell_inst) {
    const int e0 = blockIdx.x * K::TE;
    const int inst = a.cell_inst[e0];
    c = a.ctl + inst;
    active = !c->done;
    e = threadIdx.x < K::TE ? e0 + threadIdx.x : a.mesh.E;
    eend = min(e0 + K::TE, a.inst_end[inst]);
  }
  double dtl = 1e300;
  if (active && e < eend) dtl = cell_dt<K>(a, a.C + (size_t)e * K::MNP, e, c->cfl);
  dtl = block_min<256>(dtl, red);
  if (threadIdx.x == 0) {
    if (active) atomicMin(&c->dtmin_bits, (unsigned long long)__double_as_longlong(dtl));
    __threadfence();
    unsigned v = atomicAdd(&a.gctl->blocks_done, 1u);
    amLast = (v == gridDim.x - 1);
  }
  __syncthreads();
  if (!amLast) return;
  __threadfence();
  if (a.cell_inst) {
    finalize_instances<256>(a, false, true);
  } else if (threadIdx.x == 0) {
    c->blocks_done = 0;
    unsigned long long bits = atomicExch(&c->dtmin_bits, 0x7FF0000000000000ull);
    ctl_finalize(c, __longlong_as_double((long long)bits));
  }
}

// -----------------------------------------------------------------------------
// L2 projection of the law's field (DGCell::L2ProjInitial, DGCell.cc:1458-1483):
// one thread per (cell, mode), FP64 accumulation in the reference's order.
template <class K>
__global__ void project_kernel(const __grid_constant__ StageArgs<typename K::T> a, double t, double* out) {
  using T = typename K::T;
  constexpr int M = K::M, NP = K::NP, NQ = K::NQ;
  const int gid = blockIdx.x * blockDim.x + threadIdx.x;
  const int e = gid / NP, k = gid - (gid / NP) * NP;
  if (e >= a.mesh.E) return;
  const int inst = a.cell_inst ? a.cell_inst[e] : 0;
  if (inst < 0) {  // ensemble padding
    for (int j = 0; j < M; ++j) out[(size_t)e * K::MNP + j * NP + k] = 0.0;
    return;
  }
  const LawParams& lp = a.laws ? a.laws[inst] : a.law;
  const double* x0 = a.mesh.x0 + 3 * (size_t)e;
  const double* J = a.mesh.jac + 9 * (size_t)e;
  double proj[M];
#pragma unroll
  for (int j = 0; j < M; ++j) proj[j] = 0.0;
  const double detj = a.mesh.detjd[e];
  for (int q = 0; q < NQ; ++q) {
    double x[3];
    const double* xi = a.tab.qpd + 3 * q;
    for (int c = 0; c < 3; ++c) {
      x[c] = x0[c];
      for (int r = 0; r < K::DIM; ++r) x[c] += xi[r] * J[r * 3 + c];
    }
    double val[M];
    field_eval<double>(lp, x, t, val);
    const double jw = detj * a.tab.qwd[q];
    for (int j = 0; j < M; ++j) proj[j] += val[j] * a.tab.phiq[q * NP + k] * jw;
  }
  const double inv = 1. / detj;
  for (int j = 0; j < M; ++j) out[(size_t)e * K::MNP + j * NP + k] = proj[j] * inv;
}

// per-block partial sums of (u_h - u_exact)^2 |J| w of one field over the
// error rule of degree 2(p+1) (DGCell::densityErrorL2, DGError.cc:805-826)
template <class K>
__global__ void __launch_bounds__(256) l2err_kernel(const __grid_constant__ StageArgs<typename K::T> a, double t,
                                                     int field, double* partials, int e_begin, int e_end,
                                                     const LawParams* lpp) {
  constexpr int M = K::M, NP = K::NP;
  __shared__ double red[256 / 32];
  const int e = e_begin + blockIdx.x * 256 + threadIdx.x;
  const LawParams& lp = lpp ? *lpp : a.law;
  double acc = 0.0;
  if (e < e_end) {
    const double* x0 = a.mesh.x0 + 3 * (size_t)e;
    const double* J = a.mesh.jac + 9 * (size_t)e;
    const auto* c = a.C + (size_t)e * K::MNP;
    const double detj = a.mesh.detjd[e];
    for (int q = 0; q < a.tab.nqe; ++q) {
      double x[3];
      const double* xi = a.tab.eqp + 3 * q;
      for (int cc = 0; cc < 3; ++cc) {
        x[cc] = x0[cc];
        for (int r = 0; r < K::DIM; ++r) x[cc] += xi[r] * J[r * 3 + cc];
      }
      double uh = 0.0;
      for (int k = 0; k < NP; ++k) uh += a.tab.ephi[q * NP + k] * (double)c[field * NP + k];
      double ex[M];
      field_eval<double>(lp, x, t, ex);
      const double d = uh - ex[field];
      acc += d * d * detj * a.tab.eqw[q];
    }
  }
  acc = block_sum<256>(acc, red);
  if (threadIdx.x == 0) partials[blockIdx.x] = acc;
}

// Error family of DGError.cc (DGCell::L1exact :549, LinfError :567,
// L1exactPressure :601, entropyErrorL1_2D/3D :621-665, pressureErrorL2 :774,
// densityErrorL2 :805, entropyErrorL2_2D :687): per-block partial L1 and
// squared-L2 sums and the maximum of |d| over the rule's points, where d is the
// difference to the exact field of a field (quantity >= 0), of the pressure
// (-1) or the entropy deviation (p / p_ex) / (rho / rho_ex)^gamma - 1 (-2),
// gamma = 1.4 as those functions fix it.  rule 0: the volume rule of degree
// 2p; rule 1: degree 2(p+1).  partials[3 * block + {0, 1, 2}].
template <int LAW, int DIM>
__device__ __forceinline__ double err_pressure(const double* v) {
  double m2 = v[1] * v[1] + v[2] * v[2];
  if constexpr (LAW == DGP_LAW_EULER3D) m2 += v[4] * v[4];
  return (1.4 - 1.) * (v[3] - 0.5 * m2 / v[0]);
}

template <class K>
__global__ void __launch_bounds__(256) norms_kernel(const __grid_constant__ StageArgs<typename K::T> a, double t,
                                                     int quantity, int rule, double* partials, int e_begin,
                                                     int e_end, const LawParams* lpp) {
  constexpr int M = K::M, NP = K::NP;
  __shared__ double red[256 / 32];
  const int e = e_begin + blockIdx.x * 256 + threadIdx.x;
  const LawParams& lp = lpp ? *lpp : a.law;
  double l1 = 0.0, l2 = 0.0, li = 0.0;
  if (e < e_end) {
    const double* x0 = a.mesh.x0 + 3 * (size_t)e;
    const double* J = a.mesh.jac + 9 * (size_t)e;
    const double* c = a.C + (size_t)e * K::MNP;
    const double detj = a.mesh.detjd[e];
    const int nq = rule ? a.tab.nqe : K::NQ;
    for (int q = 0; q < nq; ++q) {
      const double* xi = rule ? a.tab.eqp + 3 * q : a.tab.qpd + 3 * q;
      const double* ph = rule ? a.tab.ephi + q * NP : a.tab.phiq + q * NP;
      const double w = rule ? a.tab.eqw[q] : a.tab.qwd[q];
      double x[3];
      for (int cc = 0; cc < 3; ++cc) {
        x[cc] = x0[cc];
        for (int r = 0; r < K::DIM; ++r) x[cc] += xi[r] * J[r * 3 + cc];
      }
      double v[M], ex[M];
#pragma unroll
      for (int j = 0; j < M; ++j) {
        double acc = 0.0;
        for (int k = 0; k < NP; ++k) acc += ph[k] * c[j * NP + k];
        v[j] = acc;
      }
      field_eval<double>(lp, x, t, ex);
      double d = 0.0;
      if constexpr (K::LAW == DGP_LAW_EULER2D || K::LAW == DGP_LAW_EULER3D) {
        if (quantity == -2) {
          d = (err_pressure<K::LAW, K::DIM>(v) / err_pressure<K::LAW, K::DIM>(ex)) / pow(v[0] / ex[0], 1.4) - 1.;
        } else if (quantity == -1) {
          d = err_pressure<K::LAW, K::DIM>(v) - err_pressure<K::LAW, K::DIM>(ex);
        }
      }
      if (quantity >= 0) {
#pragma unroll
        for (int j = 0; j < M; ++j)
          if (j == quantity) d = v[j] - ex[j];
      }
      const double jw = detj * w;
      l1 += fabs(d) * jw;
      l2 += d * d * jw;
      li = fabs(d) > li ? fabs(d) : li;
    }
  }
  l1 = block_sum<256>(l1, red);
  l2 = block_sum<256>(l2, red);
  for (int o = 16; o > 0; o >>= 1) li = fmax(li, __shfl_xor_sync(0xffffffffu, li, o));
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = li;
  __syncthreads();
  if (threadIdx.x == 0) {
    double m = 0.0;
    for (int w = 0; w < 256 / 32; ++w) m = fmax(m, red[w]);
    partials[3 * (size_t)blockIdx.x] = l1;
    partials[3 * (size_t)blockIdx.x + 1] = l2;
    partials[3 * (size_t)blockIdx.x + 2] = m;
  }
}

// per-block partial cell integrals of every field: |J| * |ref| * phi0 * c[j][0]
template <class K>
__global__ void __launch_bounds__(256) totals_kernel(const __grid_constant__ StageArgs<typename K::T> a, double refm,
                                                      double* partials, int e_begin, int e_end) {
  __shared__ double red[256 / 32];
  const int e = e_begin + blockIdx.x * 256 + threadIdx.x;
  for (int j = 0; j < K::M; ++j) {
    double v = 0.0;
    if (e < e_end)
      v = a.mesh.detjd[e] * refm * a.tab.phi0 * a.C[(size_t)e * K::MNP + j * K::NP];
    v = block_sum<256>(v, red);
    if (threadIdx.x == 0) partials[(size_t)blockIdx.x * K::M + j] = v;
  }
}


}  // namespace dgp
