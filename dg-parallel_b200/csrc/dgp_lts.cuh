// Local time stepping: the kernels of RungeKuttaTVD2adaptive
// (TimeIntegrator.cc:442-836) on the size bins of DGAnalysis::sortCellsBySize
// (DGAnalysis.cc:749-890), FP64 only.
//
// The integrator works on groups of cells (inner cells of a bin, large and
// small cells on the interface between two bins) and classes of faces (the
// faces of a bin, the faces of an interface).  Each cell has a right-hand side
// that accumulates across assembly calls and is zeroed where the integrator
// calls ZeroRHS, a copy slot (DG_Dofs::copy / copyBack / swap) and the saved
// state of the step (the integrator's soln buffer).  Assembly calls become
//   lts_vol_kernel   volume term of the listed cells, added to the accumulator;
//   lts_face_kernel  the face kernel's face-point flux over a face list, into
//                    the face slots of both sides;
//   lts_lift_kernel  the slots of a set of face classes lifted into the
//                    accumulators of the cells that touch them (per cell, its
//                    local faces in order: no atomics);
// and every coefficient update is lts_update_kernel with one of the
// integrator's operations, which also refreshes the row's face-point traces.
// The cell kernels stage CPB listed cells per CTA in shared memory (LtsTile),
// so that their global loads and stores are element-parallel and coalesced.
// Every kernel returns at once when the run is done (ctl->done), so that a
// step captured in a CUDA graph turns into no-ops past the end.
#pragma once

#include "dgp_kernels.cuh"

namespace dgp {

// the integrator's coefficient operations (c: state, c1: copy slot, s: saved
// u_n, r: right-hand side, dt = DT * 2^-k, det = |det J|)
enum LtsUpdateOp : int {
  LTS_EULER_IN = 0,      // s = c; c += r / det * dt; r = 0        (TimeIntegrator.cc:486-490)
  LTS_TWO_HALF = 1,      // s = c; c += r dt / det; c1 = c; c += r dt / det; r = 0 (:508-518, :560-571)
  LTS_EULER = 2,         // s = c; c += r dt / det; r = 0          (:537-541)
  LTS_SECOND = 3,        // c = (c + r dt / det + s) / 2; r = 0    (:647-653, :697-704)
  LTS_SECOND_SWAP = 4,   // c1 = (c + r dt / det + s) / 2; c = old c1  (:670-678 + DG_Dofs::swap)
  LTS_COPYBACK_ZERO = 5, // r = 0; c = c1                          (:615-621)
  LTS_LI_HALF = 6,       // c = s + (c - s) + (c1 - 2c + s) / 4; s = c + (c1 - s) / 2  (:735-738)
  LTS_RESTORE = 7,       // c = s                                  (:759-760)
  LTS_FINAL_RESET = 8,   // c = c1; r = 0                          (:777)
};

// A launch covers several lists (segments): segment i is lists[off[i] ..
// off[i] + cnt[i]), with its own update operation and 2^-k factor, and owns
// CTAs block0[i] .. block0[i + 1] - 1.  Segments of one launch never share a
// cell (cell kernels) or a face (face kernel).
constexpr int kLtsMaxSegs = 32;
struct LtsSegs {
  int nseg;
  int off[kLtsMaxSegs];
  int cnt[kLtsMaxSegs];
  int op[kLtsMaxSegs];
  double fac[kLtsMaxSegs];
  int block0[kLtsMaxSegs + 1];
};

// the segment of CTA blk and the CTA's index inside it
__device__ __forceinline__ int lts_segment(const LtsSegs& S, int blk, int& local) {
  int i = 0;
  while (i + 1 < S.nseg && blk >= S.block0[i + 1]) ++i;
  local = blk - S.block0[i];
  return i;
}

// tile shape of the cell kernels: CPB listed cells per 128-thread CTA (one
// (cell, field) row per thread at most), their coefficients and the volume
// kernel's flux rows and tables in at most 40 KB of shared memory
template <class K>
struct LtsTile {
  static constexpr int M = K::M, MNP = K::MNP, KV = K::KV;
  static constexpr int KVP = KV | 1;  // row stride of the flux rows (odd: no bank conflicts)
  // the volume kernel's tables (phi, grad phi, weights) in shared memory when
  // they take at most 8 KB
  static constexpr int TAB = K::NQ * K::NP + KV * K::NP + K::NQ;
  static constexpr bool STAGE_TAB = TAB * 8 <= 8 * 1024;
  static constexpr int TAB_SMEM = STAGE_TAB ? TAB : 1;
  static constexpr int BYTES_PER_CELL = 8 * (MNP + M * KVP);
  static constexpr int BY_ROWS = 128 / M;
  static constexpr int BY_SMEM = (40 * 1024 - 8 * TAB_SMEM) / BYTES_PER_CELL;
  static constexpr int CPB = BY_ROWS < BY_SMEM ? BY_ROWS : (BY_SMEM < 1 ? 1 : BY_SMEM);
  static int grid(int n) { return (n + CPB - 1) / CPB; }
};

// the tile's cells: s_e[i] = list[c0 + i], i < nc, for the CTA's tile `blk`
template <int CPB>
__device__ __forceinline__ int lts_tile_cells(const int* __restrict__ list, int n, int blk, int* s_e) {
  const int c0 = blk * CPB;
  const int nc = n - c0 < CPB ? n - c0 : CPB;
  for (int i = threadIdx.x; i < nc; i += blockDim.x) s_e[i] = list[c0 + i];
  __syncthreads();
  return nc;
}

// racc[cell] += s_c[cell] for the tile's cells, element-parallel (128-thread
// CTAs; unrolled so that several loads are in flight)
template <int MNP>
__device__ __forceinline__ void lts_add_rows(const int* s_e, int nc, const double* s_c, double* racc) {
#pragma unroll 4
  for (int x = threadIdx.x; x < nc * MNP; x += 128) {
    const int i = x / MNP;
    racc[(size_t)s_e[i] * MNP + (x - i * MNP)] += s_c[x];
  }
}

// volume term of the listed cells, r[j][k] += sum_q F_j(U_q) . J^-T grad phi_k
// |J| w_q: one thread per (cell, quadrature point) evaluates the flux once for
// all fields into the rows G[(cell, j)][(q, r)]; one thread per (cell, field)
// row contracts its G row with grad phi
template <class K>
__global__ void __launch_bounds__(128) lts_vol_kernel(const __grid_constant__ StageArgs<double> a,
                                                       const int* __restrict__ lists,
                                                       const __grid_constant__ LtsSegs S,
                                                       double* __restrict__ racc) {
  using S_ = LtsTile<K>;
  constexpr int M = K::M, NP = K::NP, NQ = K::NQ, DIM = K::DIM, MNP = K::MNP, KV = K::KV;
  constexpr int CPB = S_::CPB, KVP = S_::KVP;
  __shared__ double s_c[CPB * MNP];
  __shared__ double s_g[CPB * M * KVP];
  __shared__ double s_tab[S_::TAB_SMEM];
  __shared__ int s_e[CPB];
  if (a.gctl->done) return;
  const int tid = threadIdx.x;
  const double* phi = a.tab.phi;
  const double* dphi = a.tab.dphi;
  const double* qw = a.tab.qw;
  if constexpr (S_::STAGE_TAB) {
    for (int x = tid; x < NQ * NP; x += 128) s_tab[x] = a.tab.phi[x];
    for (int x = tid; x < KV * NP; x += 128) s_tab[NQ * NP + x] = a.tab.dphi[x];
    for (int x = tid; x < NQ; x += 128) s_tab[NQ * NP + KV * NP + x] = a.tab.qw[x];
    phi = s_tab;
    dphi = s_tab + NQ * NP;
    qw = s_tab + NQ * NP + KV * NP;
  }
  int blk;
  const int sg = lts_segment(S, blockIdx.x, blk);
  const int nc = lts_tile_cells<CPB>(lists + S.off[sg], S.cnt[sg], blk, s_e);
#pragma unroll 4
  for (int x = tid; x < nc * MNP; x += 128) {
    const int i = x / MNP;
    s_c[x] = a.C[(size_t)s_e[i] * MNP + (x - i * MNP)];
  }
  __syncthreads();
  for (int x = tid; x < nc * NQ; x += 128) {
    const int i = x / NQ, q = x - i * NQ, e = s_e[i];
    const double* c = s_c + i * MNP;
    double U[M];
#pragma unroll
    for (int jj = 0; jj < M; ++jj) {
      double u = 0.0;
#pragma unroll
      for (int k = 0; k < NP; ++k) u += phi[q * NP + k] * c[jj * NP + k];
      U[jj] = u;
    }
    if (!is_physical<K::LAW, double>(a.law, U)) flag_nonphysical(a.status, e);
    double F[M][DIM];
    volume_flux<K::LAW, DIM, double>(a.law, U, F);
    double J[DIM * DIM];
#pragma unroll
    for (int t = 0; t < DIM * DIM; ++t) J[t] = a.mesh.jinv[(size_t)e * DIM * DIM + t];
    const double jw = a.mesh.detjd[e] * qw[q];
#pragma unroll
    for (int j = 0; j < M; ++j)
#pragma unroll
      for (int r = 0; r < DIM; ++r) {
        double g = 0.0;
#pragma unroll
        for (int t = 0; t < DIM; ++t) g += F[j][t] * J[t * DIM + r];
        s_g[(i * M + j) * KVP + q * DIM + r] = g * jw;
      }
  }
  __syncthreads();
  for (int row = tid; row < nc * M; row += 128) {
    double acc[NP];
#pragma unroll
    for (int k = 0; k < NP; ++k) acc[k] = 0.0;
    const double* g = s_g + row * KVP;
    for (int kk = 0; kk < KV; ++kk) {
      const double gv = g[kk];
#pragma unroll
      for (int k = 0; k < NP; ++k) acc[k] += gv * dphi[kk * NP + k];
    }
#pragma unroll
    for (int k = 0; k < NP; ++k) s_c[row * NP + k] = acc[k];  // row < nc * M: own row only
  }
  __syncthreads();
  lts_add_rows<MNP>(s_e, nc, s_c, racc);
}

// the face kernel over face lists: one thread per (listed face, face point);
// the boundary data time of segment i is ctl->t + fac[i] * ctl->dt
template <class K>
__global__ void __launch_bounds__(K::FACE_BLOCK) lts_face_kernel(const __grid_constant__ StageArgs<double> a,
                                                                 const int* __restrict__ lists,
                                                                 const __grid_constant__ LtsSegs S) {
  if (a.gctl->done) return;
  __shared__ double s_fqw[K::NQF];
  __shared__ int s_qmap[K::NPERM * K::NQF];
  const int tid = threadIdx.x;
  for (int i = tid; i < K::NQF; i += blockDim.x) s_fqw[i] = a.tab.fqw[i];
  for (int i = tid; i < K::NPERM * K::NQF; i += blockDim.x) s_qmap[i] = a.tab.qmap[i];
  __syncthreads();
  int blk;
  const int sg = lts_segment(S, blockIdx.x, blk);
  const int fl = tid / K::NQF, q = tid - (tid / K::NQF) * K::NQF;
  const int i = blk * K::FPB + fl;
  if (fl >= K::FPB || i >= S.cnt[sg]) return;
  face_point<K, false, false>(a, lists[S.off[sg] + i], q, nullptr, s_fqw, s_qmap, S.fac[sg]);
}

// lift of the face slots of the classes in `mask` (bit c: class c) into the
// accumulators of the listed cells (every cell touching one of them, once):
// one thread per (cell, field) row over the cell's local faces in order
// (slots read row-coalesced), the sums added element-parallel
template <class K>
__global__ void __launch_bounds__(128) lts_lift_kernel(const __grid_constant__ StageArgs<double> a,
                                                        const int* __restrict__ list, int n,
                                                        const int* __restrict__ cface,
                                                        const int* __restrict__ fcls, unsigned mask,
                                                        double* __restrict__ racc) {
  constexpr int M = K::M, NP = K::NP, NQF = K::NQF, NLF = K::NLF, MNP = K::MNP, NS = K::NS;
  constexpr int CPB = LtsTile<K>::CPB;
  // the face-point basis in shared memory when it takes at most 8 KB
  constexpr bool STAGE = NS * NP * 8 <= 8 * 1024;
  __shared__ double s_c[CPB * MNP];
  __shared__ double s_phif[STAGE ? NS * NP : 1];
  __shared__ int s_e[CPB];
  if (a.gctl->done) return;
  const double* phif = a.tab.phif;
  if constexpr (STAGE) {
    for (int x = threadIdx.x; x < NS * NP; x += 128) s_phif[x] = a.tab.phif[x];
    phif = s_phif;
  }
  const int nc = lts_tile_cells<CPB>(list, n, blockIdx.x, s_e);  // its barrier covers s_phif
  for (int row = threadIdx.x; row < nc * M; row += 128) {
    const int i = row / M, j = row - i * M, e = s_e[i];
    double acc[NP];
#pragma unroll
    for (int k = 0; k < NP; ++k) acc[k] = 0.0;
    for (int lf = 0; lf < NLF; ++lf) {
      const int f = cface[(size_t)e * NLF + lf];
      if (f < 0) continue;
      if (!((mask >> fcls[f]) & 1u)) continue;
      for (int q = 0; q < NQF; ++q) {
        const int s = lf * NQF + q;
        const double sv = a.slots[slot_index<K>(e, s, j)];
#pragma unroll
        for (int k = 0; k < NP; ++k) acc[k] += sv * phif[s * NP + k];
      }
    }
#pragma unroll
    for (int k = 0; k < NP; ++k) s_c[row * NP + k] = acc[k];
  }
  __syncthreads();
  lts_add_rows<MNP>(s_e, nc, s_c, racc);
}

// one of the integrator's coefficient operations on the listed cells,
// element-parallel (every product, quotient and sum rounded once, in the
// reference's order: no contraction); then one thread per (cell, field) row
// writes the row's face-point traces from the new coefficients
template <class K>
__global__ void __launch_bounds__(128) lts_update_kernel(const __grid_constant__ StageArgs<double> a,
                                                          const int* __restrict__ lists,
                                                          const __grid_constant__ LtsSegs S,
                                                          double* __restrict__ c1, double* __restrict__ save,
                                                          double* __restrict__ racc) {
  constexpr int M = K::M, NP = K::NP, NS = K::NS, MNP = K::MNP;
  constexpr int CPB = LtsTile<K>::CPB;
  __shared__ double s_c[CPB * MNP];
  __shared__ int s_e[CPB];
  if (a.gctl->done) return;
  const int tid = threadIdx.x;
  int blk;
  const int sg = lts_segment(S, blockIdx.x, blk);
  const int nc = lts_tile_cells<CPB>(lists + S.off[sg], S.cnt[sg], blk, s_e);
  const int op = S.op[sg];
  const double dt = __dmul_rn(a.ctl->dt, S.fac[sg]);  // fac = 2^-k: exact
  const int ne = nc * MNP;
  double* C = a.Cout;
  // one loop per operation (the operation is uniform over the CTA), unrolled
  // so that each thread has several independent loads in flight
#define LTS_ELEMS(...)                                           \
  _Pragma("unroll 4") for (int xi = tid; xi < ne; xi += 128) {   \
    const int i = xi / MNP;                                      \
    const size_t g = (size_t)s_e[i] * MNP + (xi - i * MNP);      \
    const double det = a.mesh.detjd[s_e[i]];                     \
    (void)det;                                                   \
    double out;                                                  \
    __VA_ARGS__                                                  \
    C[g] = out;                                                  \
    s_c[xi] = out;                                               \
  }
  switch (op) {
    case LTS_EULER_IN:
      LTS_ELEMS({
        const double x = C[g], r = racc[g];
        save[g] = x;
        out = __dadd_rn(x, __dmul_rn(__ddiv_rn(r, det), dt));
        racc[g] = 0.0;
      })
      break;
    case LTS_TWO_HALF:
      LTS_ELEMS({
        const double x = C[g], r = racc[g];
        save[g] = x;
        const double inc = __ddiv_rn(__dmul_rn(r, dt), det);
        const double h = __dadd_rn(x, inc);
        c1[g] = h;
        out = __dadd_rn(h, inc);
        racc[g] = 0.0;
      })
      break;
    case LTS_EULER:
      LTS_ELEMS({
        const double x = C[g], r = racc[g];
        save[g] = x;
        out = __dadd_rn(x, __ddiv_rn(__dmul_rn(r, dt), det));
        racc[g] = 0.0;
      })
      break;
    case LTS_SECOND:
      LTS_ELEMS({
        const double x = C[g], r = racc[g], s0 = save[g];
        out = __dmul_rn(__dadd_rn(__dadd_rn(x, __ddiv_rn(__dmul_rn(r, dt), det)), s0), 0.5);
        racc[g] = 0.0;
      })
      break;
    case LTS_SECOND_SWAP:
      LTS_ELEMS({
        const double x = C[g], r = racc[g], s0 = save[g], x1 = c1[g];
        c1[g] = __dmul_rn(__dadd_rn(__dadd_rn(x, __ddiv_rn(__dmul_rn(r, dt), det)), s0), 0.5);
        out = x1;
      })
      break;
    case LTS_COPYBACK_ZERO:
    case LTS_FINAL_RESET:
      LTS_ELEMS({
        out = c1[g];
        racc[g] = 0.0;
      })
      break;
    case LTS_LI_HALF:
      LTS_ELEMS({
        const double x = C[g], s0 = save[g], x1 = c1[g];
        const double xn = __dadd_rn(__dadd_rn(s0, __dsub_rn(x, s0)),
                                    __dmul_rn(0.25, __dadd_rn(__dsub_rn(x1, __dmul_rn(2.0, x)), s0)));
        save[g] = __dadd_rn(xn, __dmul_rn(0.5, __dsub_rn(x1, s0)));
        out = xn;
      })
      break;
    default:  // LTS_RESTORE
      LTS_ELEMS({ out = save[g]; })
      break;
  }
#undef LTS_ELEMS
  __syncthreads();
  for (int row = tid; row < nc * M; row += 128) {
    const int i = row / M, j = row - i * M, e = s_e[i];
    double o[NP];
#pragma unroll
    for (int k = 0; k < NP; ++k) o[k] = s_c[row * NP + k];
#pragma unroll 4
    for (int s = 0; s < NS; ++s) {
      double t = 0.0;
#pragma unroll
      for (int k = 0; k < NP; ++k) t += a.tab.phif[s * NP + k] * o[k];
      a.tr[slot_index<K>(e, s, j)] = t;
    }
  }
}

}  // namespace dgp
