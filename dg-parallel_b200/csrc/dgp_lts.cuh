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
//   lts_lift_kernel  the slots of one or two face classes lifted into the
//                    accumulators of the cells that touch them (per cell, its
//                    local faces in order: no atomics);
// and every coefficient update is lts_update_kernel with one of the
// integrator's operations, which also refreshes the row's face-point traces.
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

// volume term of the listed cells: one thread per (cell, field) row,
// r[j][k] += sum_q F_j(U_q) . J^-T grad phi_k |J| w_q
template <class K>
__global__ void __launch_bounds__(128) lts_vol_kernel(const __grid_constant__ StageArgs<double> a,
                                                       const int* __restrict__ list, int n,
                                                       double* __restrict__ racc) {
  constexpr int M = K::M, NP = K::NP, NQ = K::NQ, DIM = K::DIM, MNP = K::MNP;
  if (a.gctl->done) return;
  const int gid = blockIdx.x * blockDim.x + threadIdx.x;
  if (gid >= n * M) return;
  const int e = list[gid / M], j = gid - (gid / M) * M;
  const double* c = a.C + (size_t)e * MNP;
  double J[DIM * DIM];
#pragma unroll
  for (int i = 0; i < DIM * DIM; ++i) J[i] = a.mesh.jinv[(size_t)e * DIM * DIM + i];
  const double det = a.mesh.detjd[e];
  double acc[NP];
#pragma unroll
  for (int k = 0; k < NP; ++k) acc[k] = 0.0;
  for (int q = 0; q < NQ; ++q) {
    double U[M];
#pragma unroll
    for (int jj = 0; jj < M; ++jj) {
      double u = 0.0;
#pragma unroll
      for (int k = 0; k < NP; ++k) u += a.tab.phi[q * NP + k] * c[jj * NP + k];
      U[jj] = u;
    }
    if (j == 0 && !is_physical<K::LAW, double>(a.law, U)) flag_nonphysical(a.status, e);
    double F[M][DIM];
    volume_flux<K::LAW, DIM, double>(a.law, U, F);
    const double jw = det * a.tab.qw[q];
#pragma unroll
    for (int r = 0; r < DIM; ++r) {
      double g = 0.0;
#pragma unroll
      for (int i = 0; i < DIM; ++i) g += F[j][i] * J[i * DIM + r];
      g *= jw;
#pragma unroll
      for (int k = 0; k < NP; ++k) acc[k] += g * a.tab.dphi[(q * DIM + r) * NP + k];
    }
  }
  double* ro = racc + (size_t)e * MNP + j * NP;
#pragma unroll
  for (int k = 0; k < NP; ++k) ro[k] += acc[k];
}

// the face kernel over a face list: one thread per (listed face, face point);
// the boundary data time is ctl->t + stage_time_factor * ctl->dt
template <class K>
__global__ void __launch_bounds__(K::FACE_BLOCK) lts_face_kernel(const __grid_constant__ StageArgs<double> a,
                                                                 const int* __restrict__ flist, int n) {
  if (a.gctl->done) return;
  __shared__ double s_fqw[K::NQF];
  __shared__ int s_qmap[K::NPERM * K::NQF];
  const int tid = threadIdx.x;
  for (int i = tid; i < K::NQF; i += blockDim.x) s_fqw[i] = a.tab.fqw[i];
  for (int i = tid; i < K::NPERM * K::NQF; i += blockDim.x) s_qmap[i] = a.tab.qmap[i];
  __syncthreads();
  const int fl = tid / K::NQF, q = tid - (tid / K::NQF) * K::NQF;
  const int i = blockIdx.x * K::FPB + fl;
  if (fl >= K::FPB || i >= n) return;
  face_point<K, false, false>(a, flist[i], q, nullptr, s_fqw, s_qmap);
}

// lift of the face slots of classes clsA / clsB into the accumulators of the
// listed cells: one thread per (cell, field) row, local faces in order
template <class K>
__global__ void __launch_bounds__(128) lts_lift_kernel(const __grid_constant__ StageArgs<double> a,
                                                        const int* __restrict__ list, int n,
                                                        const int* __restrict__ cface,
                                                        const int* __restrict__ fcls, int clsA, int clsB,
                                                        double* __restrict__ racc) {
  constexpr int M = K::M, NP = K::NP, NQF = K::NQF, NLF = K::NLF, MNP = K::MNP;
  if (a.gctl->done) return;
  const int gid = blockIdx.x * blockDim.x + threadIdx.x;
  if (gid >= n * M) return;
  const int e = list[gid / M], j = gid - (gid / M) * M;
  double acc[NP];
#pragma unroll
  for (int k = 0; k < NP; ++k) acc[k] = 0.0;
  for (int lf = 0; lf < NLF; ++lf) {
    const int f = cface[(size_t)e * NLF + lf];
    if (f < 0) continue;
    const int c = fcls[f];
    if (c != clsA && c != clsB) continue;
    for (int q = 0; q < NQF; ++q) {
      const int s = lf * NQF + q;
      const double sv = a.slots[slot_index<K>(e, s, j)];
#pragma unroll
      for (int k = 0; k < NP; ++k) acc[k] += sv * a.tab.phif[s * NP + k];
    }
  }
  double* ro = racc + (size_t)e * MNP + j * NP;
#pragma unroll
  for (int k = 0; k < NP; ++k) ro[k] += acc[k];
}

// one of the integrator's coefficient operations on the listed cells, one
// thread per (cell, field) row, each product, quotient and sum rounded once
// in the reference's order (no contraction); then the row's face-point traces
template <class K>
__global__ void __launch_bounds__(128) lts_update_kernel(const __grid_constant__ StageArgs<double> a,
                                                          const int* __restrict__ list, int n, int op,
                                                          double dt_factor, double* __restrict__ c1,
                                                          double* __restrict__ save, double* __restrict__ racc) {
  constexpr int M = K::M, NP = K::NP, NS = K::NS, MNP = K::MNP;
  if (a.gctl->done) return;
  const int gid = blockIdx.x * blockDim.x + threadIdx.x;
  if (gid >= n * M) return;
  const int e = list[gid / M], j = gid - (gid / M) * M;
  const double dt = __dmul_rn(a.ctl->dt, dt_factor);  // dt_factor = 2^-k: exact
  const double det = a.mesh.detjd[e];
  const size_t base = (size_t)e * MNP + j * NP;
  double* c = a.Cout + base;
  double* cc = c1 + base;
  double* sv = save + base;
  double* r = racc + base;
  double o[NP];
#pragma unroll
  for (int k = 0; k < NP; ++k) {
    double x = c[k];
    switch (op) {
      case LTS_EULER_IN:
        sv[k] = x;
        x = __dadd_rn(x, __dmul_rn(__ddiv_rn(r[k], det), dt));
        r[k] = 0.0;
        break;
      case LTS_TWO_HALF: {
        sv[k] = x;
        const double inc = __ddiv_rn(__dmul_rn(r[k], dt), det);
        x = __dadd_rn(x, inc);
        cc[k] = x;
        x = __dadd_rn(x, inc);
        r[k] = 0.0;
        break;
      }
      case LTS_EULER:
        sv[k] = x;
        x = __dadd_rn(x, __ddiv_rn(__dmul_rn(r[k], dt), det));
        r[k] = 0.0;
        break;
      case LTS_SECOND:
      case LTS_SECOND_SWAP: {
        const double xn = __dmul_rn(__dadd_rn(__dadd_rn(x, __ddiv_rn(__dmul_rn(r[k], dt), det)), sv[k]), 0.5);
        if (op == LTS_SECOND) {
          x = xn;
          r[k] = 0.0;
        } else {
          x = cc[k];
          cc[k] = xn;
        }
        break;
      }
      case LTS_COPYBACK_ZERO:
      case LTS_FINAL_RESET:
        x = cc[k];
        r[k] = 0.0;
        break;
      case LTS_LI_HALF: {
        const double s0 = sv[k], x1 = cc[k];
        const double xn = __dadd_rn(__dadd_rn(s0, __dsub_rn(x, s0)),
                                    __dmul_rn(0.25, __dadd_rn(__dsub_rn(x1, __dmul_rn(2.0, x)), s0)));
        sv[k] = __dadd_rn(xn, __dmul_rn(0.5, __dsub_rn(x1, s0)));
        x = xn;
        break;
      }
      default:  // LTS_RESTORE
        x = sv[k];
        break;
    }
    c[k] = x;
    o[k] = x;
  }
  // face-point traces of the new row for the face kernel
#pragma unroll 4
  for (int s = 0; s < NS; ++s) {
    double t = 0.0;
#pragma unroll
    for (int k = 0; k < NP; ++k) t += a.tab.phif[s * NP + k] * o[k];
    a.tr[slot_index<K>(e, s, j)] = t;
  }
}

}  // namespace dgp
