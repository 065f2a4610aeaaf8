// Discrete adjoint of one SSP-RK3 stage: the transpose of the linearised
// right-hand side L(u) = M^{-1} R(u) applied to an adjoint vector, fused with
// the reversed stage combination.  The forward operator is the one of
// dgp_kernels.cuh / dgp_elem.cuh (DGCell::computeVolumeContribution,
// DGCell.cc:184-249; DGBoundaryCell::computeBoundaryContributions,
// DGCell.cc:639-732; RungeKuttaTVD3::advanceInTime, TimeIntegrator.cc:838-990).
//
// With nu = mu / |J| per cell (the inverse mass is diagonal):
//   faces   per face point, the traces of nu on both sides give the flux
//           cotangent Fbar = (nu_R - nu_L) |J_f| w; the Jacobians dF^/dU_L and
//           dF^/dU_R come from evaluating the law's numerical (or boundary)
//           flux on dual numbers; U_L^bar = Fbar dF^/dU_L is written into the
//           left cell's face slot, U_R^bar into the right cell's (no atomics,
//           the forward slot layout);
//   volume  H[(cell,j)][(q,r)] = sum_k dphi_(q,r),k nu[j][k] (the transposed
//           contraction), flux cotangent Fbar_ji = sum_r H_jr J^{-1}_ir |J| w_q,
//           U^bar_m(q) = sum_ji Fbar_ji dF_ji/dU_m(U(q)) (dual numbers), and
//           w[m][k] = sum_q phi_k(q) U^bar_m(q) + sum_s slot_s[m] phi_s,k (the
//           same lift as the forward face term).
// Stage combination (per row, FP64): out = ca mu + cb dt w + cc acc and
// acc <- cd acc + ce mu, which runs the three reversed stages
//   lambda2 = 2/3 lambda3 + 2/3 dt L'(u2)^T lambda3,  acc = 1/3 lambda3
//   lambda1 = 1/4 lambda2 + 1/4 dt L'(u1)^T lambda2,  acc += 3/4 lambda2
//   lambda_n = acc + lambda1 + dt L'(u_n)^T lambda1.
#pragma once

#include "dgp_dual.cuh"
#include "dgp_elem.cuh"

namespace dgp {

template <typename T>
struct AdjArgs {
  StageArgs<T> s;      // forward state of the stage in s.C, tables, geometry, slots
  const double* mu;    // adjoint input [cell][field][mode] (internal order)
  double* out;         // adjoint output
  double* acc;         // running sum of the reversed stages (read and/or written)
  double ca, cb, cc, cd, ce;
  double dt;
  const double* t_seg; // device: time at the start of the step
  double t_factor;     // stage time = *t_seg + t_factor * dt (as the forward stage)
};

// input directions per dual-number pass of the face Jacobians: the 2M
// directions of both sides in as few passes of at most 8 lanes as possible,
// split evenly (one pass for the 2D Euler law: 0.90x the backward time of two
// lanes a pass on the adjoint workload); two lanes for the exact Riemann
// solver, whose iteration would otherwise carry 8-lane dual numbers
template <class K>
constexpr int adj_lanes() {
  constexpr int dirs = 2 * K::M, passes = (dirs + 7) / 8;
  return K::FLUX == DGP_FLUX_GODUNOV ? 2 : (dirs + passes - 1) / passes;
}

// trace of nu = mu / |J| at one face point
template <class K>
__device__ __forceinline__ void nu_trace(const double* __restrict__ mu, double inv_detj,
                                         const typename K::T* phi, typename K::T* V) {
  using T = typename K::T;
#pragma unroll
  for (int j = 0; j < K::M; ++j) {
    T acc = 0;
#pragma unroll
    for (int k = 0; k < K::NP; ++k) acc += phi[k] * (T)__ldg(mu + j * K::NP + k);
    V[j] = acc * (T)inv_detj;
  }
}

template <class K>
__global__ void __launch_bounds__(K::FACE_BLOCK) adj_face_kernel(const __grid_constant__ AdjArgs<typename K::T> a) {
  using T = typename K::T;
  constexpr int M = K::M, NP = K::NP, NQF = K::NQF, DIM = K::DIM, MNP = K::MNP;
  __shared__ T s_phif[K::NLF * NQF * NP];
  __shared__ T s_fqw[NQF];
  __shared__ int s_qmap[K::NPERM * NQF];
  face_tables<K>(a.s, s_phif, s_fqw, s_qmap);
  const int tid = threadIdx.x;
  const int fl = tid / NQF, q = tid - (tid / NQF) * NQF;
  const int f = blockIdx.x * K::FPB + fl;
  if (fl >= K::FPB || f >= a.s.mesh.F) return;
  const auto& m = a.s.mesh;
  const int eL = m.fel[2 * f], eR = m.fel[2 * f + 1];
  const int code = m.fcode[f];
  const int lfL = code & 15, lfR = (code >> 4) & 15, perm = code >> 8;
  T n[DIM];
#pragma unroll
  for (int i = 0; i < DIM; ++i) n[i] = m.fnrm[f * DIM + i];
  const T jw = m.fj[f] * s_fqw[q];
  T UL[M], UR[M], VL[M], VR[M], gL[M], gR[M];
  const T* phiL = s_phif + (lfL * NQF + q) * NP;
  cell_trace<K>(a.s.C + (size_t)eL * MNP, phiL, UL);
  nu_trace<K>(a.mu + (size_t)eL * MNP, 1.0 / m.detjd[eL], phiL, VL);
  if (eR >= 0) {
    const int qR = s_qmap[perm * NQF + q];
    const T* phiR = s_phif + (lfR * NQF + qR) * NP;
    cell_trace<K>(a.s.C + (size_t)eR * MNP, phiR, UR);
    nu_trace<K>(a.mu + (size_t)eR * MNP, 1.0 / m.detjd[eR], phiR, VR);
    // the Jacobian W input directions per pass (narrow dual numbers keep the
    // flux in registers); direction c < M is d/dU_L[c], c >= M is d/dU_R[c - M]
    constexpr int W = adj_lanes<K>();
    using D = Dual<T, W>;
    T fb[M];
#pragma unroll
    for (int j = 0; j < M; ++j) fb[j] = (VR[j] - VL[j]) * jw;
#pragma unroll 1
    for (int c0 = 0; c0 < 2 * M; c0 += W) {
      D dl[M], dr[M], nd[DIM], F[M];
#pragma unroll
      for (int j = 0; j < M; ++j) {
        dl[j] = D::var(UL[j], j - c0);
        dr[j] = D::var(UR[j], M + j - c0);
      }
#pragma unroll
      for (int i = 0; i < DIM; ++i) nd[i] = D(n[i]);
      numerical_flux<K::LAW, K::FLUX, DIM, D>(a.s.law, nd, dl, dr, F);
#pragma unroll
      for (int w = 0; w < W; ++w) {
        T g = 0;
#pragma unroll
        for (int j = 0; j < M; ++j) g += fb[j] * F[j].d[w];
        const int c = c0 + w;
#pragma unroll
        for (int k = 0; k < M; ++k) {
          if (k == c) gL[k] = g;
          if (k + M == c) gR[k] = g;
        }
      }
    }
    T* sr = a.s.slots + slot_index<K>(eR, lfR * NQF + qR, 0);
#pragma unroll
    for (int c = 0; c < M; ++c) sr[c] = gR[c];
  } else {
    constexpr int W = adj_lanes<K>();
    using D = Dual<T, W>;
    const int b = -eR - 1;
    const double* x = m.bpts + ((size_t)b * NQF + q) * 3;
    const double time = __fma_rn(a.t_factor, a.dt, *a.t_seg);
#pragma unroll 1
    for (int c0 = 0; c0 < M; c0 += W) {
      D dl[M], nd[DIM], F[M];
#pragma unroll
      for (int j = 0; j < M; ++j) dl[j] = D::var(UL[j], j - c0);
#pragma unroll
      for (int i = 0; i < DIM; ++i) nd[i] = D(n[i]);
      boundary_flux<K::LAW, K::FLUX, DIM, D>(a.s.law, m.bbid[b], nd, x, time, dl, F);
#pragma unroll
      for (int w = 0; w < W; ++w) {
        T g = 0;
#pragma unroll
        for (int j = 0; j < M; ++j) g += -VL[j] * jw * F[j].d[w];
#pragma unroll
        for (int k = 0; k < M; ++k)
          if (k == c0 + w) gL[k] = g;
      }
    }
  }
  T* sl = a.s.slots + slot_index<K>(eL, lfL * NQF + q, 0);
#pragma unroll
  for (int c = 0; c < M; ++c) sl[c] = gL[c];
}

template <class K>
struct AdjSmem {
  using T = typename K::T;
  using L = ElemSmem<K>;
  static constexpr int NQP = K::NQ | 1;  // row stride of U^bar (odd)
  static constexpr size_t oU = L::r16(L::bytes);                                   // T [ROWS][NQP]
  static constexpr size_t oN = oU + L::r16((size_t)K::ROWS * NQP * sizeof(T));     // T [ROWS][NP] nu
  static constexpr size_t oM = oN + L::r16((size_t)K::ROWS * K::NP * sizeof(T));   // FP64 [ROWS][NP] mu
  static constexpr size_t bytes = oM + (size_t)K::ROWS * K::NP * 8;
};

template <class K>
constexpr size_t adj_elem_smem() {
  return AdjSmem<K>::bytes;
}

template <class K>
__global__ void __launch_bounds__(K::BLOCK) adj_elem_kernel(const __grid_constant__ AdjArgs<typename K::T> a) {
  using T = typename K::T;
  using L = ElemSmem<K>;
  using A = AdjSmem<K>;
  constexpr int M = K::M, NP = K::NP, NQ = K::NQ, DIM = K::DIM, TE = K::TE, BLOCK = K::BLOCK;
  constexpr int MNP = K::MNP, NS = K::NS, KV = K::KV, LDK = K::LDK, ROWS = K::ROWS;
  constexpr int NPP = L::NPP, DD = L::DD, NQP = A::NQP;
  extern __shared__ __align__(128) unsigned char smem_raw[];
  T* sT = reinterpret_cast<T*>(smem_raw);
  const T* sDphi = sT + L::oDphi;
  const T* sPhif = sT + L::oPhif;
  const T* sPhi = sT + L::oPhi;
  const T* sQw = sT + L::oQw;
  double* sC = reinterpret_cast<double*>(smem_raw + L::oCB);
  T* sH = reinterpret_cast<T*>(smem_raw + L::oGB);
  double* sJ = reinterpret_cast<double*>(smem_raw + L::oJB);
  T* sUb = reinterpret_cast<T*>(smem_raw + A::oU);
  T* sNu = reinterpret_cast<T*>(smem_raw + A::oN);
  double* sMu = reinterpret_cast<double*>(smem_raw + A::oM);
  const int tid = threadIdx.x;
  const int e0 = blockIdx.x * TE;
  const int ne = min(TE, a.s.mesh.E - e0);
  const auto& m = a.s.mesh;

  for (int i = tid; i < (int)(L::blob_bytes / sizeof(T)); i += BLOCK) sT[i] = a.s.tab.blob[i];
  for (int i = tid; i < ne * MNP; i += BLOCK) {
    sC[i] = a.s.C[(size_t)e0 * MNP + i];
    sMu[i] = a.mu[(size_t)e0 * MNP + i];
  }
  for (int i = tid; i < ne * DD; i += BLOCK) {
    const int e = i / DD, c = i - (i / DD) * DD;
    sJ[i] = c < DIM * DIM ? (double)m.jinv[(size_t)(e0 + e) * DIM * DIM + c] : m.detjd[e0 + e];
  }
  __syncthreads();
  for (int i = tid; i < ne * MNP; i += BLOCK) sNu[i] = (T)(sMu[i] / sJ[(i / MNP) * DD + DIM * DIM]);
  __syncthreads();

  // transposed contraction: H[row][kk] = sum_k dphi[kk][k] nu[row][k]
  const int row = tid;
  if (row < ne * M) {
    T nu[NP];
#pragma unroll
    for (int k = 0; k < NP; ++k) nu[k] = sNu[row * NP + k];
    for (int kk = 0; kk < KV; ++kk) {
      T acc = 0;
#pragma unroll
      for (int k = 0; k < NP; ++k) acc += sDphi[kk * NPP + k] * nu[k];
      sH[row * LDK + kk] = acc;
    }
  }
  __syncthreads();

  // volume: U^bar_m(q) = sum_ji Fbar_ji dF_ji/dU_m at each quadrature point
  if (tid < K::EG * NQ) {
    const int q = tid % NQ, g = tid / NQ;
    T phi[NP];
#pragma unroll
    for (int k = 0; k < NP; ++k) phi[k] = sPhi[q * NPP + k];
    const T w = sQw[q];
    using D = Dual<T, M>;
    for (int e = g; e < ne; e += K::EG) {
      D U[M];
#pragma unroll
      for (int j = 0; j < M; ++j) {
        T acc = 0;
#pragma unroll
        for (int k = 0; k < NP; ++k) acc += phi[k] * (T)sC[(e * M + j) * NP + k];
        U[j] = D::var(acc, j);
      }
      D F[M][DIM];
      volume_flux<K::LAW, DIM, D>(a.s.law, U, F);
      const double* Jd = sJ + e * DD;
      const T jw = (T)Jd[DIM * DIM] * w;
      T ub[M];
#pragma unroll
      for (int c = 0; c < M; ++c) ub[c] = 0;
#pragma unroll
      for (int j = 0; j < M; ++j)
#pragma unroll
        for (int i = 0; i < DIM; ++i) {
          T fb = 0;
#pragma unroll
          for (int r = 0; r < DIM; ++r) fb += sH[(e * M + j) * LDK + q * DIM + r] * (T)Jd[i * DIM + r];
          fb *= jw;
#pragma unroll
          for (int c = 0; c < M; ++c) ub[c] += fb * F[j][i].d[c];
        }
#pragma unroll
      for (int c = 0; c < M; ++c) sUb[(e * M + c) * NQP + q] = ub[c];
    }
  }
  __syncthreads();

  // w = sum_q phi_k(q) U^bar(q) + lift of the adjoint face slots, then the
  // reversed stage combination in FP64
  if (row < ne * M) {
    T acc[NP];
#pragma unroll
    for (int k = 0; k < NP; ++k) acc[k] = 0;
    for (int q = 0; q < NQ; ++q) {
      const T ub = sUb[row * NQP + q];
#pragma unroll
      for (int k = 0; k < NP; ++k) acc[k] += ub * sPhi[q * NPP + k];
    }
    const T* sl = a.s.slots + (size_t)blockIdx.x * NS * ROWS + row;
    for (int s = 0; s < NS; ++s) {
      const T sv = __ldg(sl + (size_t)s * ROWS);
#pragma unroll
      for (int k = 0; k < NP; ++k) acc[k] += sv * sPhif[s * NPP + k];
    }
    const size_t gbase = ((size_t)e0 * M + row) * NP;
#pragma unroll
    for (int k = 0; k < NP; ++k) {
      const double mu = sMu[row * NP + k];
      const double w = (double)acc[k];
      double o = a.ca * mu + a.cb * a.dt * w;
      if (a.cc != 0.0) o += a.cc * a.acc[gbase + k];
      a.out[gbase + k] = o;
      if (a.cd != 0.0 || a.ce != 0.0) a.acc[gbase + k] = (a.cd != 0.0 ? a.cd * a.acc[gbase + k] : 0.0) + a.ce * mu;
    }
  }
}

// ---- objective: J = sum_r (rho(x_r) - obs_r)^2 at receiver points ----------
struct Receivers {
  int n;
  const int* cell;       // internal cell of each receiver
  const double* phi;     // [n][NP] basis at the receiver's reference point
  const double* obs;     // [n]
  int np, mnp;
};

// rho at the receivers (field 0) and J, one block of 256 threads
static __global__ void receiver_values_kernel(Receivers r, const double* C, double* rho, double* J) {
  __shared__ double red[32];
  double acc = 0.0;
  for (int i = threadIdx.x; i < r.n; i += blockDim.x) {
    const double* c = C + (size_t)r.cell[i] * r.mnp;
    double v = 0.0;
    for (int k = 0; k < r.np; ++k) v += r.phi[(size_t)i * r.np + k] * c[k];
    rho[i] = v;
    const double d = v - r.obs[i];
    acc += d * d;
  }
  for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = acc;
  __syncthreads();
  if (threadIdx.x == 0) {
    double s = 0.0;
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) s += red[w];
    *J = s;
  }
}

// dJ/du_T: 2 (rho_r - obs_r) phi_k(x_r) in row (cell_r, field 0); one thread
// walks the receivers in order (receivers may share a cell)
static __global__ void receiver_seed_kernel(Receivers r, const double* rho, double* lam) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  for (int i = 0; i < r.n; ++i) {
    const double g = 2.0 * (rho[i] - r.obs[i]);
    double* l = lam + (size_t)r.cell[i] * r.mnp;
    for (int k = 0; k < r.np; ++k) l[k] += g * r.phi[(size_t)i * r.np + k];
  }
}

}  // namespace dgp
