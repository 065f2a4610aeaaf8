// Element kernel of one explicit DG stage: volume term + lift of the face
// slots + inverse mass + SSP-RK3 combination for a tile of TE cells, with the
// last stage's CFL and residual reductions fused in.
//
// Work mapping (BLOCK = 128 threads):
//   volume   thread (q, g) owns quadrature point q and keeps phi(q,:) in
//            registers; it walks cells g, g+EG, ... of the tile: interpolate the
//            state (DGCell::interpolate, DGCell.h:217-227), evaluate the flux
//            (ConservationLaw::Fi) and map it to reference directions with the
//            cell's J^{-1} |J| w, writing G[(q,r)][(cell,field)].
//   contract thread = one (cell, field) row; all modes of the row accumulate in
//            registers: R[row][k] = sum_(q,r) G[(q,r)][row] dphi[(q,r)][k]
//                                  + sum_s S[s][row] phi_face[s][k];
//            every k-step reads one value of its own row and one table row that
//            all lanes share (a broadcast), so shared-memory traffic per FMA is
//            ~1/NP of a naive (row, mode) mapping.
//   update   RungeKuttaTVD3::advanceInTime (TimeIntegrator.cc:838-990) for the
//            row's modes, coalesced per row.
#pragma once

#include "dgp_kernels.cuh"

namespace dgp {

template <typename T>
struct Vec16;
template <>
struct Vec16<double> { using type = double2; static constexpr int N = 2; };
template <>
struct Vec16<float> { using type = float4; static constexpr int N = 4; };

// padded length of a table row so that rows start on 16-byte boundaries
template <typename T, int N>
struct Padded {
  static constexpr int V = Vec16<T>::N;
  static constexpr int value = (N + V - 1) / V * V;
};

template <typename T, int N>
__device__ __forceinline__ void load_row16(const T* __restrict__ p, T (&out)[N]) {
  using V = typename Vec16<T>::type;
  constexpr int W = Vec16<T>::N;
#pragma unroll
  for (int i = 0; i < N / W; ++i) {
    V v = reinterpret_cast<const V*>(p)[i];
    if constexpr (W == 2) {
      out[2 * i] = v.x;
      out[2 * i + 1] = v.y;
    } else {
      out[4 * i] = v.x;
      out[4 * i + 1] = v.y;
      out[4 * i + 2] = v.z;
      out[4 * i + 3] = v.w;
    }
  }
}

template <class K>
struct ElemSmem {
  using T = typename K::T;
  static constexpr int NPP = Padded<T, K::NP>::value;
  static constexpr int DD = K::DIM * K::DIM + 1;
  static constexpr size_t oC = 0;                                         // [ROWS][NP]
  static constexpr size_t oG = oC + (size_t)K::ROWS * K::NP;              // [KV][LDR]
  static constexpr size_t oS = oG + (size_t)K::KV * K::LDR;               // [NS][LDR]
  static constexpr size_t oDphi = (oS + (size_t)K::NS * K::LDR + 3) / 4 * 4;  // [KV][NPP]
  static constexpr size_t oPhif = oDphi + (size_t)K::KV * NPP;            // [NS][NPP]
  static constexpr size_t oPhi = oPhif + (size_t)K::NS * NPP;             // [NQ][NP]
  static constexpr size_t oQw = oPhi + (size_t)K::NQ * K::NP;             // [NQ]
  static constexpr size_t t_bytes = ((oQw + K::NQ) * sizeof(T) + 15) / 16 * 16;
  static constexpr size_t bytes = t_bytes + 8 * ((size_t)K::TE * DD + (size_t)K::TE * K::NV);
};

template <class K>
constexpr size_t elem_kernel_smem() {
  return ElemSmem<K>::bytes;
}

template <class K>
__global__ void __launch_bounds__(K::BLOCK) elem_kernel(StageArgs<typename K::T> a) {
  using T = typename K::T;
  using L = ElemSmem<K>;
  constexpr int M = K::M, NP = K::NP, NQ = K::NQ, DIM = K::DIM, TE = K::TE, BLOCK = K::BLOCK;
  constexpr int MNP = K::MNP, NS = K::NS, KV = K::KV, LDR = K::LDR, NV = K::NV;
  constexpr int NPP = L::NPP, DD = L::DD;
  if (a.ctl->done) return;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  T* sT = reinterpret_cast<T*>(smem_raw);
  T* sC = sT + L::oC;
  T* sG = sT + L::oG;
  T* sS = sT + L::oS;
  T* sDphi = sT + L::oDphi;
  T* sPhif = sT + L::oPhif;
  T* sPhi = sT + L::oPhi;
  T* sQw = sT + L::oQw;
  double* sJ = reinterpret_cast<double*>(smem_raw + L::t_bytes);
  double* sEig = sJ + TE * DD;
  __shared__ double red[BLOCK / 32];
  __shared__ bool amLast;

  const int tid = threadIdx.x;
  const int e0 = blockIdx.x * TE;
  const int ne = min(TE, a.mesh.E - e0);

  // stage tables (rows padded to 16 bytes), the state tile, the slots
  // transposed to [point][row], and the cells' J^{-1} and |J|
  for (int i = tid; i < KV * NPP; i += BLOCK) {
    const int kk = i / NPP, k = i - (i / NPP) * NPP;
    sDphi[i] = k < NP ? a.tab.dphi[kk * NP + k] : T(0);
  }
  for (int i = tid; i < NS * NPP; i += BLOCK) {
    const int s = i / NPP, k = i - (i / NPP) * NPP;
    sPhif[i] = k < NP ? a.tab.phif[s * NP + k] : T(0);
  }
  for (int i = tid; i < NQ * NP; i += BLOCK) sPhi[i] = a.tab.phi[i];
  for (int i = tid; i < NQ; i += BLOCK) sQw[i] = a.tab.qw[i];
  {
    const T* src = a.C + (size_t)e0 * MNP;
    for (int i = tid; i < ne * MNP; i += BLOCK) sC[i] = src[i];
    const T* ss = a.slots + (size_t)e0 * NS * M;
    for (int i = tid; i < ne * NS * M; i += BLOCK) {
      const int e = i / (NS * M), rem = i - e * (NS * M);
      const int s = rem / M, j = rem - (rem / M) * M;
      sS[s * LDR + e * M + j] = ss[i];
    }
    for (int i = tid; i < ne * DD; i += BLOCK) {
      const int e = i / DD, c = i - (i / DD) * DD;
      sJ[i] = c < DIM * DIM ? (double)a.mesh.jinv[(size_t)(e0 + e) * DIM * DIM + c]
                            : (double)a.mesh.detj[e0 + e];
    }
  }
  __syncthreads();

  // volume: fixed quadrature point per thread
  if (tid < K::EG * NQ) {
    const int q = tid % NQ, g = tid / NQ;
    T phi[NP];
#pragma unroll
    for (int k = 0; k < NP; ++k) phi[k] = sPhi[q * NP + k];
    const T w = sQw[q];
    for (int e = g; e < ne; e += K::EG) {
      const T* c = sC + e * MNP;
      T U[M];
#pragma unroll
      for (int j = 0; j < M; ++j) {
        T acc = 0;
#pragma unroll
        for (int k = 0; k < NP; ++k) acc += phi[k] * c[j * NP + k];
        U[j] = acc;
      }
      if (!is_physical<K::LAW, T>(a.law, U)) flag_nonphysical(a.status, e0 + e);
      T F[M][DIM];
      volume_flux<K::LAW, DIM, T>(a.law, U, F);
      const double* Jd = sJ + e * DD;
      T J[DIM * DIM];
#pragma unroll
      for (int i = 0; i < DIM * DIM; ++i) J[i] = (T)Jd[i];
      const T jw = (T)Jd[DIM * DIM] * w;
#pragma unroll
      for (int j = 0; j < M; ++j)
#pragma unroll
        for (int r = 0; r < DIM; ++r) {
          T acc = 0;
#pragma unroll
          for (int i = 0; i < DIM; ++i) acc += F[j][i] * J[i * DIM + r];
          sG[(q * DIM + r) * LDR + e * M + j] = acc * jw;
        }
    }
  }
  __syncthreads();

  // contraction + lift + inverse mass + stage combination, one row per thread
  double rsum = 0.0;
  const int row = tid;
  if (row < ne * M) {
    T acc[NPP];
#pragma unroll
    for (int k = 0; k < NPP; ++k) acc[k] = 0;
#pragma unroll 4
    for (int kk = 0; kk < KV; ++kk) {
      const T gv = sG[kk * LDR + row];
      T d[NPP];
      load_row16<T, NPP>(sDphi + kk * NPP, d);
#pragma unroll
      for (int k = 0; k < NPP; ++k) acc[k] += gv * d[k];
    }
#pragma unroll 4
    for (int s = 0; s < NS; ++s) {
      const T sv = sS[s * LDR + row];
      T p[NPP];
      load_row16<T, NPP>(sPhif + s * NPP, p);
#pragma unroll
      for (int k = 0; k < NPP; ++k) acc[k] += sv * p[k];
    }
    const size_t gbase = ((size_t)e0 * M + row) * NP;
    if (a.stage == 0) {
#pragma unroll
      for (int k = 0; k < NP; ++k) a.Cout[gbase + k] = acc[k];
    } else {
      const int e = row / M;
      const T dtj = (T)(a.ctl->dt / sJ[e * DD + DIM * DIM]);
      T* crow = sC + row * NP;
#pragma unroll
      for (int k = 0; k < NP; ++k) {
        const T c = crow[k];
        T out;
        if (a.stage == 1) {
          a.U0out[gbase + k] = c;
          out = c + acc[k] * dtj;
        } else if (a.stage == 2) {
          out = (T)0.25 * (c + acc[k] * dtj + (T)3. * a.U0[gbase + k]);
        } else {
          const T u0 = a.U0[gbase + k];
          out = ((T)2.0 * (c + acc[k] * dtj) + u0) / (T)3.0;
          const double dd = (double)out - (double)u0;
          rsum += dd * dd;
        }
        crow[k] = out;
        a.Cout[gbase + k] = out;
      }
    }
  }
  if (a.stage != 3) return;

  // last stage: residual partial and the CFL step of the next step
  rsum = block_sum<BLOCK>(rsum, red);
  if (tid == 0) a.partials[blockIdx.x] = rsum;
  if (a.fuse_cfl) {
    __syncthreads();
    // eigenvalue at the cell mean (v = 0) and, on triangles, at the three
    // reference vertices (DGCell::computeMAXEV, DGCell.cc:1155-1207)
    for (int it = tid; it < ne * NV; it += BLOCK) {
      const int e = it / NV, v = it - (it / NV) * NV;
      const T* c = sC + e * MNP;
      T val[M];
      if (v == 0) {
#pragma unroll
        for (int j = 0; j < M; ++j) val[j] = c[j * NP] * (T)a.tab.phi0;
      } else {
        const double* pv = a.tab.phiv + (v - 1) * NP;
#pragma unroll
        for (int j = 0; j < M; ++j) {
          T acc = 0;
#pragma unroll
          for (int k = 0; k < NP; ++k) acc += (T)pv[k] * c[j * NP + k];
          val[j] = acc;
        }
      }
      sEig[it] = (double)max_eigen<K::LAW, T>(a.law, val);
    }
    __syncthreads();
    double dtl = 1e300;
    if (tid < ne) {
      double am = sEig[tid * NV];
#pragma unroll
      for (int v = 1; v < NV; ++v) {
        const double b = sEig[tid * NV + v];
        am = (b > am ? b : am);
      }
      dtl = a.mesh.csize[e0 + tid] * a.ctl->cfl / (am * (2. * K::ORDER + 1.0));
    }
    dtl = block_min<BLOCK>(dtl, red);
    if (tid == 0) atomicMin(&a.ctl->dtmin_bits, (unsigned long long)__double_as_longlong(dtl));
  }
  if (tid == 0) {
    __threadfence();
    const unsigned v = atomicAdd(&a.ctl->blocks_done, 1u);
    amLast = (v == gridDim.x - 1);
  }
  __syncthreads();
  if (!amLast) return;
  // the last CTA: residual in a fixed order (strided partial sums + tree)
  __threadfence();
  double r = 0.0;
  for (unsigned b = tid; b < gridDim.x; b += BLOCK) r += ((volatile double*)a.partials)[b];
  r = block_sum<BLOCK>(r, red);
  if (tid == 0) {
    TimeCtl* c = a.ctl;
    c->resid = r;
    c->blocks_done = 0;
    c->t = c->t + c->dt;
    c->steps += 1;
    if (a.fuse_cfl) {
      const unsigned long long bits = atomicExch(&c->dtmin_bits, 0x7FF0000000000000ull);
      ctl_finalize(c, __longlong_as_double((long long)bits));
    }
  }
}

}  // namespace dgp
