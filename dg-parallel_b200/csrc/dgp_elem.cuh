// Element kernel of one explicit DG stage: volume term + lift of the face
// slots + inverse mass + SSP-RK3 combination for a tile of TE cells, with the
// last stage's CFL and residual reductions fused in.
//
// Staging: one elected thread issues two bulk (1D TMA) copies completed on an
// mbarrier -- the reference tables (basis at the volume points, reference
// gradients, face traces, weights: one blob already in shared-memory layout)
// and the tile's coefficients (contiguous [cell][field][mode]).
//
// Work mapping (BLOCK = 128 threads):
//   volume   thread (q, g) owns quadrature point q and keeps phi(q,:) in
//            registers; it walks cells g, g+EG, ... of the tile: interpolate the
//            state (DGCell::interpolate, DGCell.h:217-227) with 16-byte reads of
//            the cell's rows, evaluate the flux (ConservationLaw::Fi) and map it
//            to reference directions with the cell's J^{-1} |J| w, writing
//            G[(cell,field)][(q,r)] (odd row stride).  (A thread-per-row
//            interpolation with broadcast table rows measured slower: as many
//            shared loads plus a round trip of the point states.)
//   contract thread = one (cell, field) row; all modes of the row accumulate in
//            registers: R[row][k] = sum_(q,r) G[row][(q,r)] dphi[(q,r)][k]
//                                  + sum_s S[s][row] phi_face[s][k];
//            each k-step reads one value of the thread's own row and one table
//            row all lanes share (a 16-byte broadcast); the face slots S come
//            straight from global memory in their tile-transposed layout
//            (row-coalesced), never staged.
//   update   RungeKuttaTVD3::advanceInTime (TimeIntegrator.cc:838-990) for the
//            row's modes in the reference's operation order.
#pragma once

#include "dgp_kernels.cuh"
#include "dgp_tma.cuh"

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

// N consecutive values from shared memory with the widest aligned vector
// loads (p is aligned to N*sizeof(T) modulo 16)
template <typename T, int N>
__device__ __forceinline__ void load_vec(const T* __restrict__ p, T (&out)[N]) {
  if constexpr ((N * sizeof(T)) % 16 == 0) {
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
  } else if constexpr (sizeof(T) == 4 && (N * sizeof(T)) % 8 == 0) {
#pragma unroll
    for (int i = 0; i < N / 2; ++i) {
      float2 v = reinterpret_cast<const float2*>(p)[i];
      out[2 * i] = v.x;
      out[2 * i + 1] = v.y;
    }
  } else {
#pragma unroll
    for (int i = 0; i < N; ++i) out[i] = p[i];
  }
}

template <class K>
struct ElemSmem {
  using T = typename K::T;
  static constexpr int V = Vec16<T>::N;
  static constexpr int NPP = Padded<T, K::NP>::value;
  static constexpr int DD = K::DIM * K::DIM + 1;
  // table blob (bulk copied as one piece, same layout in global memory)
  static constexpr size_t oDphi = 0;                                   // [KV][NPP]
  static constexpr size_t oPhif = oDphi + (size_t)K::KV * NPP;         // [NS][NPP]
  static constexpr size_t oPhi = oPhif + (size_t)K::NS * NPP;          // [NQ][NPP]
  static constexpr size_t oQw = oPhi + (size_t)K::NQ * NPP;            // [NQ] padded
  static constexpr size_t blob_elems = oQw + (K::NQ + V - 1) / V * V;
  static constexpr size_t blob_bytes = blob_elems * sizeof(T);
  // tile, byte offsets: FP64 coefficients [ROWS][NP], G [ROWS][LDK] (T),
  // FP64 J^{-1}, |J| [TE][DD] and CFL eigenvalues [TE][NV], FP64 u_n
  // [ROWS][NP], face slots [NS][ROWS] (T)
  static constexpr size_t r16(size_t n) { return (n + 15) / 16 * 16; }
  static constexpr size_t oCB = r16(blob_bytes);
  static constexpr size_t oGB = oCB + r16((size_t)K::ROWS * K::NP * 8);
  static constexpr size_t oJB = oGB + r16((size_t)K::ROWS * K::LDK * sizeof(T));
  static constexpr size_t oUB = oJB + r16(8 * ((size_t)K::TE * DD + (size_t)K::TE * K::NV));
  static constexpr size_t oSB = oUB + r16((size_t)K::ROWS * K::NP * 8);
  static constexpr size_t bytes = oSB + r16((size_t)K::NS * K::ROWS * sizeof(T));
  // the tile's coefficients (and u_n) can be bulk copied when every tile starts
  // on a 16-byte boundary; the slots of a tile are one contiguous block
  static constexpr bool bulk_c = ((size_t)K::TE * K::MNP * 8) % 16 == 0;
  static constexpr bool bulk_s = ((size_t)K::NS * K::ROWS * sizeof(T)) % 16 == 0;
};

template <class K>
constexpr size_t elem_kernel_smem() {
  return ElemSmem<K>::bytes;
}

// host-side layout of the table blob (FP64; converted to T on upload)
template <class K>
void fill_table_blob(const double* dphi, const double* phif, const double* phi, const double* qw,
                     double* blob) {
  using L = ElemSmem<K>;
  constexpr int NP = K::NP, NPP = L::NPP;
  for (size_t i = 0; i < L::blob_elems; ++i) blob[i] = 0.0;
  for (int kk = 0; kk < K::KV; ++kk)
    for (int k = 0; k < NP; ++k) blob[L::oDphi + (size_t)kk * NPP + k] = dphi[kk * NP + k];
  for (int s = 0; s < K::NS; ++s)
    for (int k = 0; k < NP; ++k) blob[L::oPhif + (size_t)s * NPP + k] = phif[s * NP + k];
  for (int q = 0; q < K::NQ; ++q)
    for (int k = 0; k < NP; ++k) blob[L::oPhi + (size_t)q * NPP + k] = phi[q * NP + k];
  for (int q = 0; q < K::NQ; ++q) blob[L::oQw + q] = qw[q];
}

constexpr int kMbarPolls = 1 << 22;  // bound of the bulk-copy wait

// Last stage, per tile after the update: residual partial of the tile and
// its contribution to the CFL step of the next step (fused).  Tiles of
// finished ensemble instances join with active = false (partial 0).
template <class K, int LD = K::MNP>
__device__ __forceinline__ void elem_tile_tail(const StageArgs<typename K::T>& a, TimeCtl* c, int tile,
                                               double rsum, bool active, const double* sC, double* sEig,
                                               int ne, int e0, double* red, const double* sPv, double csz) {
  constexpr int M = K::M, NP = K::NP, NV = K::NV, BLOCK = K::BLOCK;
  const int tid = threadIdx.x;
  rsum = block_sum<BLOCK>(rsum, red);
  if (tid == 0) a.partials[tile] = rsum;
  if (a.fuse_cfl && active) {
    // eigenvalue at the cell mean (v = 0) and, on triangles, at the three
    // reference vertices (DGCell::computeMAXEV, DGCell.cc:1155-1207)
    for (int it = tid; it < ne * NV; it += BLOCK) {
      const int e = it / NV, v = it - (it / NV) * NV;
      const double* cc = sC + e * LD;
      double val[M];
      if (v == 0) {
#pragma unroll
        for (int j = 0; j < M; ++j) val[j] = cc[j * NP] * a.tab.phi0;
      } else {
        const double* pv = sPv + (v - 1) * NP;
#pragma unroll
        for (int j = 0; j < M; ++j) {
          double acc = 0;
#pragma unroll
          for (int k = 0; k < NP; ++k) acc += pv[k] * cc[j * NP + k];
          val[j] = acc;
        }
      }
      sEig[it] = max_eigen<K::LAW, double>(a.law, val);
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
      dtl = csz * c->cfl / (am * (2. * K::ORDER + 1.0));
    }
    dtl = block_min<BLOCK>(dtl, red);
    if (tid == 0) atomicMin(&c->dtmin_bits, (unsigned long long)__double_as_longlong(dtl));
  }
}

// Last stage, once per CTA: completion count; the last CTA advances the time
// (residual summed over the ntiles tile partials in a fixed order) and, with
// the fused CFL, finalizes the next step.
template <class K>
__device__ __forceinline__ void elem_finish(const StageArgs<typename K::T>& a, TimeCtl* c, int ntiles,
                                            double* red) {
  constexpr int BLOCK = K::BLOCK;
  __shared__ bool amLast;
  const int tid = threadIdx.x;
  if (tid == 0) {
    __threadfence();
    const unsigned v = atomicAdd(&a.gctl->blocks_done, 1u);
    amLast = (v == gridDim.x - 1);
  }
  __syncthreads();
  if (!amLast) return;
  __threadfence();
  if (a.cell_inst) {
    finalize_instances<BLOCK>(a, true, a.fuse_cfl != 0);
    return;
  }
  // single solver: residual in a fixed order (strided partial sums + tree)
  double r = 0.0;
  for (int b = tid; b < ntiles; b += BLOCK) r += ((volatile double*)a.partials)[b];
  r = block_sum<BLOCK>(r, red);
  if (tid == 0) {
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

// One tile, its inputs in shared memory: volume term, contraction with the
// reference gradients, lift of the face slots, FP64 inverse mass and stage
// combination, then the face-point traces of the new state.  sJi: J^{-1} in T
// [TE][DIM*DIM]; sDet: |J| FP64 [TE]; sU0: u_n (stages 2, 3); sS: face slots
// [NS][ROWS].  The last stage accumulates the residual into rsum.
template <class K>
__device__ __forceinline__ void elem_tile(const StageArgs<typename K::T>& a, const TimeCtl* c, int tile, int e0,
                                          int ne, const typename K::T* sT, double* sC, typename K::T* sG,
                                          const typename K::T* sJi, const double* sDet, const double* sU0,
                                          const typename K::T* sS, double& rsum) {
  using T = typename K::T;
  using L = ElemSmem<K>;
  constexpr int M = K::M, NP = K::NP, NQ = K::NQ, DIM = K::DIM;
  constexpr int NS = K::NS, KV = K::KV, LDK = K::LDK, ROWS = K::ROWS;
  constexpr int NPP = L::NPP;
  const T* sDphi = sT + L::oDphi;
  const T* sPhif = sT + L::oPhif;
  const T* sPhi = sT + L::oPhi;
  const T* sQw = sT + L::oQw;
  const int tid = threadIdx.x;

  // volume: fixed quadrature point per thread
  if (tid < K::EG * NQ) {
    const int q = tid % NQ, g = tid / NQ;
    T phi[NP];
#pragma unroll
    for (int k = 0; k < NP; ++k) phi[k] = sPhi[q * NPP + k];
    const T w = sQw[q];
    for (int e = g; e < ne; e += K::EG) {
      T U[M];
#pragma unroll
      for (int j = 0; j < M; ++j) {
        double cv[NP];
        load_vec<double, NP>(sC + (e * M + j) * NP, cv);
        T acc = 0;
#pragma unroll
        for (int k = 0; k < NP; ++k) acc += phi[k] * (T)cv[k];
        U[j] = acc;
      }
      if (!is_physical<K::LAW, T>(a.law, U)) flag_nonphysical(a.status, e0 + e);
      T F[M][DIM];
      volume_flux<K::LAW, DIM, T>(a.law, U, F);
      T J[DIM * DIM];
#pragma unroll
      for (int i = 0; i < DIM * DIM; ++i) J[i] = sJi[e * DIM * DIM + i];
      const T jw = (T)sDet[e] * w;
#pragma unroll
      for (int j = 0; j < M; ++j)
#pragma unroll
        for (int r = 0; r < DIM; ++r) {
          T acc = 0;
#pragma unroll
          for (int i = 0; i < DIM; ++i) acc += F[j][i] * J[i * DIM + r];
          sG[(e * M + j) * LDK + q * DIM + r] = acc * jw;
        }
    }
  }
  __syncthreads();

  // contraction + lift + inverse mass + stage combination, one row per thread
  const int row = tid;
  if (row < ne * M) {
    T acc[NPP];
#pragma unroll
    for (int k = 0; k < NPP; ++k) acc[k] = 0;
    const T* g = sG + row * LDK;
#pragma unroll 4
    for (int kk = 0; kk < KV; ++kk) {
      const T gv = g[kk];
      T d[NPP];
      load_vec<T, NPP>(sDphi + kk * NPP, d);
#pragma unroll
      for (int k = 0; k < NPP; ++k) acc[k] += gv * d[k];
    }
#pragma unroll 4
    for (int s = 0; s < NS; ++s) {
      const T sv = sS[s * ROWS + row];
      T p[NPP];
      load_vec<T, NPP>(sPhif + s * NPP, p);
#pragma unroll
      for (int k = 0; k < NPP; ++k) acc[k] += sv * p[k];
    }
    const size_t gbase = ((size_t)e0 * M + row) * NP;
    if (a.stage == 0) {
#pragma unroll
      for (int k = 0; k < NP; ++k) a.Cout[gbase + k] = (double)acc[k];
    } else {
      const int e = row / M;
      // FP64 update in the reference's operation order (dt/|J| in FP64)
      const double dtj = c->dt / sDet[e];
      double* crow = sC + row * NP;
      double cv[NP];
      load_vec<double, NP>(crow, cv);
#pragma unroll
      for (int k = 0; k < NP; ++k) {
        const double r = (double)acc[k];
        double out;
        if (a.stage == 1) {
          a.U0out[gbase + k] = cv[k];
          out = cv[k] + r * dtj;
        } else if (a.stage == 2) {
          out = 0.25 * (cv[k] + r * dtj + 3. * sU0[row * NP + k]);
        } else {
          const double u0 = sU0[row * NP + k];
          out = (2.0 * (cv[k] + r * dtj) + u0) / 3.0;
          const double dd = out - u0;
          rsum += dd * dd;
        }
        crow[k] = out;
        a.Cout[gbase + k] = out;
      }
      // face-point traces of the new state for the next stage's face kernel
      T o[NP];
#pragma unroll
      for (int k = 0; k < NP; ++k) o[k] = (T)crow[k];
      T* tr = a.tr + (size_t)tile * NS * ROWS + row;
#pragma unroll 4
      for (int s = 0; s < NS; ++s) {
        T p[NPP];
        load_vec<T, NPP>(sPhif + s * NPP, p);
        T t = 0;
#pragma unroll
        for (int k = 0; k < NP; ++k) t += p[k] * o[k];
        tr[(size_t)s * ROWS] = t;
      }
    }
  }
}

// geometry of a tile inside the ElemSmem geometry area: |J| FP64 [TE], CFL
// eigenvalues FP64 [TE][NV], J^{-1} T [TE][DIM*DIM]
template <class K>
struct GeoArea {
  static constexpr size_t oDet = 0;
  static constexpr size_t oEig = 8 * (size_t)K::TE;
  static constexpr size_t oJi = oEig + 8 * (size_t)K::TE * K::NV;
};

// One CTA per tile of TE cells.  Used where the persistent kernel's 16-byte
// alignment conditions do not hold.
template <class K>
__global__ void __launch_bounds__(K::BLOCK) elem_kernel(const __grid_constant__ StageArgs<typename K::T> a) {
  using T = typename K::T;
  using L = ElemSmem<K>;
  using G = GeoArea<K>;
  constexpr int MNP = K::MNP, NS = K::NS, DIM = K::DIM, TE = K::TE, BLOCK = K::BLOCK, ROWS = K::ROWS;
  if (a.gctl->done) return;
  extern __shared__ __align__(128) unsigned char smem_raw[];
  T* sT = reinterpret_cast<T*>(smem_raw);
  double* sC = reinterpret_cast<double*>(smem_raw + L::oCB);
  T* sG = reinterpret_cast<T*>(smem_raw + L::oGB);
  double* sDet = reinterpret_cast<double*>(smem_raw + L::oJB + G::oDet);
  double* sEig = reinterpret_cast<double*>(smem_raw + L::oJB + G::oEig);
  T* sJi = reinterpret_cast<T*>(smem_raw + L::oJB + G::oJi);
  double* sU0 = reinterpret_cast<double*>(smem_raw + L::oUB);
  T* sS = reinterpret_cast<T*>(smem_raw + L::oSB);
  __shared__ __align__(8) uint64_t bar;
  __shared__ double red[BLOCK / 32];
  __shared__ int s_fail;

  const int tid = threadIdx.x;
  const int tile = blockIdx.x;
  const int e0 = tile * TE;
  TimeCtl* c = a.ctl;
  int eend = a.mesh.E;
  if (a.cell_inst) {  // ensemble: the tile belongs to one instance
    const int inst = a.cell_inst[e0];
    c = a.ctl + inst;
    eend = a.inst_end[inst];
    if (c->done) {
      if (a.stage == 3) {
        elem_tile_tail<K>(a, c, tile, 0.0, false, nullptr, nullptr, 0, e0, red, nullptr, 0.0);
        elem_finish<K>(a, c, gridDim.x, red);
      }
      return;
    }
  }
  const int ne = min(TE, eend - e0);
  const uint32_t c_bytes = (uint32_t)(((size_t)ne * MNP * 8 + 15) / 16 * 16);

  if (tid == 0) {
    s_fail = 0;
    mbar_init(&bar, 1);
  }
  __syncthreads();
  // one mbarrier for every input of the tile: tables, state, u_n (stages 2
  // and 3), face slots; the geometry is loaded by the threads meanwhile
  const bool need_u0 = a.stage >= 2;
  constexpr uint32_t s_bytes = (uint32_t)(NS * ROWS * sizeof(T));
  const T* slot_src = a.slots + (size_t)tile * NS * ROWS;
  if (tid == 0) {
    uint32_t tx = (uint32_t)L::blob_bytes;
    if constexpr (L::bulk_c) tx += c_bytes * (need_u0 ? 2u : 1u);
    if constexpr (L::bulk_s) tx += s_bytes;
    mbar_arrive_expect_tx(&bar, tx);
    bulk_g2s(sT, a.tab.blob, (uint32_t)L::blob_bytes, &bar);
    if constexpr (L::bulk_c) {
      bulk_g2s(sC, a.C + (size_t)e0 * MNP, c_bytes, &bar);
      if (need_u0) bulk_g2s(sU0, a.U0 + (size_t)e0 * MNP, c_bytes, &bar);
    }
    if constexpr (L::bulk_s) bulk_g2s(sS, slot_src, s_bytes, &bar);
  }
  if constexpr (!L::bulk_c) {
    const double* src = a.C + (size_t)e0 * MNP;
    for (int i = tid; i < ne * MNP; i += BLOCK) sC[i] = src[i];
    if (need_u0) {
      const double* u0 = a.U0 + (size_t)e0 * MNP;
      for (int i = tid; i < ne * MNP; i += BLOCK) sU0[i] = u0[i];
    }
  }
  if constexpr (!L::bulk_s) {
    for (int i = tid; i < NS * ROWS; i += BLOCK) sS[i] = slot_src[i];
  }
  const bool p0_mark = a.p0 && tid < ne && a.bad[e0 + tid];
  // the last stage's CFL inputs, fetched while the copies fly
  __shared__ double sPv[(K::NV - 1) * K::NP + 1];
  double csz = 0.0;
  if (a.stage == 3 && a.fuse_cfl) {
    if (tid < ne) csz = a.mesh.csize[e0 + tid];
    for (int i = tid; i < (K::NV - 1) * K::NP; i += BLOCK) sPv[i] = a.tab.phiv[i];
  }
  for (int i = tid; i < ne * DIM * DIM; i += BLOCK) sJi[i] = a.mesh.jinv[(size_t)e0 * DIM * DIM + i];
  for (int i = tid; i < ne; i += BLOCK) sDet[i] = a.mesh.detjd[e0 + i];
  if (tid == 0 && !mbar_wait(&bar, 0, kMbarPolls)) {
    // record the failure, then wait once more (bounded) for the copies this
    // CTA issued before its shared memory is released
    s_fail = 1;
    atomicAdd(&a.status->timeouts, 1);
    mbar_wait(&bar, 0, kMbarPolls);
  }
  __syncthreads();
  if (s_fail) return;
  // P0 fallback: the face passes marked cells and zeroed their modes; the
  // marks of this tile's cells are consumed here
  if (p0_mark) a.bad[e0 + tid] = 0;
  if (a.p0 && blockIdx.x == 0 && tid == 0) a.status->stage_bad = 0;

  double rsum = 0.0;
  elem_tile<K>(a, c, tile, e0, ne, sT, sC, sG, sJi, sDet, sU0, sS, rsum);
  if (a.stage != 3) return;
  __syncthreads();
  elem_tile_tail<K>(a, c, tile, rsum, true, sC, sEig, ne, e0, red, sPv, csz);
  elem_finish<K>(a, c, gridDim.x, red);
}

}  // namespace dgp
