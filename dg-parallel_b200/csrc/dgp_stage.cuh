// Fused stage kernel: one CTA per tile of TE cells computes every face flux
// that touches the tile, the volume term, the lift of the face slots, the
// diagonal inverse mass and the SSP-RK3 stage combination, with the last
// stage's residual and CFL reductions fused in.
//
// The tile reads the stage input rows of its own cells and of its halo (the
// cells across its faces, periodic partners included), staged into shared
// memory by 16-byte asynchronous copies (the tables by one bulk copy on an
// mbarrier); face-point traces and face slots live in shared memory only.  A face between two tiles is evaluated by both,
// from identical inputs with identical arithmetic, so each side receives the
// same flux it would get from a separate face pass.  The stage writes a
// different buffer from the one it reads (u_n -> u1 -> u2 -> u_n in place,
// own rows only), so no tile reads a row another tile is writing.
//
// Replaces DGBoundaryCell::computeBoundaryContributions (DGCell.cc:639-732),
// DGCell::computeVolumeContribution (DGCell.cc:184-249) and the
// RungeKuttaTVD3::advanceInTime update loops (TimeIntegrator.cc:838-990).
//
// P0 fallback (DGCell::setToZero, DGCell.cc:785-811; DGAnalysis.cc:392-417,
// and the correction inside DGCell::computeVolumeContribution,
// DGCell.cc:197-221): a cell is marked when its value at any of its volume
// quadrature points or its trace at any of its face points is not physical.
// Each tile checks its own cells at their face points during the face pass,
// at their volume points after it, and its halo cells at all of theirs, so it
// knows every mark that reaches its faces without a grid-wide pass; a tile
// that sees one zeroes the modes k >= 1 of the marked rows (own and halo, in
// shared memory) and evaluates its faces again.  Marks of stage 1 persist
// into u_n for stages 2 and 3 (bad[e]).
#pragma once

#include "dgp_elem.cuh"
#include "dgp_umma.cuh"

namespace dgp {

// row stride (in elements) of staged rows: a whole, odd number of `unit`-byte
// vectors, so that rows stay aligned for vector loads and threads reading
// different rows hit different banks
constexpr int padded_stride(int n, int esize, int unit) {
  const int per = unit / esize;                  // elements per vector unit
  const int s = (n + per - 1) / per * per;       // whole units
  return ((s / per) % 2 == 1) ? s : s + per;     // odd number of units
}

template <class K, bool TC = false>
struct FusedSmem {
  using T = typename K::T;
  using L = ElemSmem<K>;
  static constexpr size_t r16(size_t n) { return (n + 15) / 16 * 16; }
  static constexpr bool MIXED = sizeof(T) == 4;
  // FP64 rows: 16-byte units (2 doubles); FP32 trace rows: 8-byte units (2 floats)
  static constexpr int RS = padded_stride(K::MNP, 8, 16);
  static constexpr int RSF = padded_stride(K::MNP, 4, 8);
  static constexpr int RST = MIXED ? RSF : RS;  // stride of the rows the traces read
  // The mixed form's volume contraction on the tensor cores (tcgen05, TF32
  // with split operands) where TC asks for it: one M = 128 MMA tile covers
  // the tile's rows, N = 16 the modes, K = KPAD the (direction, point) pairs
  // padded to whole k-steps.  UMMA_OK: the shape allows it.
  static constexpr bool UMMA_OK = MIXED && K::BLOCK == 128 && K::ROWS <= 128 && K::NP <= 16;
  static constexpr bool UMMA = UMMA_OK && TC;
  static constexpr int KPAD = (K::KV + 7) / 8 * 8;
  static constexpr int UN = 16;
  static constexpr size_t a_bytes = (size_t)128 * KPAD * 4;  // one split part of A
  static constexpr size_t b_bytes = (size_t)UN * KPAD * 4;   // one split part of B
  // the fused kernel's table blob: the element kernel's tables, then (tensor
  // cores) B = the reference gradients as TF32 high and low parts in the MMA layout
  static constexpr size_t oBhi = L::blob_bytes;
  static constexpr size_t oBlo = oBhi + b_bytes;
  static constexpr size_t fblob_bytes = L::blob_bytes + (UMMA_OK ? 2 * b_bytes : 0);
  static constexpr size_t fblob_elems = fblob_bytes / sizeof(T);
  // table blob | own rows FP64 [TE][RS] | face slots T [NS][ROWS] | geometry |
  // own rows FP32 [TE][RSF] (mixed) |
  // union { halo rows FP64 [nh][RS] + FP32 [nh][RSF] (face pass),
  //         G T [ROWS][LDK] or the MMA's A high and low parts (volume) }
  static constexpr size_t oC = r16(fblob_bytes);
  static constexpr size_t oS = oC + r16((size_t)K::TE * RS * 8);
  static constexpr size_t oJ = oS + r16((size_t)K::NS * K::ROWS * sizeof(T));
  static constexpr size_t oCf = oJ + r16(8 * ((size_t)K::TE * L::DD + (size_t)K::TE * K::NV));
  static constexpr size_t oX = oCf + (MIXED ? r16((size_t)K::TE * RSF * 4) : 0);
  static constexpr size_t g_bytes = UMMA ? 2 * a_bytes : r16((size_t)K::ROWS * K::LDK * sizeof(T));
  static constexpr size_t halo_bytes(int nh) { return r16((size_t)nh * RS * 8) + (MIXED ? r16((size_t)nh * RSF * 4) : 0); }
  static constexpr size_t bytes(int nh) { return oX + (halo_bytes(nh) > g_bytes ? halo_bytes(nh) : g_bytes); }
  // rows are bulk copied one by one when a row is a whole number of 16-byte units
  static constexpr bool bulk_rows = (K::MNP * 8) % 16 == 0;
  static constexpr int HMAX = K::TE * K::NLF;  // a tile's halo never exceeds one cell per own face
  // at most 128 registers a thread, so that 64k registers hold 512 threads
  static constexpr int MIN_BLOCKS = 65536 / (K::BLOCK * 128) > 0 ? 65536 / (K::BLOCK * 128) : 1;
};

// host-side table blob of the fused kernel: the element kernel's layout with
// the reference-gradient rows in the order kk = r * NQ + q of its G rows
template <class K>
void fill_fused_blob(const double* dphi, const double* phif, const double* phi, const double* qw, double* blob) {
  using L = ElemSmem<K>;
  constexpr int NP = K::NP, NPP = L::NPP;
  using FS = FusedSmem<K>;
  fill_table_blob<K>(dphi, phif, phi, qw, blob);
  for (int q = 0; q < K::NQ; ++q)
    for (int r = 0; r < K::DIM; ++r)
      for (int k = 0; k < NP; ++k)
        blob[L::oDphi + (size_t)(r * K::NQ + q) * NPP + k] = dphi[(q * K::DIM + r) * NP + k];
  if constexpr (FS::UMMA_OK) {
    // B[n][kk] = dphi of row kk = r * NQ + q at mode n, as FP32 split into
    // TF32 high and low parts, zero beyond the modes and the rows
    double* bhi = blob + FS::oBhi / 4;
    double* blo = blob + FS::oBlo / 4;
    for (int n = 0; n < FS::UN; ++n)
      for (int kk = 0; kk < FS::KPAD; ++kk) {
        float v = 0.0f;
        if (kk < K::KV && n < NP) {
          const int r = kk / K::NQ, q = kk - r * K::NQ;
          v = (float)dphi[(q * K::DIM + r) * NP + n];
        }
        const float hi = host_tf32(v), lo = host_tf32(v - hi);
        const uint32_t o = umma_off(n, kk, FS::KPAD) / 4;
        bhi[o] = hi;
        blo[o] = lo;
      }
  }
}

// trace of one row at a face point: U[j] = sum_k phi[k] row[j][k] in T, in the
// order of the volume interpolation (the rows are the FP64 state, or its FP32
// copy in the mixed form)
template <class K>
__device__ __forceinline__ void row_trace(const typename K::T* __restrict__ row, const typename K::T* phi,
                                          typename K::T* U) {
  using T = typename K::T;
  constexpr int NP = K::NP;
#pragma unroll
  for (int j = 0; j < K::M; ++j) {
    T cv[NP];
    load_vec<T, NP>(row + j * NP, cv);
    T acc = 0;
#pragma unroll
    for (int k = 0; k < NP; ++k) acc += phi[k] * cv[k];
    U[j] = acc;
  }
}

// the periodic partner's trace, its basis values at the mirrored point read
// from global memory
template <class K>
__device__ __forceinline__ void row_trace_g(const typename K::T* __restrict__ row,
                                            const typename K::T* __restrict__ phi, typename K::T* U) {
  using T = typename K::T;
  constexpr int NP = K::NP;
#pragma unroll
  for (int j = 0; j < K::M; ++j) {
    T acc = 0;
#pragma unroll
    for (int k = 0; k < NP; ++k) acc += __ldg(phi + k) * row[j * NP + k];
    U[j] = acc;
  }
}

struct FusedTile {
  int e0, ne, nh, f0, nf;
};

// Rounding probe (error decomposition of the mixed form): with RND, the terms
// whose bit is set in the mask are rounded to FP32 inside the FP64 kernel.
// Bits: geometry (J^{-1}, |J| w, face normals, |J_f| w), face-point traces,
// volume-point values, volume flux products G, face slots, the contraction's
// result, the reference tables.
enum : int {
  kRndGeometry = 1, kRndTraces = 2, kRndVolumeValues = 4, kRndVolumeFlux = 8, kRndSlots = 16,
  kRndContraction = 32, kRndTables = 64
};

template <bool RND, typename T>
__device__ __forceinline__ T probe(T x, int mask, int bit) {
  if constexpr (RND) {
    if (mask & bit) return (T)(float)x;
  }
  return x;
}

// the one configuration the probe is built for: the FP64 P3 Euler vortex
// workload with Roe flux and 128-thread tiles
template <class K>
constexpr bool probe_built() {
  return sizeof(typename K::T) == 8 && K::LAW == DGP_LAW_EULER2D && K::FLUX == DGP_FLUX_ROE && K::DIM == 2 &&
         K::ORDER == 3 && K::BLOCK == 128;
}

constexpr int kFinalizeThreads = 1024;

// Last stage, per tile: the residual partial of the tile and the smallest CFL
// step of its cells (DGCell::computeMAXEV, DGCell.cc:1155-1207: eigenvalue at
// the mean and, on triangles, at the three reference vertices), written to
// partials[tile] and partials[ntiles + tile] for stage_finalize_kernel.
template <class K, int LD>
__device__ __forceinline__ void fused_tile_tail(const StageArgs<typename K::T>& a, const TimeCtl* c, int tile,
                                                double rsum, const double* sC, double* sEig, int ne, double* red,
                                                const double* sPv, double csz) {
  constexpr int M = K::M, NP = K::NP, NV = K::NV, BLOCK = K::BLOCK;
  const int tid = threadIdx.x;
  const int ntiles = (a.mesh.E + K::TE - 1) / K::TE;
  rsum = block_sum<BLOCK>(rsum, red);
  if (tid == 0) a.partials[tile] = rsum;
  if (!a.fuse_cfl) return;
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
  if (tid == 0) a.partials[ntiles + tile] = dtl;
}

// a tile that computes nothing in the last stage (its instance has finished,
// or its copies gave up) leaves neutral partials
template <class K>
__device__ __forceinline__ void fused_tile_idle(const StageArgs<typename K::T>& a, int tile) {
  if (a.stage != 3 || threadIdx.x != 0) return;
  const int ntiles = (a.mesh.E + K::TE - 1) / K::TE;
  a.partials[tile] = 0.0;
  a.partials[ntiles + tile] = 1e300;
}

// One face point of a tile face: traces of both sides from the staged rows,
// the law's numerical, periodic or boundary flux, and the slots of the own
// sides.  CHECK: count non-physical own traces and, with the P0 fallback on,
// mark their cells (returns true when it marked one).
template <class K, bool ENS, bool CHECK, bool RND = false>
__device__ __forceinline__ bool fused_face_point(const StageArgs<typename K::T>& a, const TimeCtl* c, int inst,
                                                 const FusedTile& ft, int tf, int q, const typename K::T* sPhif,
                                                 const typename K::T* s_fqw, const int* s_qmap,
                                                 const typename K::T* sC, const typename K::T* sH,
                                                 typename K::T* sS, unsigned char* s_mark) {
  using T = typename K::T;
  using L = ElemSmem<K>;
  constexpr int M = K::M, NQF = K::NQF, DIM = K::DIM, TE = K::TE, ROWS = K::ROWS;
  constexpr int NPP = L::NPP, RST = FusedSmem<K>::RST;
  const int side = a.tm.tf_side[tf], code = a.tm.tf_code[tf];
  const int lL = side & 0xffff, hi = side >> 16;
  const int lfL = code & 15, lfR = (code >> 4) & 15, perm = (code >> 8) & 15;
  const bool ownL = (code >> 12) & 1, ownR = (code >> 13) & 1;
  const int kind = (code >> 14) & 3;
  auto rowp = [&](int l) -> const T* { return l < TE ? sC + l * RST : sH + (l - TE) * RST; };
  T n[DIM];
#pragma unroll
  for (int i = 0; i < DIM; ++i) n[i] = probe<RND, T>((T)a.tm.tf_nrm[(size_t)tf * DIM + i], a.round_mask, kRndGeometry);
  const T jw = probe<RND, T>((T)a.tm.tf_fj[tf] * s_fqw[q], a.round_mask, kRndGeometry);
  bool marked = false;
  T UL[M], UR[M], flux[M];
  row_trace<K>(rowp(lL), sPhif + (lfL * NQF + q) * NPP, UL);
  if constexpr (RND) {
#pragma unroll
    for (int j = 0; j < M; ++j) UL[j] = probe<RND, T>(UL[j], a.round_mask, kRndTraces);
  }
  if (CHECK && ownL && !is_physical<K::LAW, T>(a.law, UL)) {
    flag_nonphysical(a.status, ft.e0 + lL);
    if (a.p0) {
      s_mark[lL] = 1;
      marked = true;
    }
  }
  int qR = 0;
  if (kind == 0) {
    const int lR = hi - 1;
    qR = s_qmap[perm * NQF + q];
    row_trace<K>(rowp(lR), sPhif + (lfR * NQF + qR) * NPP, UR);
    if constexpr (RND) {
#pragma unroll
      for (int j = 0; j < M; ++j) UR[j] = probe<RND, T>(UR[j], a.round_mask, kRndTraces);
    }
    if (CHECK && ownR && !is_physical<K::LAW, T>(a.law, UR)) {
      flag_nonphysical(a.status, ft.e0 + lR);
      if (a.p0) {
        s_mark[lR] = 1;
        marked = true;
      }
    }
    numerical_flux<K::LAW, K::FLUX, DIM, T>(a.law, n, UL, UR, flux);
  } else if (kind == 2) {
    // periodic edge (DGCell.cc:687-705): the partner cell's trace at the
    // mirrored point through the numerical flux; only the left cell gets it
    const int b = a.tm.tf_bnd[tf];
    row_trace_g<K>(rowp(hi - 1), a.mesh.bpphi + ((size_t)b * NQF + q) * K::NP, UR);
    numerical_flux<K::LAW, K::FLUX, DIM, T>(a.law, n, UL, UR, flux);
  } else {
    const int b = a.tm.tf_bnd[tf];
    const double* x = a.mesh.bpts + ((size_t)b * NQF + q) * 3;
    const double time = __fma_rn(a.stage_time_factor, c->dt, c->t);
    if constexpr (ENS)
      boundary_flux<K::LAW, K::FLUX, DIM, T>(a.laws[inst], a.mesh.bbid[b], n, x, time, UL, flux);
    else
      boundary_flux<K::LAW, K::FLUX, DIM, T>(a.law, a.mesh.bbid[b], n, x, time, UL, flux);
  }
  if (ownL) {
    T* dst = sS + (lfL * NQF + q) * ROWS + lL * M;
#pragma unroll
    for (int j = 0; j < M; ++j) dst[j] = probe<RND, T>(-flux[j] * jw, a.round_mask, kRndSlots);
  }
  if (kind == 0 && ownR) {
    T* dst = sS + (lfR * NQF + qR) * ROWS + (hi - 1) * M;
#pragma unroll
    for (int j = 0; j < M; ++j) dst[j] = probe<RND, T>(flux[j] * jw, a.round_mask, kRndSlots);
  }
  return marked;
}

template <class K, bool ENS, bool CHECK, bool RND = false>
__device__ __forceinline__ bool fused_face_pass(const StageArgs<typename K::T>& a, const TimeCtl* c, int inst,
                                                const FusedTile& ft, const typename K::T* sPhif,
                                                const typename K::T* s_fqw, const int* s_qmap,
                                                const typename K::T* sC, const typename K::T* sH,
                                                typename K::T* sS, unsigned char* s_mark) {
  constexpr int NQF = K::NQF;
  bool mk = false;
  for (int t = threadIdx.x; t < ft.nf * NQF; t += K::BLOCK) {
    const int f = t / NQF, q = t - f * NQF;
    mk |= fused_face_point<K, ENS, CHECK, RND>(a, c, inst, ft, ft.f0 + f, q, sPhif, s_fqw, s_qmap, sC, sH, sS, s_mark);
  }
  return mk;
}

// The P0 check of one staged cell: true when its value at a volume
// quadrature point or (halo cell, e < 0) its trace at a face point is not
// physical; an own cell's non-physical volume points are counted.  A cell
// whose modes k >= 1 cannot move a field past the limit anywhere
// (physical_bound, from the largest basis values phimax, in shared memory) is
// cleared without evaluating its points.
template <class K>
__device__ __forceinline__ bool p0_cell_bad(const StageArgs<typename K::T>& a, const typename K::T* row,
                                            const typename K::T* sPhi, const typename K::T* sPhif,
                                            const typename K::T* phimax, int e) {
  using T = typename K::T;
  constexpr int M = K::M, NP = K::NP;
  constexpr int NPP = ElemSmem<K>::NPP;
  T mean[M], B[M];
#pragma unroll
  for (int j = 0; j < M; ++j) {
    mean[j] = row[j * NP] * sPhi[0];
    T b = 0;
#pragma unroll
    for (int k = 1; k < NP; ++k) b += fabs(row[j * NP + k]) * phimax[k];
    B[j] = b;
  }
  if (physical_bound<K::LAW, T>(a.law, mean, B)) return false;
  bool bad = false;
  const int np = e >= 0 ? K::NQ : K::NQ + K::NS;
#pragma unroll 1
  for (int p = 0; p < np; ++p) {
    T U[M];
    row_trace<K>(row, p < K::NQ ? sPhi + p * NPP : sPhif + (p - K::NQ) * NPP, U);
    if (!is_physical<K::LAW, T>(a.law, U)) {
      bad = true;
      if (e >= 0) flag_nonphysical(a.status, e);
    }
  }
  return bad;
}

template <class K, bool ENS, bool TC = false, bool RND = false>
__global__ void __launch_bounds__(K::BLOCK, FusedSmem<K>::MIN_BLOCKS)
    stage_kernel(const __grid_constant__ StageArgs<typename K::T> a) {
  using T = typename K::T;
  using L = ElemSmem<K>;
  using FS = FusedSmem<K, TC>;
  using G = GeoArea<K>;
  constexpr int M = K::M, NP = K::NP, MNP = K::MNP, NQ = K::NQ, NS = K::NS, NQF = K::NQF, DIM = K::DIM;
  constexpr int TE = K::TE, BLOCK = K::BLOCK, ROWS = K::ROWS, KV = K::KV, LDK = K::LDK, NPP = L::NPP;
  constexpr int RS = FS::RS, RSF = FS::RSF, RST = FS::RST;
  if (a.gctl->done) return;
  extern __shared__ __align__(128) unsigned char smem_raw[];
  T* sT = reinterpret_cast<T*>(smem_raw);
  const T* sDphi = sT + L::oDphi;
  const T* sPhif = sT + L::oPhif;
  const T* sPhi = sT + L::oPhi;
  const T* sQw = sT + L::oQw;
  double* sC = reinterpret_cast<double*>(smem_raw + FS::oC);
  T* sS = reinterpret_cast<T*>(smem_raw + FS::oS);
  double* sDet = reinterpret_cast<double*>(smem_raw + FS::oJ + G::oDet);
  double* sEig = reinterpret_cast<double*>(smem_raw + FS::oJ + G::oEig);
  T* sJi = reinterpret_cast<T*>(smem_raw + FS::oJ + G::oJi);
  double* sH = reinterpret_cast<double*>(smem_raw + FS::oX);
  T* sG = reinterpret_cast<T*>(smem_raw + FS::oX);
  __shared__ __align__(8) uint64_t bar;
  __shared__ double red[BLOCK / 32];
  __shared__ int s_fail;
  __shared__ T s_fqw[NQF];
  __shared__ int s_qmap[K::NPERM * NQF];
  __shared__ unsigned char s_mark[TE + FS::HMAX];
  __shared__ T s_phimax[NP];
  __shared__ double sPv[(K::NV - 1) * NP + 1];
  __shared__ __align__(8) uint64_t mma_bar;
  __shared__ uint32_t s_tmem;

  const int tid = threadIdx.x;
  const int tile = blockIdx.x;
  FusedTile ft;
  ft.e0 = tile * TE;
  TimeCtl* c = a.ctl;
  int inst = 0, eend = a.mesh.E;
  if constexpr (ENS) {  // the tile belongs to one instance
    inst = a.cell_inst[ft.e0];
    c = a.ctl + inst;
    eend = a.inst_end[inst];
    if (c->done) {
      if (a.stage == 3) {
        fused_tile_idle<K>(a, tile);
      }
      return;
    }
  }
  ft.ne = min(TE, eend - ft.e0);
  const int h0 = a.tm.th_off[tile];
  ft.nh = a.tm.th_off[tile + 1] - h0;
  ft.f0 = a.tm.tf_off[tile];
  ft.nf = a.tm.tf_off[tile + 1] - ft.f0;
  // rows the traces and the volume interpolation read: the FP64 rows, or
  // their FP32 copies (made once per tile) in the mixed form
  T* sCt;
  T* sHt;
  if constexpr (FS::MIXED) {
    sCt = reinterpret_cast<T*>(smem_raw + FS::oCf);
    sHt = reinterpret_cast<T*>(smem_raw + FS::oX + FS::r16((size_t)ft.nh * RS * 8));
  } else {
    sCt = reinterpret_cast<T*>(sC);
    sHt = reinterpret_cast<T*>(sH);
  }

  if (tid == 0) {
    s_fail = 0;
    mbar_init(&bar, 1);
    if constexpr (FS::UMMA) mbar_init(&mma_bar, 1);
  }
  for (int i = tid; i < NQF; i += BLOCK) s_fqw[i] = a.tab.fqw[i];
  if (a.p0)
    for (int i = tid; i < NP; i += BLOCK) s_phimax[i] = a.tab.phimax[i];
  for (int i = tid; i < K::NPERM * NQF; i += BLOCK) s_qmap[i] = a.tab.qmap[i];
  for (int i = tid; i < TE + ft.nh; i += BLOCK) s_mark[i] = 0;
  if constexpr (FS::UMMA) {
    // 32 columns of tensor memory for D, allocated while the copies fly and
    // freed on every way out of the kernel
    if (tid < 32) tmem_alloc(&s_tmem, 32);
    tc_fence_before();
  }
  __syncthreads();
  // the tables: one bulk copy on the mbarrier (a bound on its first wait
  // counts the polls from the copy's issue)
  if (tid == 0) {
    mbar_arrive_expect_tx(&bar, (uint32_t)FS::fblob_bytes);
    bulk_g2s(sT, a.tab.blob, (uint32_t)FS::fblob_bytes, &bar);
    if (a.mbar_polls > 0 && !mbar_test_polls(&bar, 0, a.mbar_polls)) s_fail = 1;
  }
  // the rows (own, then halo) at the padded stride: 16-byte asynchronous
  // copies spread over every thread, all in flight at once (many small bulk
  // copies would queue on the SM's one bulk-copy engine)
  if constexpr (FS::bulk_rows) {
    constexpr int CH = MNP * 8 / 16;  // 16-byte chunks a row
    for (int i = tid; i < (ft.ne + ft.nh) * CH; i += BLOCK) {
      const int l = i / CH, w = i - l * CH;
      const double* src = (l < ft.ne ? a.C + (size_t)(ft.e0 + l) * MNP
                                     : a.C + (size_t)a.tm.th_cell[h0 + l - ft.ne] * MNP) + 2 * w;
      double* dst = (l < ft.ne ? sC + (size_t)l * RS : sH + (size_t)(l - ft.ne) * RS) + 2 * w;
      cp_async16(dst, src);
    }
  }
  if constexpr (!FS::bulk_rows) {
    for (int i = tid; i < ft.ne * MNP; i += BLOCK) {
      const int l = i / MNP;
      sC[(size_t)l * RS + (i - l * MNP)] = a.C[(size_t)ft.e0 * MNP + i];
    }
    for (int i = tid; i < ft.nh * MNP; i += BLOCK) {
      const int h = i / MNP;
      sH[(size_t)h * RS + (i - h * MNP)] = a.C[(size_t)a.tm.th_cell[h0 + h] * MNP + (i - h * MNP)];
    }
  }
  double csz = 0.0;
  if (a.stage == 3 && a.fuse_cfl) {
    if (tid < ft.ne) csz = a.mesh.csize[ft.e0 + tid];
    for (int i = tid; i < (K::NV - 1) * NP; i += BLOCK) sPv[i] = a.tab.phiv[i];
  }
  for (int i = tid; i < ft.ne * DIM * DIM; i += BLOCK) sJi[i] = a.mesh.jinv[(size_t)ft.e0 * DIM * DIM + i];
  for (int i = tid; i < ft.ne; i += BLOCK) sDet[i] = a.mesh.detjd[ft.e0 + i];
  if constexpr (FS::bulk_rows) cp_async_wait_all();
  if (tid == 0 && (s_fail || !mbar_wait(&bar, 0, kMbarPolls))) {
    // record the failure, then wait once more (bounded) for the copies this
    // CTA issued before its shared memory is released
    s_fail = 1;
    atomicAdd(&a.status->timeouts, 1);
    mbar_wait(&bar, 0, kMbarPolls);
  }
  __syncthreads();
  if (s_fail) {
    // the tile's output is not written; the last stage still leaves neutral
    // partials for the finalize
    if (a.stage == 3) {
      fused_tile_idle<K>(a, tile);
    }
    if constexpr (FS::UMMA) {
      tc_fence_after();
      if (tid < 32) tmem_dealloc(s_tmem, 32);
    }
    return;
  }
  if constexpr (FS::MIXED) {
    // one conversion of every staged row to the arithmetic type
    for (int i = tid; i < (ft.ne + ft.nh) * MNP; i += BLOCK) {
      const int l = i / MNP, k = i - l * MNP;
      if (l < ft.ne)
        sCt[(size_t)l * RSF + k] = (T)sC[(size_t)l * RS + k];
      else
        sHt[(size_t)(l - ft.ne) * RSF + k] = (T)sH[(size_t)(l - ft.ne) * RS + k];
    }
    __syncthreads();
  }

  // ---- faces: every face point of the tile's faces into the slots --------
  if constexpr (RND) {
    if (a.round_mask & kRndTables) {
      for (int i = tid; i < (int)(L::blob_bytes / sizeof(T)); i += BLOCK) sT[i] = (T)(float)sT[i];
      __syncthreads();
    }
  }
  bool mk = fused_face_pass<K, ENS, true, RND>(a, c, inst, ft, sPhif, s_fqw, s_qmap, sCt, sHt, sS, s_mark);
  if (a.p0) {
    // the face pass marked the own cells with a non-physical trace; also
    // marked: own cells with a non-physical value at a volume quadrature
    // point (the correction inside DGCell::computeVolumeContribution,
    // DGCell.cc:197-221) and halo cells with one at a volume or a face point
    // (what their own tiles find)
    for (int l = tid; l < TE + ft.nh; l += BLOCK) {
      if (l >= ft.ne && l < TE) continue;
      const T* row = l < TE ? sCt + l * RST : sHt + (size_t)(l - TE) * RST;
      if (p0_cell_bad<K>(a, row, sPhi, sPhif, s_phimax, l < TE ? ft.e0 + l : -1)) {
        s_mark[l] = 1;
        mk = true;
      }
    }
    if (__syncthreads_or(mk)) {
      // P0: marked rows drop to their means, then the faces again
      for (int i = tid; i < (TE + ft.nh) * M; i += BLOCK) {
        const int l = i / M, j = i - l * M;
        if (l < TE && l >= ft.ne) continue;
        if (!s_mark[l]) continue;
        T* row = (l < TE ? sCt + l * RST : sHt + (size_t)(l - TE) * RST) + j * NP;
        for (int k = 1; k < NP; ++k) row[k] = (T)0;
        if constexpr (FS::MIXED) {
          if (l < TE)
            for (int k = 1; k < NP; ++k) sC[(size_t)l * RS + j * NP + k] = 0.0;
        }
      }
      __syncthreads();
      fused_face_pass<K, ENS, false, RND>(a, c, inst, ft, sPhif, s_fqw, s_qmap, sCt, sHt, sS, s_mark);
    }
    // stage 1: the marks persist into u_n for stages 2 and 3
    if (a.stage == 1)
      for (int l = tid; l < ft.ne; l += BLOCK) a.bad[ft.e0 + l] = s_mark[l];
  }
  __syncthreads();  // halo rows are dead from here on: G takes their place

  // ---- volume: thread (q, g) owns quadrature point q ------------------------
  if (tid < K::EG * NQ) {
    const int q = tid % NQ, g = tid / NQ;
    T phi[NP];
#pragma unroll
    for (int k = 0; k < NP; ++k) phi[k] = sPhi[q * NPP + k];
    const T w = sQw[q];
    for (int e = g; e < ft.ne; e += K::EG) {
      T U[M];
#pragma unroll
      for (int j = 0; j < M; ++j) {
        T cv[NP];
        load_vec<T, NP>(sCt + e * RST + j * NP, cv);
        T acc = 0;
#pragma unroll
        for (int k = 0; k < NP; ++k) acc += phi[k] * cv[k];
        U[j] = acc;
      }
      if constexpr (RND) {
#pragma unroll
        for (int j = 0; j < M; ++j) U[j] = probe<RND, T>(U[j], a.round_mask, kRndVolumeValues);
      }
      if (!is_physical<K::LAW, T>(a.law, U)) flag_nonphysical(a.status, ft.e0 + e);
      T F[M][DIM];
      volume_flux<K::LAW, DIM, T>(a.law, U, F);
      T J[DIM * DIM];
#pragma unroll
      for (int i = 0; i < DIM * DIM; ++i) J[i] = probe<RND, T>(sJi[e * DIM * DIM + i], a.round_mask, kRndGeometry);
      const T jw = probe<RND, T>((T)sDet[e] * w, a.round_mask, kRndGeometry);
      // G[(cell, field)][r * NQ + q]: consecutive points of a cell land in
      // consecutive words
#pragma unroll
      for (int j = 0; j < M; ++j)
#pragma unroll
        for (int r = 0; r < DIM; ++r) {
          T acc = 0;
#pragma unroll
          for (int i = 0; i < DIM; ++i) acc += F[j][i] * J[i * DIM + r];
          if constexpr (FS::UMMA) {
            // A[(cell, field)][r * NQ + q] as TF32 high and low parts
            uint32_t hi, lo;
            tf32_split((float)(acc * jw), hi, lo);
            const uint32_t o = umma_off(e * M + j, r * NQ + q, FS::KPAD);
            *reinterpret_cast<uint32_t*>(smem_raw + FS::oX + o) = hi;
            *reinterpret_cast<uint32_t*>(smem_raw + FS::oX + FS::a_bytes + o) = lo;
          } else {
            sG[(e * M + j) * LDK + r * NQ + q] = probe<RND, T>(acc * jw, a.round_mask, kRndVolumeFlux);
          }
        }
    }
  }
  if constexpr (FS::UMMA) {
    // the padding columns of A are zero (the padding rows of B are): then the
    // generic writes of A are ordered before the tensor cores read it
    constexpr int NPAD = FS::KPAD - KV;
    if constexpr (NPAD > 0) {
      for (int i = tid; i < 128 * NPAD; i += BLOCK) {
        const uint32_t o = umma_off(i / NPAD, KV + i % NPAD, FS::KPAD);
        *reinterpret_cast<uint32_t*>(smem_raw + FS::oX + o) = 0u;
        *reinterpret_cast<uint32_t*>(smem_raw + FS::oX + FS::a_bytes + o) = 0u;
      }
    }
    fence_proxy_async_smem();
  }
  // u_n of the row (stages 2 and 3) from global memory while the volume and
  // contraction run; stage-1 P0 marks zero its modes k >= 1
  const int row = tid;
  const bool live = row < ft.ne * M;
  const size_t gbase = ((size_t)ft.e0 * M + row) * NP;
  constexpr int RALIGN = pow2_div(NP * 8) < 16 ? pow2_div(NP * 8) : 16;
  double u0[NP];
  if (live && a.stage >= 2) {
    ldg_vec<double, NP, RALIGN>(a.U0 + gbase, u0);
    if (a.p0 && a.bad[ft.e0 + row / M]) {
#pragma unroll
      for (int k = 1; k < NP; ++k) u0[k] = 0.0;
    }
  }
  __syncthreads();

  // ---- contraction + lift + inverse mass + stage combination ---------------
  if constexpr (FS::UMMA) {
    // D[row][mode] = sum over K of A B: per k-step of 8, the products
    // hi hi + hi lo + lo hi (TF32), accumulated in FP32 in tensor memory; the
    // CUDA cores lift the face slots meanwhile
    tc_fence_after();
    if (tid == 0) {
      constexpr uint32_t idesc = umma_idesc_tf32(128, FS::UN);
      constexpr uint32_t SBO_A = (FS::KPAD / 4) * 128, SBO_B = SBO_A;
      const unsigned char* A = smem_raw + FS::oX;
      const unsigned char* B = smem_raw + FS::oBhi;
      uint32_t accum = 0;
#pragma unroll
      for (int kb = 0; kb < FS::KPAD / 8; ++kb) {
        const uint32_t ko = (uint32_t)kb * 256;
        const uint64_t ahi = umma_desc(A + ko, 128, SBO_A), alo = umma_desc(A + FS::a_bytes + ko, 128, SBO_A);
        const uint64_t bhi = umma_desc(B + ko, 128, SBO_B), blo = umma_desc(B + FS::b_bytes + ko, 128, SBO_B);
        umma_tf32(s_tmem, ahi, bhi, idesc, accum);
        accum = 1;
        umma_tf32(s_tmem, ahi, blo, idesc, 1);
        umma_tf32(s_tmem, alo, bhi, idesc, 1);
      }
      umma_commit(&mma_bar);
    }
  }
  double rsum = 0.0;
  T acc[NPP];
#pragma unroll
  for (int k = 0; k < NPP; ++k) acc[k] = 0;
  if (live) {
    if constexpr (!FS::UMMA) {
      const T* gr = sG + row * LDK;
#pragma unroll 4
      for (int kk = 0; kk < KV; ++kk) {
        const T gv = gr[kk];
        T d[NPP];
        load_vec<T, NPP>(sDphi + kk * NPP, d);
#pragma unroll
        for (int k = 0; k < NPP; ++k) acc[k] += gv * d[k];
      }
    }
#pragma unroll 4
    for (int s = 0; s < NS; ++s) {
      const T sv = sS[s * ROWS + row];
      T p[NPP];
      load_vec<T, NPP>(sPhif + s * NPP, p);
#pragma unroll
      for (int k = 0; k < NPP; ++k) acc[k] += sv * p[k];
    }
  }
  if constexpr (FS::UMMA) {
    if (!mbar_wait(&mma_bar, 0, kMbarPolls)) {
      // never expected: record it, then wait once more (bounded) so that the
      // tensor memory is not read or freed under a running MMA
      if (tid == 0) atomicAdd(&a.status->timeouts, 1);
      mbar_wait(&mma_bar, 0, kMbarPolls);
    }
    tc_fence_after();
    float dv[16];
    tmem_ld16(s_tmem + ((uint32_t)(tid & ~31) << 16), dv);
#pragma unroll
    for (int k = 0; k < NPP; ++k) acc[k] += (k < 16 ? dv[k < 16 ? k : 0] : (T)0);
  }
  if (live) {
    const int e = row / M, j = row - (row / M) * M;
    double* crow = sC + (size_t)e * RS + j * NP;
    if (a.stage == 0) {
#pragma unroll
      for (int k = 0; k < NP; ++k) a.Cout[gbase + k] = (double)acc[k];
    } else {
      // FP64 update in the reference's operation order (dt/|J| in FP64)
      const double dtj = c->dt / sDet[e];
      double cv[NP];
      load_vec<double, NP>(crow, cv);
      if (a.stage == 1 && a.U0out) {
#pragma unroll
        for (int k = 0; k < NP; ++k) a.U0out[gbase + k] = cv[k];
      }
      double out[NP];
#pragma unroll
      for (int k = 0; k < NP; ++k) {
        const double r = probe<RND, double>((double)acc[k], a.round_mask, kRndContraction);
        if (a.stage == 1) {
          out[k] = cv[k] + r * dtj;
        } else if (a.stage == 2) {
          out[k] = 0.25 * (cv[k] + r * dtj + 3. * u0[k]);
        } else {
          out[k] = (2.0 * (cv[k] + r * dtj) + u0[k]) / 3.0;
          const double dd = out[k] - u0[k];
          rsum += dd * dd;
        }
      }
#pragma unroll
      for (int k = 0; k < NP; ++k) crow[k] = out[k];
      st_vec<double, NP, RALIGN>(a.Cout + gbase, out);
    }
  }
  if constexpr (FS::UMMA) {
    tc_fence_before();
    __syncthreads();
    if (tid < 32) tmem_dealloc(s_tmem, 32);
  }
  if (a.stage != 3) return;
  __syncthreads();
  fused_tile_tail<K, RS>(a, c, tile, rsum, sC, sEig, ft.ne, red, sPv, csz);
}

// After the last stage: one CTA sums the tiles' residual partials in tile
// order, takes the minimum of their CFL steps, advances the time and, with the
// fused CFL, finalizes the next step (per instance for ensembles).  Keeping
// this out of the stage kernel spares every tile a fence and an atomic round
// trip on one address.
template <class K>
__global__ void __launch_bounds__(kFinalizeThreads) stage_finalize_kernel(
    const __grid_constant__ StageArgs<typename K::T> a, int ntiles) {
  constexpr int NT = kFinalizeThreads;
  __shared__ double red[NT / 32];
  if (a.gctl->done) return;
  const double* part = a.partials;
  const double* dtp = a.partials + ntiles;
  const int tid = threadIdx.x;
  if (a.cell_inst) {
    for (int i = tid; i < a.ninst; i += NT) {
      TimeCtl* c = a.ctl + i;
      if (c->done) continue;
      double r = 0.0, d = 1e300;
      for (int b = a.tile_first[i]; b < a.tile_first[i + 1]; ++b) {
        r += part[b];
        d = fmin(d, dtp[b]);
      }
      c->resid = r;
      c->t = c->t + c->dt;
      c->steps += 1;
      if (a.fuse_cfl) {
        ctl_finalize(c, d);
        if (c->done) c->t_mark_ns = device_clock_ns();
      }
    }
    __syncthreads();
    if (tid == 0) {
      int all = 1;
      for (int i = 0; i < a.ninst; ++i) all &= (*(volatile int*)&a.ctl[i].done) != 0;
      a.gctl->done = all;
    }
    return;
  }
  double r = 0.0, d = 1e300;
  for (int b = tid; b < ntiles; b += NT) {
    r += part[b];
    d = fmin(d, dtp[b]);
  }
  r = block_sum<NT>(r, red);
  d = block_min<NT>(d, red);
  if (tid == 0) {
    TimeCtl* c = a.ctl;
    c->resid = r;
    c->t = c->t + c->dt;
    c->steps += 1;
    if (a.fuse_cfl) ctl_finalize(c, d);
  }
}

}  // namespace dgp
