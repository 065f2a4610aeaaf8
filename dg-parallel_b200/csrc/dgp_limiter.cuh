// Triangle moment limiter (the limiter of DGMomentLimiter::limit,
// DGLimiter.cc:963-1133, rebuilt for triangles) and the DGSensor trigger.
//
// The reference limiter indexes the tensor Legendre basis of quadrilaterals
// ((p+1)^2-1, ...) and reads past a triangle's coefficient row, so on
// triangles the limiter is defined as follows; the CPU oracle restates the
// same definition independently.
//   * Neighbours left/right/bottom/top by bounding boxes, as DGLimiter.cc:
//     970-993 (faces in local-face order, a later face overwrites).
//   * Every difference reads the unlimited state (the reference reads slot 0
//     and writes the copy slot; TimeIntegrator::limit copies back after all
//     cells, TimeIntegrator.cc:1414-1434): a first kernel writes the moments
//     of every degree of every (cell, field) row of the unlimited state, a
//     second limits each row from those moments alone, so that it can write
//     the limited blocks (and the row's face-point traces) in place.
//   * Per field, degrees n = p..1: a degree whose modes are all below 1e-10 in
//     magnitude is skipped; a degree with no limited component ends the
//     descent.  minmod and absmin as DGLimiter.cc:1424-1447.
//   * The moments of degree n are the n+1 physical derivatives
//     d^n/dx^(n-a)dy^a of the cell's degree-n modal block (constant on the
//     cell).  Component a is bounded in x by the differences of the
//     derivative d^(n-1)/dx^(n-1-a)dy^a of the degree-(n-1) blocks of the
//     left/right neighbours, in y by d^(n-1)/dx^(n-a)dy^(a-1) of the
//     bottom/top neighbours, each times the reciprocal (rounded once) of the
//     distance of the bounding-box centres (degree 0: the cell mean).  A limited degree maps back to its
//     modal block exactly; the mean never changes.
//   * Trigger (the sensor) of a cell: lowest limited degree over its fields,
//     0 when untouched (the kernels record it per row; the host reduces).
// Products and sums are single-rounding intrinsics in a fixed order (no FMA
// contraction), so the moments -- and therefore the trigger set -- match the
// CPU restatement bit for bit on the same state.
#pragma once

#include "dgp_kernels.cuh"

namespace dgp {

// per-cell FP64 limiter geometry: d xi/dx (A, B), d xi/dy (C, D), d x/du,
// d y/du, d x/dv, d y/dv, bounding-box centre
constexpr int kLimGeo = 10;
constexpr double kLimSmall = 1.0e-10;

struct LimArgs {
  double* C;            // state, limited in place
  double* Mo;           // [E * M][NP] moments of every degree of each row of the unlimited state
  unsigned char* big;   // [E * M] bit n: a mode of degree n above kLimSmall in magnitude
  unsigned char* trig;  // [E * M] trigger degree of each row (0: untouched)
  const int* nb;        // [E][4] left, right, bottom, top (-1: none)
  const double* geo;    // [E][kLimGeo]
  const double* Dn;     // per degree n: (n+1)^2 block at n(n+1)(2n+1)/6
  const double* Dinv;
  void* tr;             // face-point traces (slot layout, type of the right-hand side)
  const void* phif;     // [NS][NP] face-point basis values (same type)
  const TimeCtl* ctl;   // kernels are no-ops once the run is done (nullptr: always run)
  const TimeCtl* gctl;
  const int* cell_inst; // ensembles: instance of each cell (-1: padding); finished
                        // instances are left alone
  int E;
};

__device__ __forceinline__ bool lim_skip_cell(const LimArgs& a, int e) {
  if (!a.cell_inst) return false;
  const int i = a.cell_inst[e];
  return i < 0 || (a.ctl && a.ctl[i].done);
}

__device__ __forceinline__ double lim_minmod3(double a, double b, double c, bool& lim) {
  const bool sa = a < 0.0, sb = b < 0.0, sc = c < 0.0;
  if (sa == sb && sb == sc) {
    const double aa = fabs(a), ab = fabs(b), ac = fabs(c);
    if (aa < ab && aa < ac) {
      lim = false;
      return a;
    }
    lim = true;
    return ab < ac ? b : c;
  }
  lim = true;
  return 0.0;
}

__device__ __forceinline__ double lim_minmod2(double a, double b, bool& lim) {
  if ((a < 0.0) == (b < 0.0)) {
    if (fabs(a) < fabs(b)) {
      lim = false;
      return a;
    }
    lim = true;
    return b;
  }
  lim = true;
  return 0.0;
}

// P[a][i]: coefficient of s^(N-i) t^i in (A s + B t)^(N-a) (C s + D t)^a
template <int N>
__device__ __forceinline__ void lim_transform(double A, double B, double C, double D,
                                              double (&P)[N + 1][N + 1]) {
#pragma unroll
  for (int a = 0; a <= N; ++a) {
    double poly[N + 2];
    poly[0] = 1.0;
#pragma unroll
    for (int i = 1; i < N + 2; ++i) poly[i] = 0.0;
#pragma unroll
    for (int k = 0; k < N; ++k) {
      const double u = (k < N - a) ? A : C, v = (k < N - a) ? B : D;
      // degree of poly before this factor is k
#pragma unroll
      for (int i = k + 1; i >= 0; --i) {
        const double x = (i <= k) ? __dmul_rn(poly[i], u) : 0.0;
        const double y = (i >= 1) ? __dmul_rn(poly[i - 1], v) : 0.0;
        poly[i] = __dadd_rn(x, y);
      }
    }
#pragma unroll
    for (int i = 0; i <= N; ++i) P[a][i] = poly[i];
  }
}

// physical degree-N derivatives of the degree-N block of one coefficient row
template <int N>
__device__ __forceinline__ void lim_moments(const double* __restrict__ row, const double* __restrict__ Dn,
                                            const double (&P)[N + 1][N + 1], double (&g)[N + 1]) {
  constexpr int base = N * (N + 1) / 2, off = N * (N + 1) * (2 * N + 1) / 6, w = N + 1;
  double r[N + 1];
#pragma unroll
  for (int i = 0; i <= N; ++i) {
    double acc = 0.0;
#pragma unroll
    for (int m = 0; m <= N; ++m) acc = __dadd_rn(acc, __dmul_rn(__ldg(Dn + off + i * w + m), row[base + m]));
    r[i] = acc;
  }
#pragma unroll
  for (int a = 0; a <= N; ++a) {
    double acc = 0.0;
#pragma unroll
    for (int i = 0; i <= N; ++i) acc = __dadd_rn(acc, __dmul_rn(P[a][i], r[i]));
    g[a] = acc;
  }
}

// one thread per (cell, field) row: the degree-n physical derivatives of
// every degree-n block, n = 0..p, and the mask of the degrees with a mode above
// kLimSmall
template <int N, int NP>
__device__ __forceinline__ void lim_row_moments(const double* __restrict__ row, const double* __restrict__ Dn,
                                                const double* gg, double* __restrict__ mo, unsigned& big) {
  constexpr int base = N * (N + 1) / 2;
  double P[N + 1][N + 1], g[N + 1];
  lim_transform<N>(gg[0], gg[1], gg[2], gg[3], P);
  lim_moments<N>(row, Dn, P, g);
  bool b = false;
#pragma unroll
  for (int m = 0; m <= N; ++m) {
    mo[base + m] = g[m];
    b |= fabs(row[base + m]) > kLimSmall;
  }
  if (b) big |= 1u << N;
  if constexpr (N >= 1) lim_row_moments<N - 1, NP>(row, Dn, gg, mo, big);
}

template <class K>
__global__ void __launch_bounds__(128) limit_moments_kernel(LimArgs a) {
  constexpr int M = K::M, NP = K::NP, P = K::ORDER;
  // the CTA's 128 rows are contiguous in the state and in the moments: both
  // move through shared memory with coalesced loads and stores
  __shared__ double s[128 * NP];
  __shared__ unsigned char s_act[128];
  if (a.ctl && a.gctl->done) return;
  const size_t R = (size_t)a.E * M;
  const size_t r0 = blockIdx.x * (size_t)128;
  const int nr = (int)(R - r0 < 128 ? R - r0 : 128);
  const int t = threadIdx.x;
  for (int i = t; i < nr * NP; i += 128) s[i] = a.C[r0 * NP + i];
  __syncthreads();
  const size_t r = r0 + t;
  bool active = t < nr;
  const int e = active ? static_cast<int>(r / M) : 0;
  if (active && lim_skip_cell(a, e)) active = false;
  s_act[t] = active ? 1 : 0;
  if (active) {
    double gg[4];
#pragma unroll
    for (int i = 0; i < 4; ++i) gg[i] = __ldg(a.geo + (size_t)e * kLimGeo + i);
    double row[NP], mo[NP];
#pragma unroll
    for (int k = 0; k < NP; ++k) row[k] = s[t * NP + k];
    unsigned big = 0;
    lim_row_moments<P, NP>(row, a.Dn, gg, mo, big);
#pragma unroll
    for (int k = 0; k < NP; ++k) s[t * NP + k] = mo[k];  // the thread's own row
    a.big[r] = static_cast<unsigned char>(big);
  }
  __syncthreads();
  for (int i = t; i < nr * NP; i += 128)
    if (s_act[i / NP]) a.Mo[r0 * NP + i] = s[i];
}

// one degree N of one row from the moments in registers (mo: the row's own,
// mn: the neighbours' degrees 0..p-1, rc: reciprocals of the signed distances
// to the neighbours' bounding-box centres); returns false when the descent ends
template <int N, int NP, int NL>
__device__ __forceinline__ bool lim_degree(const LimArgs& a, const double (&mo)[NP], const double (&mn)[4][NL],
                                           const double (&rc)[4], const int (&nb)[4], const double* gg,
                                           unsigned big, double* row, unsigned& mod) {
  constexpr int base = N * (N + 1) / 2, lo = (N - 1) * N / 2, w = N + 1, off = N * (N + 1) * (2 * N + 1) / 6;
  if (!((big >> N) & 1u)) return true;
  double gl[N + 1];
  bool any = false;
#pragma unroll
  for (int c = 0; c <= N; ++c) {
    const double g = mo[base + c];
    gl[c] = g;
    const bool hasx = c <= N - 1 && (nb[0] >= 0 || nb[1] >= 0);
    const bool hasy = c >= 1 && (nb[2] >= 0 || nb[3] >= 0);
    double t1 = 0.0, t2 = 0.0;
    bool l1 = false, l2 = false;
    if (hasx) {
      double fwd = 0.0, bwd = 0.0;
      if (c <= N - 1) {
        const double he = mo[lo + c];
        if (nb[1] >= 0) fwd = __dmul_rn(__dsub_rn(mn[1][lo + c], he), rc[1]);
        if (nb[0] >= 0) bwd = __dmul_rn(__dsub_rn(he, mn[0][lo + c]), rc[0]);
      }
      if (nb[0] >= 0 && nb[1] >= 0) t1 = lim_minmod3(g, fwd, bwd, l1);
      else if (nb[0] >= 0) t1 = lim_minmod2(g, bwd, l1);
      else t1 = lim_minmod2(g, fwd, l1);
    }
    if (hasy) {
      double fwd = 0.0, bwd = 0.0;
      if (c >= 1) {
        const double he = mo[lo + c - 1];
        if (nb[3] >= 0) fwd = __dmul_rn(__dsub_rn(mn[3][lo + c - 1], he), rc[3]);
        if (nb[2] >= 0) bwd = __dmul_rn(__dsub_rn(he, mn[2][lo + c - 1]), rc[2]);
      }
      if (nb[2] >= 0 && nb[3] >= 0) t2 = lim_minmod3(g, fwd, bwd, l2);
      else if (nb[2] >= 0) t2 = lim_minmod2(g, bwd, l2);
      else t2 = lim_minmod2(g, fwd, l2);
    }
    if (hasx && hasy) {
      if (l1 || l2) {
        gl[c] = fabs(t1) < fabs(t2) ? t1 : t2;
        any = true;
      }
    } else if (hasx) {
      if (l1) {
        gl[c] = t1;
        any = true;
      }
    } else if (hasy) {
      if (l2) {
        gl[c] = t2;
        any = true;
      }
    }
  }
  if (!any) return false;
  // back to reference derivatives (d/du = x_u d/dx + y_u d/dy, ...) and modes
  double Q[N + 1][N + 1], q[N + 1];
  lim_transform<N>(gg[0], gg[1], gg[2], gg[3], Q);
#pragma unroll
  for (int i = 0; i <= N; ++i) {
    double acc = 0.0;
#pragma unroll
    for (int c = 0; c <= N; ++c) acc = __dadd_rn(acc, __dmul_rn(Q[i][c], gl[c]));
    q[i] = acc;
  }
#pragma unroll
  for (int k = 0; k <= N; ++k) {
    double acc = 0.0;
#pragma unroll
    for (int i = 0; i <= N; ++i) acc = __dadd_rn(acc, __dmul_rn(__ldg(a.Dinv + off + k * w + i), q[i]));
    row[base + k] = acc;
  }
  mod |= 1u << N;
  return true;
}

template <int N, int NP, int NL>
__device__ __forceinline__ void lim_descend(const LimArgs& a, const double (&mo)[NP], const double (&mn)[4][NL],
                                            const double (&rc)[4], const int (&nb)[4], const double* gg,
                                            unsigned big, double* row, unsigned& mod) {
  if constexpr (N >= 1) {
    if (lim_degree<N, NP, NL>(a, mo, mn, rc, nb, gg, big, row, mod))
      lim_descend<N - 1, NP, NL>(a, mo, mn, rc, nb, gg, big, row, mod);
  }
}

// one thread per (cell, field) row: limits the row from the moments, writes the
// limited blocks into the state and the row's face-point traces.  Every input
// of the descent (the row's moments, the neighbours' moments of degrees below
// p and their centres) is loaded up front, so the descent waits on one round
// of loads whatever its depth.
template <class K>
__global__ void __launch_bounds__(128) limit_kernel(LimArgs a) {
  using T = typename K::T;
  constexpr int M = K::M, NP = K::NP, P = K::ORDER, NS = K::NS;
  constexpr int NL = P * (P + 1) / 2;  // moments of degrees 0..p-1
  if (a.ctl && a.gctl->done) return;
  const size_t R = (size_t)a.E * M;
  const size_t r = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
  if (r >= R) return;
  const int e = static_cast<int>(r / M);
  if (lim_skip_cell(a, e)) return;
  const int j = static_cast<int>(r - (size_t)e * M);
  const unsigned big = a.big[r];
  const int4 n4 = __ldg(reinterpret_cast<const int4*>(a.nb) + e);
  // Q needs d x/du, d y/du, d x/dv, d y/dv; then the bounding-box centre
  double gg[6];
#pragma unroll
  for (int i = 0; i < 6; ++i) gg[i] = __ldg(a.geo + (size_t)e * kLimGeo + 4 + i);
  int trig = 0;
  if (big >> 1) {
    const int nb[4] = {n4.x, n4.y, n4.z, n4.w};
    double mo[NP], mn[4][NL], rc[4];
#pragma unroll
    for (int k = 0; k < NP; ++k) mo[k] = a.Mo[r * NP + k];
#pragma unroll
    for (int d = 0; d < 4; ++d) {
      const int n = nb[d] >= 0 ? nb[d] : e;  // a missing neighbour is never read
      const double* src = a.Mo + ((size_t)n * M + j) * NP;
#pragma unroll
      for (int k = 0; k < NL; ++k) mn[d][k] = src[k];
      const double pc = __ldg(a.geo + (size_t)n * kLimGeo + (d < 2 ? 8 : 9));
      const double own = gg[d < 2 ? 4 : 5];
      // left / bottom: own - theirs; right / top: theirs - own
      rc[d] = 1.0 / ((d & 1) ? __dsub_rn(pc, own) : __dsub_rn(own, pc));
    }
    double row[NP];
    unsigned mod = 0;
    lim_descend<P, NP, NL>(a, mo, mn, rc, nb, gg, big, row, mod);
    if (mod) {
      trig = __ffs(mod) - 1;  // lowest limited degree
      // the row as it leaves the limiter: unchanged blocks from the state,
      // limited blocks from the descent (written back in place)
      double* c = a.C + r * NP;
      T ck[NP];
#pragma unroll
      for (int k = 0; k < NP; ++k) ck[k] = (T)c[k];
#pragma unroll
      for (int n = 1; n <= P; ++n)
        if ((mod >> n) & 1u)
#pragma unroll
          for (int k = n * (n + 1) / 2; k < (n + 1) * (n + 2) / 2; ++k) {
            c[k] = row[k];
            ck[k] = (T)row[k];
          }
      const T* phif = static_cast<const T*>(a.phif);
      T* tr = static_cast<T*>(a.tr);
      for (int s = 0; s < NS; ++s) {
        T acc = 0;
#pragma unroll
        for (int k = 0; k < NP; ++k) acc += __ldg(phif + s * NP + k) * ck[k];
        tr[slot_index<K>(e, s, j)] = acc;
      }
    }
  }
  a.trig[r] = static_cast<unsigned char>(trig);
}

// -----------------------------------------------------------------------------
// Barth limiter (DGBarthLimiter::limit, DGLimiter.cc:184-287), cell by cell as
// the reference computes it on the cell's coefficients:
//   * bounds: max / min over the interior-face neighbours' means (the cell's
//     own mean is not included); a cell without an interior neighbour is left
//     alone (the reference would read uninitialised bounds);
//   * every face point of every face of the cell (boundary faces included):
//     val = the cell's coefficients against the LEFT cell's basis values at the
//     point (the reference interpolates with pg->fctleft whichever side the
//     cell is on), phi = (bound - mean) / (val - mean) where val leaves
//     [min, max], 1 inside, clamped at 0; the field's slope factor is the
//     minimum over the points;
//   * degrees p..2: the block is zeroed when the factor is below 0.9; the
//     degree-1 block is scaled by the factor.
// The mean (mode 0) never changes, so every cell reads its neighbours' means
// from the state being limited in place.  Triggers: 1 where a factor is below 1.
struct BarthArgs {
  double* C;
  unsigned char* trig;  // [E * M] (the cell's value in every row)
  const int* cface;     // [E][NLF] face of each local face
  const int* fel;       // [F][2]
  const int* fcode;     // [F] lfL | lfR << 4 | perm << 8
  const double* phif;   // [NLF * NQF][NP] FP64 face-point basis values
  double phi0;          // constant basis function (mean = c0 * phi0)
  void* tr;             // face-point traces (slot layout, right-hand-side type)
  const void* phif_t;   // the same basis values in the right-hand-side type
  const TimeCtl* ctl;
  const TimeCtl* gctl;
  const int* cell_inst;
  int E;
  // the pass's slope factors per (cell, field): written when not null, or,
  // with replay, applied as recorded (the limiter frozen to a fixed linear
  // map, as the discrete adjoint linearises it); trig, tr may then be null
  double* slope;
  int replay;
};

template <class K>
__global__ void __launch_bounds__(128) barth_kernel(BarthArgs a) {
  using T = typename K::T;
  constexpr int M = K::M, NP = K::NP, NLF = K::NLF, NQF = K::NQF, NS = K::NS;
  constexpr int S1 = K::DIM == 2 ? 3 : 4;  // modes of degree <= 1
  if (a.ctl && a.gctl->done) return;
  const int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= a.E) return;
  if (a.cell_inst) {
    const int i = a.cell_inst[e];
    if (i < 0 || (a.ctl && a.ctl[i].done)) return;
  }
  if (a.replay) {
    // the recorded factors: degree 1 scaled, degrees >= 2 dropped below 0.9
    double* c = a.C + (size_t)e * M * NP;
#pragma unroll
    for (int j = 0; j < M; ++j) {
      const double sl = a.slope[(size_t)e * M + j];
      if (!(sl < 1.0)) continue;
      if (sl < 0.9)
        for (int k = S1; k < NP; ++k) c[j * NP + k] = 0.0;
#pragma unroll
      for (int k = 1; k < S1; ++k) c[j * NP + k] = __dmul_rn(c[j * NP + k], sl);
    }
    return;
  }
  int fc[NLF];
#pragma unroll
  for (int l = 0; l < NLF; ++l) fc[l] = __ldg(a.cface + (size_t)e * NLF + l);
  double mx[M], mn[M];
  int kk = 0;
#pragma unroll
  for (int l = 0; l < NLF; ++l) {
    const int f = fc[l];
    if (f < 0) continue;
    const int eL = __ldg(a.fel + 2 * f), eR = __ldg(a.fel + 2 * f + 1);
    if (eR < 0) continue;
    const int o = eL == e ? eR : eL;
#pragma unroll
    for (int j = 0; j < M; ++j) {
      const double m = __dmul_rn(a.C[((size_t)o * M + j) * NP], a.phi0);
      if (kk == 0) {
        mx[j] = m;
        mn[j] = m;
      } else {
        mx[j] = m > mx[j] ? m : mx[j];
        mn[j] = m < mn[j] ? m : mn[j];
      }
    }
    ++kk;
  }
  unsigned char trig = 0;
  if (kk > 0) {
    double* c = a.C + (size_t)e * M * NP;
    double slope[M], mean[M];
#pragma unroll
    for (int j = 0; j < M; ++j) {
      slope[j] = 1.0;
      mean[j] = __dmul_rn(c[j * NP], a.phi0);
    }
#pragma unroll
    for (int l = 0; l < NLF; ++l) {
      const int f = fc[l];
      if (f < 0) continue;
      const int lfL = __ldg(a.fcode + f) & 15;
      for (int q = 0; q < NQF; ++q) {
        const double* ph = a.phif + (size_t)(lfL * NQF + q) * NP;
#pragma unroll
        for (int j = 0; j < M; ++j) {
          double v = 0.0;
#pragma unroll
          for (int k = 0; k < NP; ++k) v = __dadd_rn(v, __dmul_rn(c[j * NP + k], __ldg(ph + k)));
          double phin = 1.0;
          if (v > mx[j]) phin = __dsub_rn(mx[j], mean[j]) / __dsub_rn(v, mean[j]);
          else if (v < mn[j]) phin = __dsub_rn(mn[j], mean[j]) / __dsub_rn(v, mean[j]);
          if (phin < 0.0) phin = 0.0;
          slope[j] = slope[j] < phin ? slope[j] : phin;
        }
      }
    }
    if (a.slope)
#pragma unroll
      for (int j = 0; j < M; ++j) a.slope[(size_t)e * M + j] = slope[j];
#pragma unroll
    for (int j = 0; j < M; ++j) {
      if (!(slope[j] < 1.0)) continue;
      trig = 1;
      if (slope[j] < 0.9)
        for (int k = S1; k < NP; ++k) c[j * NP + k] = 0.0;  // degrees p..2
#pragma unroll
      for (int k = 1; k < S1; ++k) c[j * NP + k] = __dmul_rn(c[j * NP + k], slope[j]);
    }
    if (trig) {
      // the cell's face-point traces for the next stage's face kernel
      const T* pt = static_cast<const T*>(a.phif_t);
      T* tr = static_cast<T*>(a.tr);
#pragma unroll 1
      for (int j = 0; j < M; ++j) {
        T ck[NP];
#pragma unroll
        for (int k = 0; k < NP; ++k) ck[k] = (T)c[j * NP + k];
        for (int s = 0; s < NS; ++s) {
          T acc = 0;
#pragma unroll
          for (int k = 0; k < NP; ++k) acc += __ldg(pt + s * NP + k) * ck[k];
          tr[slot_index<K>(e, s, j)] = acc;
        }
      }
    }
  }
  else if (a.slope) {
#pragma unroll
    for (int j = 0; j < M; ++j) a.slope[(size_t)e * M + j] = 1.0;
  }
#pragma unroll
  for (int j = 0; j < M; ++j) a.trig[(size_t)e * M + j] = trig;
}

}  // namespace dgp
