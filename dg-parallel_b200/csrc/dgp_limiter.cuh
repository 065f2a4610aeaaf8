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
//     cells, TimeIntegrator.cc:1414-1434): one kernel computes the limited rows
//     into L, a second copies the rows of triggered cells back.
//   * Per field, degrees n = p..1: a degree whose modes are all below 1e-10 in
//     magnitude is skipped; a degree with no limited component ends the
//     descent.  minmod and absmin as DGLimiter.cc:1424-1447.
//   * The moments of degree n are the n+1 physical derivatives
//     d^n/dx^(n-a)dy^a of the cell's degree-n modal block (constant on the
//     cell).  Component a is bounded in x by the differences of the
//     derivative d^(n-1)/dx^(n-1-a)dy^a of the degree-(n-1) blocks of the
//     left/right neighbours, in y by d^(n-1)/dx^(n-a)dy^(a-1) of the
//     bottom/top neighbours, each divided by the distance of the bounding-box
//     centres (degree 0: the cell mean).  A limited degree maps back to its
//     modal block exactly; the mean never changes.
//   * Trigger (the sensor) of a cell: lowest limited degree over its fields,
//     0 when untouched.
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
  const double* C;      // state (unlimited)
  double* L;            // limited rows (written for triggered cells)
  unsigned char* trig;  // [E] trigger degree
  const int* nb;        // [E][4] left, right, bottom, top (-1: none)
  const double* geo;    // [E][kLimGeo]
  const double* Dn;     // per degree n: (n+1)^2 block at n(n+1)(2n+1)/6
  const double* Dinv;
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

template <int N>
__device__ __forceinline__ void lim_lower(const LimArgs& a, int cell, const double* __restrict__ row,
                                          double (&h)[N + 1]) {
  const double* gg = a.geo + (size_t)cell * kLimGeo;
  double P[N + 1][N + 1];
  lim_transform<N>(__ldg(gg + 0), __ldg(gg + 1), __ldg(gg + 2), __ldg(gg + 3), P);
  lim_moments<N>(row, a.Dn, P, h);
}

// one degree N of one field; returns false when the descent ends
template <int N, int M, int NP>
__device__ __forceinline__ bool lim_degree(const LimArgs& a, int e, int j, const int (&nb)[4], const double* gg,
                                           int& trig, unsigned& modified) {
  constexpr int base = N * (N + 1) / 2, w = N + 1, off = N * (N + 1) * (2 * N + 1) / 6;
  const double* row = a.C + ((size_t)e * M + j) * NP;
  bool big = false;
#pragma unroll
  for (int m = 0; m <= N; ++m) big |= fabs(row[base + m]) > kLimSmall;
  if (!big) return true;
  double P[N + 1][N + 1], g[N + 1], gl[N + 1], he[N], hx[4][N];
  lim_transform<N>(gg[0], gg[1], gg[2], gg[3], P);
  lim_moments<N>(row, a.Dn, P, g);
  lim_lower<N - 1>(a, e, row, he);
#pragma unroll
  for (int d = 0; d < 4; ++d)
    if (nb[d] >= 0) lim_lower<N - 1>(a, nb[d], a.C + ((size_t)nb[d] * M + j) * NP, hx[d]);
  const double px = gg[8], py = gg[9];
  bool any = false;
#pragma unroll
  for (int c = 0; c <= N; ++c) {
    gl[c] = g[c];
    const bool hasx = c <= N - 1 && (nb[0] >= 0 || nb[1] >= 0);
    const bool hasy = c >= 1 && (nb[2] >= 0 || nb[3] >= 0);
    double t1 = 0.0, t2 = 0.0;
    bool l1 = false, l2 = false;
    if (hasx) {
      double fwd = 0.0, bwd = 0.0;
      if (c <= N - 1) {
        if (nb[1] >= 0) fwd = __dsub_rn(hx[1][c], he[c]) / __dsub_rn(__ldg(a.geo + (size_t)nb[1] * kLimGeo + 8), px);
        if (nb[0] >= 0) bwd = __dsub_rn(he[c], hx[0][c]) / __dsub_rn(px, __ldg(a.geo + (size_t)nb[0] * kLimGeo + 8));
      }
      if (nb[0] >= 0 && nb[1] >= 0) t1 = lim_minmod3(g[c], fwd, bwd, l1);
      else if (nb[0] >= 0) t1 = lim_minmod2(g[c], bwd, l1);
      else t1 = lim_minmod2(g[c], fwd, l1);
    }
    if (hasy) {
      double fwd = 0.0, bwd = 0.0;
      if (c >= 1) {
        if (nb[3] >= 0)
          fwd = __dsub_rn(hx[3][c - 1], he[c - 1]) / __dsub_rn(__ldg(a.geo + (size_t)nb[3] * kLimGeo + 9), py);
        if (nb[2] >= 0)
          bwd = __dsub_rn(he[c - 1], hx[2][c - 1]) / __dsub_rn(py, __ldg(a.geo + (size_t)nb[2] * kLimGeo + 9));
      }
      if (nb[2] >= 0 && nb[3] >= 0) t2 = lim_minmod3(g[c], fwd, bwd, l2);
      else if (nb[2] >= 0) t2 = lim_minmod2(g[c], bwd, l2);
      else t2 = lim_minmod2(g[c], fwd, l2);
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
  double Q[N + 1][N + 1], r[N + 1];
  lim_transform<N>(gg[4], gg[5], gg[6], gg[7], Q);
#pragma unroll
  for (int i = 0; i <= N; ++i) {
    double acc = 0.0;
#pragma unroll
    for (int c = 0; c <= N; ++c) acc = __dadd_rn(acc, __dmul_rn(Q[i][c], gl[c]));
    r[i] = acc;
  }
  double* out = a.L + ((size_t)e * M + j) * NP;
#pragma unroll
  for (int k = 0; k <= N; ++k) {
    double acc = 0.0;
#pragma unroll
    for (int i = 0; i <= N; ++i) acc = __dadd_rn(acc, __dmul_rn(__ldg(a.Dinv + off + k * w + i), r[i]));
    out[base + k] = acc;
  }
  modified |= 1u << N;
  trig = (trig == 0 || N < trig) ? N : trig;
  return true;
}

template <int N, int M, int NP>
__device__ __forceinline__ void lim_descend(const LimArgs& a, int e, int j, const int (&nb)[4], const double* gg,
                                            int& trig, unsigned& modified) {
  if constexpr (N >= 1) {
    if (lim_degree<N, M, NP>(a, e, j, nb, gg, trig, modified)) lim_descend<N - 1, M, NP>(a, e, j, nb, gg, trig, modified);
  }
}

// one thread per cell: limited rows of triggered cells into L, trigger into trig
template <class K>
__global__ void __launch_bounds__(128) limit_kernel(LimArgs a) {
  constexpr int M = K::M, NP = K::NP, P = K::ORDER;
  if (a.ctl && a.gctl->done) return;
  const int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= a.E || lim_skip_cell(a, e)) return;
  int nb[4];
#pragma unroll
  for (int d = 0; d < 4; ++d) nb[d] = __ldg(a.nb + 4 * e + d);
  double gg[kLimGeo];
#pragma unroll
  for (int i = 0; i < kLimGeo; ++i) gg[i] = __ldg(a.geo + (size_t)e * kLimGeo + i);
  int trig = 0;
  unsigned modified[M];
#pragma unroll
  for (int j = 0; j < M; ++j) {
    modified[j] = 0;
    lim_descend<P, M, NP>(a, e, j, nb, gg, trig, modified[j]);
  }
  if (trig) {
    // the untouched blocks of a triggered cell complete its row in L
#pragma unroll
    for (int j = 0; j < M; ++j) {
      const double* row = a.C + ((size_t)e * M + j) * NP;
      double* out = a.L + ((size_t)e * M + j) * NP;
#pragma unroll
      for (int n = 0; n <= P; ++n)
        if (!((modified[j] >> n) & 1u))
#pragma unroll
          for (int k = 0; k <= n; ++k) out[n * (n + 1) / 2 + k] = row[n * (n + 1) / 2 + k];
    }
  }
  a.trig[e] = static_cast<unsigned char>(trig);
}

// copy the limited rows of triggered cells back into the state
template <class K>
__global__ void __launch_bounds__(256) limit_apply_kernel(LimArgs a) {
  if (a.ctl && a.gctl->done) return;
  const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (i >= (long long)a.E * K::MNP) return;
  const int e = static_cast<int>(i / K::MNP);
  if (lim_skip_cell(a, e)) return;
  if (a.trig[e]) const_cast<double*>(a.C)[i] = a.L[i];
}

}  // namespace dgp
