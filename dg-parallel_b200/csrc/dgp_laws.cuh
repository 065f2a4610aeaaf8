// Device point physics of the conservation laws: volume flux, numerical flux,
// boundary flux, maximum eigenvalue and the physical-state test.  Each
// function restates the DG-Parallel routine it cites (ConservationLaw
// virtuals, ConservationLaw.h:12-60), templated on the arithmetic type T so
// the plain form runs in FP64 and the mixed form in FP32.
#pragma once

#include <cuda_runtime.h>

#include "../../include/dgp.h"

namespace dgp {

template <int LAW>
struct LawTraits;
template <>
struct LawTraits<DGP_LAW_SCALAR> { static constexpr int M = 1; };
template <>
struct LawTraits<DGP_LAW_BURGERS2D> { static constexpr int M = 1; };
template <>
struct LawTraits<DGP_LAW_EULER2D> { static constexpr int M = 4; };
template <>
struct LawTraits<DGP_LAW_EULER3D> { static constexpr int M = 5; };
template <>
struct LawTraits<DGP_LAW_MAXWELL3D> { static constexpr int M = 6; };
template <>
struct LawTraits<DGP_LAW_MAXWELL2D> { static constexpr int M = 3; };

// Law parameters as they reach the device (DGP_NPARAMS doubles, see dgp.h)
struct LawParams {
  double p[DGP_NPARAMS];
  int field;
  int nbc;                   // boundary ids remapped by dgp_law_set_bc
  int bc_id[DGP_MAX_BC];
  int bc_kind[DGP_MAX_BC];   // DGP_BC_*
};

// the classification id a boundary face is treated as: a wall is the law's
// 40000, the far field any other id; ids without a setting keep their own rule
__host__ __device__ inline int bc_effective_id(const LawParams& lp, int bid) {
  for (int i = 0; i < lp.nbc; ++i)
    if (lp.bc_id[i] == bid) {
      if (lp.bc_kind[i] == DGP_BC_WALL) return 40000;
      if (lp.bc_kind[i] == DGP_BC_FARFIELD) return bid == 40000 ? 1 : bid;
    }
  return bid;
}

constexpr double kPi = 3.14159265358979323846;

// ---- analytic fields (FieldEvaluator::eval) ---------------------------------
template <typename T>
__device__ __forceinline__ void field_eval(const LawParams& lp, const double* x, double t, T* q) {
  const double* p = lp.p;
  switch (lp.field) {
    case DGP_FIELD_GAUSS: {
      double dx = x[0] - p[0] * t - p[3], dy = x[1] - p[1] * t - p[4];
      q[0] = (T)exp(-(dx * dx + dy * dy) / p[6]);
      break;
    }
    case DGP_FIELD_GAUSS3D: {
      double dx = x[0] - p[0] * t - p[3], dy = x[1] - p[1] * t - p[4], dz = x[2] - p[2] * t - p[5];
      q[0] = (T)exp(-(dx * dx + dy * dy + dz * dz) / p[6]);
      break;
    }
    case DGP_FIELD_VORTEX: {
      const double g = p[7], b = p[8];
      double dx = x[0] - (p[3] + t), dy = x[1] - (p[4] + t);
      double r2 = dx * dx + dy * dy;
      double e = exp(0.5 * (1.0 - r2));
      double u = 1.0 - b / (2.0 * kPi) * e * dy;
      double v = 1.0 + b / (2.0 * kPi) * e * dx;
      double T0 = 1.0 - (g - 1.0) * b * b / (8.0 * g * kPi * kPi) * e * e;
      double rho = pow(T0, 1.0 / (g - 1.0));
      double pr = pow(rho, g);
      q[0] = (T)rho;
      q[1] = (T)(rho * u);
      q[2] = (T)(rho * v);
      q[3] = (T)(pr / (g - 1.0) + 0.5 * rho * (u * u + v * v));
      break;
    }
    case DGP_FIELD_PULSE3D: {
      double dx = x[0] - p[0] * t - p[3], dy = x[1] - p[1] * t - p[4], dz = x[2] - p[2] * t - p[5];
      double rho = 1.0 + 0.2 * exp(-(dx * dx + dy * dy + dz * dz) / p[6]);
      q[0] = (T)rho;
      q[1] = (T)(rho * p[0]);
      q[2] = (T)(rho * p[1]);
      q[4] = (T)(rho * p[2]);
      q[3] = (T)(1.0 / (p[7] - 1.0) + 0.5 * rho * (p[0] * p[0] + p[1] * p[1] + p[2] * p[2]));
      break;
    }
    case DGP_FIELD_SINE:
      q[0] = (T)(0.5 + p[9] * sin(2.0 * kPi * (x[0] + x[1])));
      break;
    case DGP_FIELD_TM2D: {  // the same mode in Maxwell2d's field order (Hx, Hy, Ez)
      double L = p[10] > 0 ? p[10] : 1.0;
      double k = kPi / L, w = kPi * sqrt(2.0) / L;
      double sx = sin(k * x[0]), cx = cos(k * x[0]), sy = sin(k * x[1]), cy = cos(k * x[1]);
      q[0] = (T)(-(k / w) * sx * cy * sin(w * t));
      q[1] = (T)((k / w) * cx * sy * sin(w * t));
      q[2] = (T)(sx * sy * cos(w * t));
      break;
    }
    case DGP_FIELD_TM110: {
      double L = p[10] > 0 ? p[10] : 1.0;
      double k = kPi / L, w = kPi * sqrt(2.0) / L;
      double sx = sin(k * x[0]), cx = cos(k * x[0]), sy = sin(k * x[1]), cy = cos(k * x[1]);
      q[0] = 0;
      q[1] = 0;
      q[2] = (T)(sx * sy * cos(w * t));
      q[3] = (T)(-(k / w) * sx * cy * sin(w * t));
      q[4] = (T)((k / w) * cx * sy * sin(w * t));
      q[5] = 0;
      break;
    }
    default:
      break;
  }
}

// Euler2d::Fi (EulerLaw.cc:47-69) with 1/rho given
template <typename T>
__device__ __forceinline__ void euler2d_flux_inv(T g, const T* Q, T invrho, T (*F)[2]) {
  T Q1 = Q[1], Q2 = Q[2];
  T q12 = Q1 * Q2 * invrho, q11 = Q1 * Q1 * invrho, q22 = Q2 * Q2 * invrho;
  T p = (g - (T)1) * (Q[3] - (T)0.5 * (q11 + q22));
  T qq = invrho * (Q[3] + p);
  F[0][0] = Q1; F[0][1] = Q2;
  F[1][0] = q11 + p; F[1][1] = q12;
  F[2][0] = q12; F[2][1] = q22 + p;
  F[3][0] = Q1 * qq; F[3][1] = Q2 * qq;
}

// ---- volume flux F[j][i] (ConservationLaw::Fi) ------------------------------
template <int LAW, int DIM, typename T>
__device__ __forceinline__ void volume_flux(const LawParams& lp, const T* Q, T (*F)[DIM]) {
  if constexpr (LAW == DGP_LAW_SCALAR) {  // ScalarLaw::Fi, ScalarLaw.cc:75-83
    for (int i = 0; i < DIM; ++i) F[0][i] = (T)lp.p[i] * Q[0];
  } else if constexpr (LAW == DGP_LAW_BURGERS2D) {  // Burgers2D::Fi, Burgers2D.cc:22-28
    F[0][0] = Q[0] * Q[0] * (T)0.5;
    F[0][1] = Q[0] * Q[0] * (T)0.5;
  } else if constexpr (LAW == DGP_LAW_EULER2D) {  // Euler2d::Fi, EulerLaw.cc:47-69
    const T g = (T)lp.p[7];
    T invrho = (T)1 / Q[0];
    T Q1 = Q[1], Q2 = Q[2];
    T q12 = Q1 * Q2 * invrho, q11 = Q1 * Q1 * invrho, q22 = Q2 * Q2 * invrho;
    T p = (g - (T)1) * (Q[3] - (T)0.5 * (q11 + q22));
    T qq = invrho * (Q[3] + p);
    F[0][0] = Q1; F[0][1] = Q2;
    F[1][0] = q11 + p; F[1][1] = q12;
    F[2][0] = q12; F[2][1] = q22 + p;
    F[3][0] = Q1 * qq; F[3][1] = Q2 * qq;
  } else if constexpr (LAW == DGP_LAW_EULER3D) {  // Euler3d::Fi, EulerLaw.cc:81-107
    const T g = (T)lp.p[7];
    T invrho = (T)1 / Q[0];
    T q11 = Q[1] * Q[1] * invrho, q12 = Q[1] * Q[2] * invrho, q14 = Q[1] * Q[4] * invrho;
    T q22 = Q[2] * Q[2] * invrho, q24 = Q[2] * Q[4] * invrho, q44 = Q[4] * Q[4] * invrho;
    T p = (g - (T)1) * (Q[3] - (T)0.5 * (Q[1] * Q[1] + Q[2] * Q[2] + Q[4] * Q[4]) / Q[0]);
    F[0][0] = Q[1]; F[0][1] = Q[2]; F[0][2] = Q[4];
    F[1][0] = q11 + p; F[1][1] = q12; F[1][2] = q14;
    F[2][0] = q12; F[2][1] = q22 + p; F[2][2] = q24;
    F[4][0] = q14; F[4][1] = q24; F[4][2] = q44 + p;
    T qq = invrho * (Q[3] + p);
    F[3][0] = Q[1] * qq; F[3][1] = Q[2] * qq; F[3][2] = Q[4] * qq;
  } else if constexpr (LAW == DGP_LAW_MAXWELL2D) {  // Maxwell2d::Fi, MaxwellLaw.cc:21-37, Q = (Hx, Hy, Ez)
    F[0][0] = 0;     F[0][1] = Q[2];
    F[1][0] = -Q[2]; F[1][1] = 0;
    F[2][0] = -Q[1]; F[2][1] = Q[0];
  } else {  // 3D Maxwell, eps = mu = 1: dE/dt = curl H, dH/dt = -curl E, so
            // F_E e_i = -(e_i x H) and F_H e_i = e_i x E
    const T *E = Q, *H = Q + 3;
    F[0][0] = 0;     F[0][1] = -H[2]; F[0][2] = H[1];
    F[1][0] = H[2];  F[1][1] = 0;     F[1][2] = -H[0];
    F[2][0] = -H[1]; F[2][1] = H[0];  F[2][2] = 0;
    F[3][0] = 0;     F[3][1] = E[2];  F[3][2] = -E[1];
    F[4][0] = -E[2]; F[4][1] = 0;     F[4][2] = E[0];
    F[5][0] = E[1];  F[5][1] = -E[0]; F[5][2] = 0;
  }
}

template <typename T>
__device__ __forceinline__ T tmax(T a, T b) { return a > b ? a : b; }

// 1 / sqrt(x) (the hardware reciprocal square root with its refinement; the
// adjoint's dual numbers bring their own rsqrt)
__device__ __forceinline__ double inv_sqrt(double x) { return ::rsqrt(x); }
__device__ __forceinline__ float inv_sqrt(float x) { return ::rsqrtf(x); }
template <typename T>
__device__ __forceinline__ T inv_sqrt(const T& x) { return rsqrt(x); }

// Euler::riemann, EulerLaw.cc:610-810: exact Riemann solver, Newton on p*
// from the two-shock guess, <= 12 iterations to relative 1e-14.
template <typename T>
__device__ __noinline__ void exact_riemann(T gamma, T rhol, T ulft, T vlft, T wlft, T plft, T rhor,
                                           T urght, T vrght, T wrght, T prght, T* rhoav, T* uav,
                                           T* vav, T* wav, T* pav) {
  const T one = 1, half = 0.5;
  const T RIEM_TOL = (T)1e-14, SMALLP = (T)1e-14;
  const T rhol_inv = one / rhol, rhor_inv = one / rhor, gm1 = gamma - one;
  T clft, crght, tmp1;
  tmp1 = gamma * plft * rhol_inv;
  if (tmp1 < 0) tmp1 = fabs(tmp1);
  clft = sqrt(tmp1);
  tmp1 = gamma * prght * rhor_inv;
  if (tmp1 < 0) tmp1 = fabs(tmp1);
  crght = sqrt(tmp1);
  if (ulft >= clft && urght >= crght) {
    *rhoav = rhol; *uav = ulft; *vav = vlft; *wav = wlft; *pav = plft;
    return;
  } else if (urght <= -crght && ulft <= -clft) {
    *rhoav = rhor; *uav = urght; *vav = vrght; *wav = wrght; *pav = prght;
    return;
  }
  T tmp2, scrch1, pstar, ustar, rhostar, cstar, rhos, us, ps, cs, prevpstar, relpstar;
  T flft, dflft, frght, dfrght;
  const T invgamma = one / gamma, gp1 = gamma + one;
  const T C3 = half * gm1 * invgamma, C4 = (T)2 / gm1;
  T udiff = urght - ulft;
  T p0 = half * (plft + prght) - (T)0.125 * udiff * (rhol + rhor) * (clft + crght);
  p0 = tmax(SMALLP, p0);
  T gl = sqrt((T)2 / (rhol * (gm1 * plft + gp1 * p0)));
  T gr = sqrt((T)2 / (rhor * (gm1 * prght + gp1 * p0)));
  pstar = (gl * plft + gr * prght - udiff) / (gl + gr);
  relpstar = RIEM_TOL;
  pstar = tmax(RIEM_TOL, pstar);
  prevpstar = pstar;
  for (int i = 0; i < 12 && relpstar >= RIEM_TOL; i++) {
    if (pstar > plft) {
      tmp1 = one / (gp1 * pstar + gm1 * plft);
      tmp2 = sqrt((T)2 * tmp1 * rhol_inv);
      flft = (pstar - plft) * tmp2;
      dflft = tmp2 * (one - half * gp1 * (pstar - plft) * tmp1);
    } else {
      tmp2 = pow(pstar / plft, C3);
      flft = C4 * clft * (tmp2 - one);
      dflft = tmp2 * clft * invgamma / pstar;
    }
    if (pstar > prght) {
      tmp1 = one / (gp1 * pstar + gm1 * prght);
      tmp2 = sqrt((T)2 * tmp1 * rhor_inv);
      frght = (pstar - prght) * tmp2;
      dfrght = tmp2 * (one - half * gp1 * (pstar - prght) * tmp1);
    } else {
      tmp2 = pow(pstar / prght, C3);
      frght = C4 * crght * (tmp2 - one);
      dfrght = tmp2 * crght * invgamma / pstar;
    }
    pstar -= (flft + frght + udiff) / (dflft + dfrght);
    pstar = tmax(SMALLP, pstar);
    relpstar = fabs(pstar - prevpstar) / (half * (prevpstar + pstar));
    prevpstar = pstar;
  }
  if (pstar > plft) flft = (pstar - plft) * sqrt((T)2 * rhol_inv / (gp1 * pstar + gm1 * plft));
  else flft = C4 * clft * (pow(pstar / plft, C3) - one);
  if (pstar > prght) frght = (pstar - prght) * sqrt((T)2 * rhor_inv / (gp1 * pstar + gm1 * prght));
  else frght = C4 * crght * (pow(pstar / prght, C3) - one);
  ustar = (ulft + urght + frght - flft) * half;
  if (ustar >= 0) {
    ps = plft; us = ulft; *vav = vlft; *wav = wlft; rhos = rhol; cs = clft; scrch1 = one;
  } else {
    ps = prght; us = urght; *vav = vrght; *wav = wrght; rhos = rhor; cs = crght; scrch1 = -one;
  }
  if (pstar >= ps) {
    T C = gm1 / gp1;
    tmp1 = pstar / ps;
    *rhoav = rhos * (tmp1 + C) / (C * tmp1 + one);
    *uav = ustar;
    *pav = pstar;
  } else {
    rhostar = rhos * pow(pstar / ps, invgamma);
    cstar = sqrt(gamma * pstar / rhostar);
    if ((ustar - scrch1 * cstar) * ustar <= 0) {
      *rhoav = rhostar; *uav = ustar; *pav = pstar;
    } else {
      T C = (T)2 / gp1;
      tmp1 = C + scrch1 * gm1 * us / (cs * gp1);
      *rhoav = rhos * pow(tmp1, C4);
      *uav = C * (gm1 * half * us + scrch1 * cs);
      *pav = ps * pow(tmp1, C4 * gamma);
    }
  }
}

// ---- numerical flux F(n, uL, uR) . n (ConservationLaw::riemannSolver) --------
template <int LAW, int FLUX, int DIM, typename T>
__device__ __forceinline__ void numerical_flux(const LawParams& lp, const T* n, const T* u0,
                                               const T* u1, T* flux) {
  constexpr int M = LawTraits<LAW>::M;
  if constexpr (LAW == DGP_LAW_SCALAR) {  // ScalarLaw::riemannSolver, ScalarLaw.cc:115-134
    T vn = 0;
    for (int i = 0; i < DIM; ++i) vn += n[i] * (T)lp.p[i];
    T u = (vn > 0) ? u0[0] : u1[0];
    T f = 0;
    for (int i = 0; i < DIM; ++i) f += ((T)lp.p[i] * u) * n[i];
    flux[0] = f;
  } else if constexpr (LAW == DGP_LAW_BURGERS2D) {  // Burgers2D.cc:58-84 (central), or LLF
    T lam = 0;
    if constexpr (FLUX == DGP_FLUX_LLF) lam = tmax(fabs(u0[0]), fabs(u1[0])) * fabs(n[0] + n[1]);
    flux[0] = (T)0.5 * ((u0[0] * u0[0] + u1[0] * u1[0]) * (n[0] + n[1]) * (T)0.5 - lam * (u1[0] - u0[0]));
  } else if constexpr (LAW == DGP_LAW_EULER2D) {
    const T g = (T)lp.p[7];
    if constexpr (FLUX == DGP_FLUX_ROE) {  // Euler2dRoe::riemannSolver, EulerLaw.cc:913-1010
      // the reference's arithmetic, with its square roots and reciprocals of
      // the densities and of the sound speed taken from reciprocal square
      // roots (one hardware operation each instead of a square root and a
      // division): results agree to a few ulps
      T rho_0 = u0[0], rho_1 = u1[0];
      const T is0 = inv_sqrt(rho_0), is1 = inv_sqrt(rho_1);
      T sqrt_rho_0 = rho_0 * is0, sqrt_rho_1 = rho_1 * is1;
      T inv_rho_0 = is0 * is0, inv_rho_1 = is1 * is1;
      T rho_A = sqrt_rho_0 * sqrt_rho_1;
      const T inv_rho_A = is0 * is1;
      T inv_denom = (T)1 / (sqrt_rho_0 + sqrt_rho_1);
      T u_0 = u0[1] * inv_rho_0, u_1 = u1[1] * inv_rho_1;
      T u_A = (u_0 * sqrt_rho_0 + u_1 * sqrt_rho_1) * inv_denom;
      T v_0 = u0[2] * inv_rho_0, v_1 = u1[2] * inv_rho_1;
      T v_A = (v_0 * sqrt_rho_0 + v_1 * sqrt_rho_1) * inv_denom;
      T p_0 = (g - (T)1) * (u0[3] - (T)0.5 * (u0[1] * u0[1] + u0[2] * u0[2]) * inv_rho_0);
      T p_1 = (g - (T)1) * (u1[3] - (T)0.5 * (u1[1] * u1[1] + u1[2] * u1[2]) * inv_rho_1);
      T H_0 = (u0[3] + p_0) * inv_rho_0, H_1 = (u1[3] + p_1) * inv_rho_1;
      T H_A = (H_0 * sqrt_rho_0 + H_1 * sqrt_rho_1) * inv_denom;
      T qq = H_A - (T)0.5 * (u_A * u_A + v_A * v_A);
      T roe[4] = {0, 0, 0, 0};
      if (qq > 0) {
        const T c2 = (g - (T)1) * qq;
        T inv_c_A = inv_sqrt(c2);
        T c_A = c2 * inv_c_A;
        T vn = u_A * n[0] + v_A * n[1];
        T ev[4] = {fabs(vn), fabs(vn), fabs(vn + c_A), fabs(vn - c_A)};
        T k = (T)0.5 * rho_A * inv_c_A;
        T evec[4][4] = {
            {(T)1, u_A, v_A, (T)0.5 * (u_A * u_A + v_A * v_A)},
            {(T)0, n[1] * rho_A, -n[0] * rho_A, rho_A * (u_A * n[1] - v_A * n[0])},
            {k, k * (u_A + c_A * n[0]), k * (v_A + c_A * n[1]), k * (H_A + c_A * vn)},
            {k, k * (u_A - c_A * n[0]), k * (v_A - c_A * n[1]), k * (H_A - c_A * vn)}};
        T drho = rho_1 - rho_0, dp = p_1 - p_0, du = u_1 - u_0, dv = v_1 - v_0;
        const T dpc = dp * inv_rho_A * inv_c_A;
        T charv[4] = {drho - dp * inv_c_A * inv_c_A, n[1] * du - n[0] * dv,
                      n[0] * du + n[1] * dv + dpc, -n[0] * du - n[1] * dv + dpc};
#pragma unroll
        for (int i = 0; i < 4; i++)
#pragma unroll
          for (int j = 0; j < 4; j++) roe[j] += ev[i] * charv[i] * evec[i][j];
      }
      // Euler2d::Fi of both states with the reciprocals above
      T f1[M][DIM], f2[M][DIM];
      euler2d_flux_inv<T>(g, u0, inv_rho_0, f1);
      euler2d_flux_inv<T>(g, u1, inv_rho_1, f2);
#pragma unroll
      for (int i = 0; i < 4; i++)
        flux[i] = (T)0.5 * ((f1[i][0] + f2[i][0]) * n[0] + (f1[i][1] + f2[i][1]) * n[1] - roe[i]);
    } else if constexpr (FLUX == DGP_FLUX_LLF) {
      // local Lax-Friedrichs, lambda = Euler2d::maximumEigenValue(n, UL, UR)
      // (EulerLaw.cc:1022-1034)
      T rho_inv = (T)1 / u0[0];
      T p = (g - (T)1) * (u0[3] - (T)0.5 * (u0[1] * u0[1] + u0[2] * u0[2]) * rho_inv);
      T l1 = sqrt(g * p * rho_inv) + fabs((u0[1] * n[0] + u0[2] * n[1]) * rho_inv);
      rho_inv = (T)1 / u1[0];
      p = (g - (T)1) * (u1[3] - (T)0.5 * (u1[1] * u1[1] + u1[2] * u1[2]) * rho_inv);
      T l2 = sqrt(g * p * rho_inv) + fabs((u1[1] * n[0] + u1[2] * n[1]) * rho_inv);
      T lam = l1 > l2 ? l1 : l2;
      T f1[M][DIM], f2[M][DIM];
      volume_flux<LAW, DIM, T>(lp, u0, f1);
      volume_flux<LAW, DIM, T>(lp, u1, f2);
#pragma unroll
      for (int i = 0; i < 4; i++)
        flux[i] = (T)0.5 * ((f1[i][0] * n[0] + f1[i][1] * n[1]) + (f2[i][0] * n[0] + f2[i][1] * n[1])) -
                  (T)0.5 * lam * (u1[i] - u0[i]);
    } else {  // Euler2d::riemannSolver, EulerLaw.cc:812-851 (exact solver)
      T vn1 = n[0] * (u0[1] / u0[0]) + n[1] * (u0[2] / u0[0]);
      T vt1 = n[1] * (u0[1] / u0[0]) - n[0] * (u0[2] / u0[0]);
      T vn2 = n[0] * (u1[1] / u1[0]) + n[1] * (u1[2] / u1[0]);
      T vt2 = n[1] * (u1[1] / u1[0]) - n[0] * (u1[2] / u1[0]);
      T p1 = (g - (T)1) * u0[3] - (T)0.5 * (g - (T)1) * (u0[1] * u0[1] + u0[2] * u0[2]) / u0[0];
      T p2 = (g - (T)1) * u1[3] - (T)0.5 * (g - (T)1) * (u1[1] * u1[1] + u1[2] * u1[2]) / u1[0];
      T vnav, vtav, dummy, pav, ra[4];
      exact_riemann<T>(g, u0[0], vn1, vt1, (T)0, p1, u1[0], vn2, vt2, (T)0, p2, &ra[0], &vnav, &vtav,
                       &dummy, &pav);
      ra[1] = ra[0] * (n[0] * vnav + n[1] * vtav);
      ra[2] = ra[0] * (n[1] * vnav - n[0] * vtav);
      ra[3] = ((T)1 / (g - (T)1)) * (pav + (T)0.5 * (g - (T)1) * ra[0] * (vnav * vnav + vtav * vtav));
      T f[M][DIM];
      volume_flux<LAW, DIM, T>(lp, ra, f);
#pragma unroll
      for (int i = 0; i < 4; ++i) flux[i] = f[i][0] * n[0] + f[i][1] * n[1];
    }
  } else if constexpr (LAW == DGP_LAW_EULER3D) {  // Euler3d::riemannSolver, EulerLaw.cc:853-911
    const T g = (T)lp.p[7];
    const T n0 = n[0], n1 = n[1], n2 = n[2];
    T t[3] = {n1 + n2, -n0, -n0};
    T tl = sqrt(t[0] * t[0] + t[1] * t[1] + t[2] * t[2]);
    if (tl < (T)0.0000001) { t[0] = -n1; t[1] = n0 + n2; t[2] = -n1; }
    tl = sqrt(t[0] * t[0] + t[1] * t[1] + t[2] * t[2]);
    if (tl < (T)0.0000001) { t[0] = -n2; t[1] = -n2; t[2] = n0 + n1; }
    tl = sqrt(t[0] * t[0] + t[1] * t[1] + t[2] * t[2]);
    t[0] /= tl; t[1] /= tl; t[2] /= tl;
    T sv[3] = {n1 * t[2] - n2 * t[1], n2 * t[0] - n0 * t[2], n0 * t[1] - n1 * t[0]};
    T sl = sqrt(sv[0] * sv[0] + sv[1] * sv[1] + sv[2] * sv[2]);
    sv[0] /= sl; sv[1] /= sl; sv[2] /= sl;
    const T *Ql = u0, *Qr = u1;
    T vnl = (Ql[1] * n0 + Ql[2] * n1 + Ql[4] * n2) / Ql[0];
    T vtl = (Ql[1] * t[0] + Ql[2] * t[1] + Ql[4] * t[2]) / Ql[0];
    T vsl = (Ql[1] * sv[0] + Ql[2] * sv[1] + Ql[4] * sv[2]) / Ql[0];
    T vnr = (Qr[1] * n0 + Qr[2] * n1 + Qr[4] * n2) / Qr[0];
    T vtr = (Qr[1] * t[0] + Qr[2] * t[1] + Qr[4] * t[2]) / Qr[0];
    T vsr = (Qr[1] * sv[0] + Qr[2] * sv[1] + Qr[4] * sv[2]) / Qr[0];
    T pl = (g - (T)1) * (Ql[3] - (T)0.5 * (Ql[1] * Ql[1] + Ql[2] * Ql[2] + Ql[4] * Ql[4]) / Ql[0]);
    T pr = (g - (T)1) * (Qr[3] - (T)0.5 * (Qr[1] * Qr[1] + Qr[2] * Qr[2] + Qr[4] * Qr[4]) / Qr[0]);
    T rhoav, vnav, vtav, vsav, pav;
    exact_riemann<T>(g, Ql[0], vnl, vtl, vsl, pl, Qr[0], vnr, vtr, vsr, pr, &rhoav, &vnav, &vtav, &vsav,
                     &pav);
    flux[0] = rhoav * vnav;
    flux[1] = flux[0] * (n0 * vnav + t[0] * vtav + sv[0] * vsav) + pav * n0;
    flux[2] = flux[0] * (n1 * vnav + t[1] * vtav + sv[1] * vsav) + pav * n1;
    flux[4] = flux[0] * (n2 * vnav + t[2] * vtav + sv[2] * vsav) + pav * n2;
    flux[3] = vnav * (pav / (g - (T)1) + pav + (T)0.5 * rhoav * (vnav * vnav + vtav * vtav + vsav * vsav));
  } else if constexpr (LAW == DGP_LAW_MAXWELL2D) {
    // Maxwell2d::riemannSolver (MaxwellLaw.cc:137-195): the interface state
    // uR2 of its characteristic split, written as the reference condenses it,
    // then Maxwell2d::Fi(uR2) . n
    const T nx = n[0], ny = n[1];
    T uR2[3];
    uR2[0] = (u0[0] + u1[0]) * (nx * ny / (T)2 + ny * ny / (T)2) + (u0[1] + u1[1]) * (nx * nx / (T)2 - nx * ny / (T)2) +
             (u0[2] - u1[2]) * ny / (T)2;
    uR2[1] = (u0[0] + u1[0]) * (-nx * ny / (T)2 + ny * ny / (T)2) +
             (u0[1] + u1[1]) * (nx * nx / (T)2 + nx * ny / (T)2) + (u0[2] - u1[2]) * (-nx) / (T)2;
    uR2[2] = ny * (u0[0] - u1[0]) / (T)2 + nx * (u1[1] - u0[1]) / (T)2 + (u0[2] + u1[2]) / (T)2;
    T f[M][DIM];
    volume_flux<LAW, DIM, T>(lp, uR2, f);
#pragma unroll
    for (int i = 0; i < 3; ++i) flux[i] = f[i][0] * nx + f[i][1] * ny;
  } else {  // Maxwell upwind: F*_E = -n x {H} + n x (n x [E])/2, F*_H = n x {E} + n x (n x [H])/2
    T Ea[3], Ha[3], dE[3], dH[3];
#pragma unroll
    for (int i = 0; i < 3; ++i) {
      Ea[i] = (T)0.5 * (u0[i] + u1[i]);
      Ha[i] = (T)0.5 * (u0[3 + i] + u1[3 + i]);
      dE[i] = u1[i] - u0[i];
      dH[i] = u1[3 + i] - u0[3 + i];
    }
    auto cross = [](const T* a, const T* b, T* o) {
      o[0] = a[1] * b[2] - a[2] * b[1];
      o[1] = a[2] * b[0] - a[0] * b[2];
      o[2] = a[0] * b[1] - a[1] * b[0];
    };
    T nH[3], nE[3], ndE[3], nndE[3], ndH[3], nndH[3];
    cross(n, Ha, nH);
    cross(n, Ea, nE);
    cross(n, dE, ndE);
    cross(n, ndE, nndE);
    cross(n, dH, ndH);
    cross(n, ndH, nndH);
#pragma unroll
    for (int i = 0; i < 3; ++i) {
      flux[i] = -nH[i] + (T)0.5 * nndE[i];
      flux[3 + i] = nE[i] + (T)0.5 * nndH[i];
    }
  }
}

// ---- boundary flux for faces without a right cell (DGCell.cc:696-705) -------
template <int LAW, int FLUX, int DIM, typename T>
__device__ __forceinline__ void boundary_flux(const LawParams& lp, int bid_in, const T* n,
                                              const double* x, double time, const T* Q, T* flux) {
  constexpr int M = LawTraits<LAW>::M;
  const int bid = bc_effective_id(lp, bid_in);
  T f[M];
  if constexpr (LAW == DGP_LAW_SCALAR) {  // ScalarLaw::boundaryFlux, ScalarLaw.cc:85-105
    T nv = 0;
    for (int i = 0; i < DIM; ++i) nv += n[i] * (T)lp.p[i];
    if (nv < 0) {
      field_eval<T>(lp, x, time, f);
      flux[0] = nv * f[0];
    } else {
      flux[0] = nv * Q[0];
    }
  } else if constexpr (LAW == DGP_LAW_BURGERS2D && FLUX == DGP_FLUX_LLF) {
    // Lax-Friedrichs (no counterpart in DG-Parallel): far field as the ghost state
    field_eval<T>(lp, x, time, f);
    numerical_flux<LAW, FLUX, DIM, T>(lp, n, Q, f, flux);
  } else if constexpr (LAW == DGP_LAW_BURGERS2D) {  // Burgers2D::boundaryFlux, Burgers2D.cc:30-54
    T nvel = Q[0] * Q[0] * (T)0.5 * (n[0] + n[1]);
    if (nvel < 0) {
      field_eval<T>(lp, x, time, f);
      flux[0] = f[0] * f[0] * (T)0.5 * (n[0] + n[1]);
    } else {
      flux[0] = nvel;
    }
  } else if constexpr (LAW == DGP_LAW_EULER2D) {
    if (bid == 40000) {  // slip wall mirror state, EulerLaw.cc:280-291
      T vn = -(Q[1] * n[0] + Q[2] * n[1]);
      T vt = Q[1] * n[1] - Q[2] * n[0];
      f[0] = Q[0];
      f[1] = vn * n[0] + vt * n[1];
      f[2] = vn * n[1] - vt * n[0];
      f[3] = Q[3];
    } else {  // far field through the Riemann solver, EulerLaw.cc:293-295
      field_eval<T>(lp, x, time, f);
    }
    numerical_flux<LAW, FLUX, DIM, T>(lp, n, Q, f, flux);
  } else if constexpr (LAW == DGP_LAW_EULER3D) {
    field_eval<T>(lp, x, time, f);
    numerical_flux<LAW, FLUX, DIM, T>(lp, n, Q, f, flux);
  } else if constexpr (LAW == DGP_LAW_MAXWELL2D) {
    // Maxwell2d::boundaryFlux (MaxwellLaw.cc:113-133): reflection on 40000
    // (H mirrored about the face, Ez kept), far field elsewhere, both through
    // the Riemann solver
    if (bid == 40000) {
      const T Hdotn = Q[0] * n[0] + Q[1] * n[1];
      f[0] = -Q[0] + (T)2 * n[0] * Hdotn;
      f[1] = -Q[1] + (T)2 * n[1] * Hdotn;
      f[2] = Q[2];
    } else {
      field_eval<T>(lp, x, time, f);
    }
    numerical_flux<LAW, FLUX, DIM, T>(lp, n, Q, f, flux);
  } else {  // Maxwell: PEC ghost (E -> -E, H -> H) on 40000, far field elsewhere
    if (bid == 40000) {
#pragma unroll
      for (int i = 0; i < 3; ++i) {
        f[i] = -Q[i];
        f[3 + i] = Q[3 + i];
      }
    } else {
      field_eval<T>(lp, x, time, f);
    }
    numerical_flux<LAW, FLUX, DIM, T>(lp, n, Q, f, flux);
  }
}

// ---- maximum eigenvalue at a state (ConservationLaw::maximumEigenValue) -----
template <int LAW, typename T>
__device__ __forceinline__ T max_eigen(const LawParams& lp, const T* Q) {
  if constexpr (LAW == DGP_LAW_SCALAR) {  // ScalarLaw.cc:136-143
    return (T)(fabs(lp.p[0]) + fabs(lp.p[1]) + fabs(lp.p[2]));
  } else if constexpr (LAW == DGP_LAW_EULER2D) {  // EulerLaw.cc:1012-1020
    const T g = (T)lp.p[7];
    T rho_inv = (T)1 / Q[0];
    T v2 = (Q[1] * Q[1] + Q[2] * Q[2]) * rho_inv;
    T p = (g - (T)1) * (Q[3] - (T)0.5 * v2);
    v2 *= rho_inv;
    T c = sqrt(g * p * rho_inv);
    return c + sqrt(v2);
  } else if constexpr (LAW == DGP_LAW_EULER3D) {  // EulerLaw.cc:1160-1168
    const T g = (T)lp.p[7];
    T v2 = (Q[1] * Q[1] + Q[2] * Q[2] + Q[4] * Q[4]) / (Q[0] * Q[0]);
    T p = (g - (T)1) * (Q[3] - (T)0.5 * (Q[1] * Q[1] + Q[2] * Q[2] + Q[4] * Q[4]) / Q[0]);
    T c = sqrt(g * p / Q[0]);
    return c + sqrt(v2);
  } else {  // Burgers2D (Burgers2D.cc:88-92) and Maxwell: 1
    return (T)1;
  }
}

// isPhysical (EulerLaw.cc:1398-1421); the other laws accept every state
template <int LAW, typename T>
__device__ __forceinline__ bool is_physical(const LawParams& lp, const T* Q) {
  if constexpr (LAW == DGP_LAW_EULER2D) {
    const T g = (T)lp.p[7];
    if (Q[0] < 0) return false;
    if ((g - (T)1) * (Q[3] - (T)0.5 * (Q[1] * Q[1] + Q[2] * Q[2]) / Q[0]) < 0) return false;
    return true;
  } else if constexpr (LAW == DGP_LAW_EULER3D) {
    const T g = (T)lp.p[7];
    if (Q[0] < 0) return false;
    if ((g - (T)1) * (Q[3] - (T)0.5 * (Q[1] * Q[1] + Q[2] * Q[2] + Q[4] * Q[4]) / Q[0]) < 0) return false;
    return true;
  } else {
    return true;
  }
}

// A sufficient condition for isPhysical at every point of a cell: each field
// stays within B[j] of mean[j] (B from the modes k >= 1 and the largest basis
// values), and density and pressure keep a relative margin far above the
// rounding of a value evaluated point by point.  False means "evaluate the
// points"; laws without a physical range always pass.
template <int LAW, typename T>
__device__ __forceinline__ bool physical_bound(const LawParams& lp, const T* mean, const T* B) {
  if constexpr (LAW == DGP_LAW_EULER2D || LAW == DGP_LAW_EULER3D) {
    constexpr T tol = sizeof(T) == 8 ? (T)1e-9 : (T)1e-3;
    const T rho = mean[0] - B[0] - tol * (fabs(mean[0]) + B[0]);
    if (!(rho > (T)0)) return false;
    const T m1 = fabs(mean[1]) + B[1], m2 = fabs(mean[2]) + B[2];
    T mm = m1 * m1 + m2 * m2;
    if constexpr (LAW == DGP_LAW_EULER3D) {
      const T m3 = fabs(mean[4]) + B[4];
      mm += m3 * m3;
    }
    const T e = mean[3] - B[3] - tol * (fabs(mean[3]) + B[3]);
    return e - (T)0.5 * mm / rho * ((T)1 + tol) > (T)0;
  } else {
    return true;
  }
}

}  // namespace dgp
