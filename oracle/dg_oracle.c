/* C restatement of DG-Parallel's DG right-hand side and SSP-RK3 step.
 *
 * TEST INFRASTRUCTURE ONLY -- the oracle the CUDA path is checked against; the
 * product never links or calls it.  Every routine cites the reference code it
 * restates.  Arithmetic is plain FP64 in the reference's operation order
 * (no FMA contraction on the x86-64 baseline), with the reference's face loop
 * (scatter into both neighbours) rather than the product's gather.
 */
#include "dg_oracle.h"

#include <math.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "../dg-parallel_b200/csrc/quadrature_rules.h"

#define MAXNP 35
#define MAXM 6
#define MAXQ 64

struct or_solver {
  int dim, nvc, nfv, nlf;
  int law, flux, order, field;
  double prm[16];
  double gamma;
  int m, Np;
  /* mesh */
  int nv;
  double* X;   /* [nv][3] */
  int* vid;    /* file vertex ids */
  int E;
  int* cv;     /* [E][nvc] vertex index, file order of the cell's nodes */
  int ctag;    /* domain tag of the cells */
  int F;
  int* fv;     /* [F][nfv] face vertices in the left cell's local-face order */
  int *eL, *eR, *lfL, *lfR, *bid;
  /* geometry (FP64) */
  double* jac;   /* [E][9] rows d x / d xi_r  (Mapping.cc jacInverse convention) */
  double* jinv;  /* [E][9] inverse of jac */
  double* det;   /* [E] |det jac| */
  double* csize; /* [E] cell size of DGCell::computeCellSize */
  double* fn;    /* [F][3] unit normal, outward from the left cell */
  double* fmeas; /* [F] face measure */
  /* basis */
  double G[MAXNP][MAXNP];
  int mono[MAXNP][3];
  double phi0;
  /* volume rule of degree 2p */
  int nq;
  double qp[MAXQ][3], qw[MAXQ], phi[MAXQ][MAXNP], dphi[MAXQ][3][MAXNP];
  /* face rule of degree 2p+1 (edge: Gauss-Legendre on [-1,1]; tet face: triangle) */
  int nqf;
  double fqp[MAXQ][2], fqw[MAXQ];
  double *trL, *trR; /* [F][nqf][Np] basis traces at the face points */
  double *fx;        /* [F][nqf][3] physical face points */
  double *fjw;       /* [F][nqf] |J_f| * weight */
  /* state */
  double *C, *R, *soln;
  /* triangle moment limiter and P0 fallback (off unless enabled) */
  int limiter, p0;
  int* nb;             /* [E][4] neighbours left, right, bottom, top (-1: none) */
  double* bbc;         /* [E][2] bounding-box centres */
  double Dn[64], Dinv[64]; /* per degree n: (n+1)^2 block at n(n+1)(2n+1)/6 */
  double* L;           /* limited state */
  unsigned char* trig; /* [E] trigger degree of the last limiter application */
  unsigned char* bad;  /* [E] P0 fallback marks */
  int* pcell;          /* [F] periodic partner's cell of a boundary face (-1: none) */
  /* local time stepping (or_lts_setup) */
  int lts_nb;          /* number of size bins, 0: off */
  int *lts_bin, *lts_role, *lts_fcls; /* [E] bin, [E] role, [F] face class */
  double *lts_c1, *lts_save, *lts_r;  /* copy slot, saved u_n, RHS accumulator */
};

static void build_limiter_tables(or_solver* s);
static void build_limiter_geometry(or_solver* s);

/* ------------------------------------------------------------------------ */
/* glibc rand(): srand(seed) then the first rand(), restating the published   */
/* TYPE_3 additive generator (r[i] = r[i-3] + r[i-31], 344 warm-up outputs,   */
/* result r >> 1).  DG-Parallel keys entities by sum of this over vertex ids  */
/* (Vertex::getRAND, Vertex.cc:26-31; mEntity::computeId, mEntity.cc:248).    */
unsigned int or_glibc_rand_first(unsigned int seed) {
  int32_t r[345];
  r[0] = (int32_t)(seed ? seed : 1);
  for (int i = 1; i < 31; ++i) {
    int64_t hi = r[i - 1] / 127773, lo = r[i - 1] % 127773;
    int64_t w = 16807 * lo - 2836 * hi;
    if (w < 0) w += 2147483647;
    r[i] = (int32_t)w;
  }
  for (int i = 31; i < 34; ++i) r[i] = r[i - 31];
  for (int i = 34; i < 345; ++i) r[i] = (int32_t)((uint32_t)r[i - 31] + (uint32_t)r[i - 3]);
  return ((uint32_t)r[344]) >> 1;
}

/* ------------------------------------------------------------------------ */
/* orthonormal basis: Gram-Schmidt of monomials on the reference simplex in   */
/* DG-Parallel's monomial order (SHF::PascalgetFct ShapeFunctionList.cc:311,  */
/* SHF::getTetFct :666) with the inner product int_ref a b (comment at        */
/* ShapeFunctionList.cc:46-95).  Computed here in long double; DG-Parallel    */
/* ships the same basis as truncated decimal tables (OrthoSFTri.h, TetOrtho.h).*/
static const int kTriMono[15][2] = {{0, 0}, {1, 0}, {0, 1}, {2, 0}, {1, 1}, {0, 2}, {3, 0}, {2, 1},
                                    {1, 2}, {0, 3}, {4, 0}, {3, 1}, {2, 2}, {1, 3}, {0, 4}};
static const int kTetMono[35][3] = {
    {0, 0, 0}, {1, 0, 0}, {0, 1, 0}, {0, 0, 1}, {2, 0, 0}, {0, 2, 0}, {0, 0, 2}, {1, 1, 0}, {1, 0, 1},
    {0, 1, 1}, {3, 0, 0}, {0, 3, 0}, {0, 0, 3}, {2, 1, 0}, {2, 0, 1}, {1, 2, 0}, {0, 2, 1}, {1, 0, 2},
    {0, 1, 2}, {1, 1, 1}, {4, 0, 0}, {0, 4, 0}, {0, 0, 4}, {3, 1, 0}, {3, 0, 1}, {1, 3, 0}, {0, 3, 1},
    {1, 0, 3}, {0, 1, 3}, {2, 2, 0}, {2, 0, 2}, {0, 2, 2}, {2, 1, 1}, {1, 2, 1}, {1, 1, 2}};

static long double fact(int n) {
  long double r = 1;
  for (int i = 2; i <= n; ++i) r *= i;
  return r;
}

static void build_basis(or_solver* s) {
  int N = s->Np, d = s->dim;
  for (int i = 0; i < N; ++i)
    for (int k = 0; k < 3; ++k)
      s->mono[i][k] = (k < d) ? (d == 2 ? kTriMono[i][k] : kTetMono[i][k]) : 0;
  static long double M[MAXNP][MAXNP], V[MAXNP][MAXNP];
  for (int i = 0; i < N; ++i)
    for (int j = 0; j < N; ++j) {
      int e[3], tot = 0;
      long double num = 1;
      for (int k = 0; k < 3; ++k) {
        e[k] = s->mono[i][k] + s->mono[j][k];
        num *= fact(e[k]);
        tot += e[k];
      }
      M[i][j] = num / fact(tot + d);
    }
  for (int i = 0; i < N; ++i) {
    for (int j = 0; j < N; ++j) V[i][j] = (i == j) ? 1.0L : 0.0L;
    for (int pass = 0; pass < 2; ++pass)
      for (int j = 0; j < i; ++j) {
        long double p = 0;
        for (int a = 0; a < N; ++a)
          for (int b = 0; b < N; ++b) p += V[i][a] * V[j][b] * M[a][b];
        for (int a = 0; a < N; ++a) V[i][a] -= p * V[j][a];
      }
    long double nn = 0;
    for (int a = 0; a < N; ++a)
      for (int b = 0; b < N; ++b) nn += V[i][a] * V[i][b] * M[a][b];
    long double inv = 1.0L / sqrtl(nn);
    for (int a = 0; a < N; ++a) V[i][a] *= inv;
  }
  for (int i = 0; i < N; ++i)
    for (int j = 0; j < N; ++j) s->G[i][j] = (double)V[i][j];
}

static double mono_val(const int* e, const double* x) {
  double r = 1;
  for (int k = 0; k < 3; ++k)
    for (int p = 0; p < e[k]; ++p) r *= x[k];
  return r;
}

static double mono_der(const int* e, const double* x, int dir) {
  if (e[dir] == 0) return 0.0;
  double r = e[dir];
  for (int k = 0; k < 3; ++k) {
    int p = e[k] - (k == dir);
    for (int q = 0; q < p; ++q) r *= x[k];
  }
  return r;
}

static void basis_eval(const or_solver* s, const double* x, double* f) {
  for (int i = 0; i < s->Np; ++i) {
    double r = 0.0;
    for (int j = 0; j <= i; ++j) r += mono_val(s->mono[j], x) * s->G[i][j];
    f[i] = r;
  }
}

static void basis_grad(const or_solver* s, const double* x, double g[3][MAXNP]) {
  for (int dir = 0; dir < 3; ++dir)
    for (int i = 0; i < s->Np; ++i) {
      double r = 0.0;
      if (dir < s->dim)
        for (int j = 0; j <= i; ++j) r += mono_der(s->mono[j], x, dir) * s->G[i][j];
      g[dir][i] = r;
    }
}

/* ------------------------------------------------------------------------ */
/* analytic fields (initial condition, far field, exact solution)            */
static const double kPi = 3.14159265358979323846;

void or_field_eval(const or_solver* s, const double* x, double t, double* q) {
  const double* p = s->prm;
  switch (s->field) {
    case OR_FIELD_GAUSS: {
      double dx = x[0] - p[0] * t - p[3], dy = x[1] - p[1] * t - p[4];
      q[0] = exp(-(dx * dx + dy * dy) / p[6]);
      break;
    }
    case OR_FIELD_GAUSS3D: {
      double dx = x[0] - p[0] * t - p[3], dy = x[1] - p[1] * t - p[4], dz = x[2] - p[2] * t - p[5];
      q[0] = exp(-(dx * dx + dy * dy + dz * dz) / p[6]);
      break;
    }
    case OR_FIELD_VORTEX: {
      /* isentropic vortex, free stream (1,1,1,1), advected with (1,1) */
      const double g = p[7], b = p[8];
      double dx = x[0] - (p[3] + t), dy = x[1] - (p[4] + t);
      double r2 = dx * dx + dy * dy;
      double e = exp(0.5 * (1.0 - r2));
      double u = 1.0 - b / (2.0 * kPi) * e * dy;
      double v = 1.0 + b / (2.0 * kPi) * e * dx;
      double T = 1.0 - (g - 1.0) * b * b / (8.0 * g * kPi * kPi) * e * e;
      double rho = pow(T, 1.0 / (g - 1.0));
      double pr = pow(rho, g);
      q[0] = rho;
      q[1] = rho * u;
      q[2] = rho * v;
      q[3] = pr / (g - 1.0) + 0.5 * rho * (u * u + v * v);
      break;
    }
    case OR_FIELD_PULSE3D: {
      /* Euler3d field order (rho, rho u, rho v, E, rho w) */
      double dx = x[0] - p[0] * t - p[3], dy = x[1] - p[1] * t - p[4], dz = x[2] - p[2] * t - p[5];
      double rho = 1.0 + 0.2 * exp(-(dx * dx + dy * dy + dz * dz) / p[6]);
      q[0] = rho;
      q[1] = rho * p[0];
      q[2] = rho * p[1];
      q[4] = rho * p[2];
      q[3] = 1.0 / (p[7] - 1.0) + 0.5 * rho * (p[0] * p[0] + p[1] * p[1] + p[2] * p[2]);
      break;
    }
    case OR_FIELD_SINE:
      q[0] = 0.5 + p[9] * sin(2.0 * kPi * (x[0] + x[1]));
      break;
    case OR_FIELD_TM2D: {
      /* the TM mode Ez = sin(pi x/L) sin(pi y/L) cos(w t) of Maxwell2d's
       * equations, fields (Hx, Hy, Ez) */
      double L = p[10] > 0 ? p[10] : 1.0;
      double k = kPi / L, w = kPi * sqrt(2.0) / L;
      double sx = sin(k * x[0]), cx = cos(k * x[0]), sy = sin(k * x[1]), cy = cos(k * x[1]);
      q[0] = -(k / w) * sx * cy * sin(w * t);
      q[1] = (k / w) * cx * sy * sin(w * t);
      q[2] = sx * sy * cos(w * t);
      break;
    }
    case OR_FIELD_TM110: {
      /* TM110 mode of the PEC cube [0,L]^3: fields (Ex,Ey,Ez,Hx,Hy,Hz) */
      double L = p[10] > 0 ? p[10] : 1.0;
      double k = kPi / L, w = kPi * sqrt(2.0) / L;
      double sx = sin(k * x[0]), cx = cos(k * x[0]), sy = sin(k * x[1]), cy = cos(k * x[1]);
      q[0] = 0.0;
      q[1] = 0.0;
      q[2] = sx * sy * cos(w * t);
      q[3] = -(k / w) * sx * cy * sin(w * t);
      q[4] = (k / w) * cx * sy * sin(w * t);
      q[5] = 0.0;
      break;
    }
    default:
      for (int j = 0; j < s->m; ++j) q[j] = 0.0;
  }
}

/* ------------------------------------------------------------------------ */
/* conservation laws                                                          */
static void law_flux(const or_solver* s, const double* x, const double* Q, double F[MAXM][3]) {
  const double g = s->gamma;
  switch (s->law) {
    case OR_SCALAR: /* ScalarLaw::Fi, ScalarLaw.cc:75-83 */
      F[0][0] = s->prm[0] * Q[0];
      F[0][1] = s->prm[1] * Q[0];
      F[0][2] = s->prm[2] * Q[0];
      break;
    case OR_BURGERS2D: /* Burgers2D::Fi, Burgers2D.cc:22-28 */
      F[0][0] = Q[0] * Q[0] * 0.5;
      F[0][1] = Q[0] * Q[0] * 0.5;
      F[0][2] = 0.0;
      break;
    case OR_EULER2D: { /* Euler2d::Fi, EulerLaw.cc:47-69 */
      double invrho = 1. / Q[0];
      double Q1 = Q[1], Q2 = Q[2];
      double q12 = Q1 * Q2 * invrho, q11 = Q1 * Q1 * invrho, q22 = Q2 * Q2 * invrho;
      double p = (g - 1.) * (Q[3] - 0.5 * (q11 + q22));
      double qq = invrho * (Q[3] + p);
      F[0][0] = Q1; F[0][1] = Q2; F[0][2] = 0.0;
      F[1][0] = q11 + p; F[1][1] = q12; F[1][2] = 0.0;
      F[2][0] = q12; F[2][1] = q22 + p; F[2][2] = 0.0;
      F[3][0] = Q1 * qq; F[3][1] = Q2 * qq; F[3][2] = 0.0;
      break;
    }
    case OR_EULER3D: { /* Euler3d::Fi, EulerLaw.cc:81-107 */
      double invrho = 1. / Q[0];
      double q11 = Q[1] * Q[1] * invrho, q12 = Q[1] * Q[2] * invrho, q14 = Q[1] * Q[4] * invrho;
      double q22 = Q[2] * Q[2] * invrho, q24 = Q[2] * Q[4] * invrho, q44 = Q[4] * Q[4] * invrho;
      double p = (g - 1.) * (Q[3] - 0.5 * (Q[1] * Q[1] + Q[2] * Q[2] + Q[4] * Q[4]) / Q[0]);
      F[0][0] = Q[1]; F[0][1] = Q[2]; F[0][2] = Q[4];
      F[1][0] = q11 + p; F[1][1] = q12; F[1][2] = q14;
      F[2][0] = q12; F[2][1] = q22 + p; F[2][2] = q24;
      F[4][0] = q14; F[4][1] = q24; F[4][2] = q44 + p;
      double qq = invrho * (Q[3] + p);
      F[3][0] = Q[1] * qq; F[3][1] = Q[2] * qq; F[3][2] = Q[4] * qq;
      break;
    }
    case OR_MAXWELL2D: /* Maxwell2d::Fi, MaxwellLaw.cc:21-37, Q = (Hx, Hy, Ez) */
      F[0][0] = 0.0;   F[0][1] = Q[2];  F[0][2] = 0.0;
      F[1][0] = -Q[2]; F[1][1] = 0.0;   F[1][2] = 0.0;
      F[2][0] = -Q[1]; F[2][1] = Q[0];  F[2][2] = 0.0;
      break;
    case OR_MAXWELL3D: {
      /* dE/dt - curl H = 0, dH/dt + curl E = 0 (eps = mu = 1):
       * F_E . n = -(n x H), F_H . n = n x E */
      const double *E = Q, *H = Q + 3;
      /* columns i = spatial direction: F[j][i] with unit n = e_i */
      for (int i = 0; i < 3; ++i) {
        double n[3] = {0, 0, 0};
        n[i] = 1.0;
        double nxH[3] = {n[1] * H[2] - n[2] * H[1], n[2] * H[0] - n[0] * H[2], n[0] * H[1] - n[1] * H[0]};
        double nxE[3] = {n[1] * E[2] - n[2] * E[1], n[2] * E[0] - n[0] * E[2], n[0] * E[1] - n[1] * E[0]};
        for (int j = 0; j < 3; ++j) {
          F[j][i] = -nxH[j];
          F[3 + j][i] = nxE[j];
        }
      }
      break;
    }
  }
}

static double dot3(const double* a, const double* n) { return a[0] * n[0] + a[1] * n[1] + a[2] * n[2]; }

/* Euler::riemann, EulerLaw.cc:610-810: exact Riemann solver (Newton on p*,
 * two-shock initial guess, <= 12 iterations to relative 1e-14). */
#define RIEM_TOL 1e-14
#define RIEM_ITER 12
#define SMALLP 1e-14
static void exact_riemann(double gamma, double rhol, double ulft, double vlft, double wlft,
                          double plft, double rhor, double urght, double vrght, double wrght,
                          double prght, double* rhoav, double* uav, double* vav, double* wav,
                          double* pav) {
  const double rhol_inv = 1. / rhol, rhor_inv = 1. / rhor, gm1 = gamma - 1.;
  double clft, crght, tmp1;
  tmp1 = gamma * plft * rhol_inv;
  if (tmp1 < 0.0) tmp1 = fabs(tmp1);
  clft = sqrt(tmp1);
  tmp1 = gamma * prght * rhor_inv;
  if (tmp1 < 0.0) tmp1 = fabs(tmp1);
  crght = sqrt(tmp1);
  if (ulft >= clft && urght >= crght) {
    *rhoav = rhol; *uav = ulft; *vav = vlft; *wav = wlft; *pav = plft;
    return;
  } else if (urght <= -crght && ulft <= -clft) {
    *rhoav = rhor; *uav = urght; *vav = vrght; *wav = wrght; *pav = prght;
    return;
  }
  double tmp2, scrch1, pstar, ustar, rhostar, cstar, rhos, us, ps, cs, prevpstar, relpstar;
  double flft, dflft, frght, dfrght;
  const double invgamma = 1. / gamma, gp1 = gamma + 1.;
  const double C3 = 0.5 * gm1 * invgamma, C4 = 2. / gm1;
  double udiff = urght - ulft;
  double p0 = 0.5 * (plft + prght) - 0.125 * udiff * (rhol + rhor) * (clft + crght);
  p0 = (SMALLP > p0) ? SMALLP : p0;
  double gl = sqrt(2. / (rhol * (gm1 * plft + gp1 * p0)));
  double gr = sqrt(2. / (rhor * (gm1 * prght + gp1 * p0)));
  pstar = (gl * plft + gr * prght - udiff) / (gl + gr);
  relpstar = RIEM_TOL;
  pstar = (RIEM_TOL > pstar) ? RIEM_TOL : pstar;
  prevpstar = pstar;
  for (int i = 0; i < RIEM_ITER && relpstar >= RIEM_TOL; i++) {
    if (pstar > plft) {
      tmp1 = 1. / (gp1 * pstar + gm1 * plft);
      tmp2 = sqrt(2. * tmp1 * rhol_inv);
      flft = (pstar - plft) * tmp2;
      dflft = tmp2 * (1. - 0.5 * gp1 * (pstar - plft) * tmp1);
    } else {
      tmp2 = pow(pstar / plft, C3);
      flft = C4 * clft * (tmp2 - 1.);
      dflft = tmp2 * clft * invgamma / pstar;
    }
    if (pstar > prght) {
      tmp1 = 1. / (gp1 * pstar + gm1 * prght);
      tmp2 = sqrt(2. * tmp1 * rhor_inv);
      frght = (pstar - prght) * tmp2;
      dfrght = tmp2 * (1. - 0.5 * gp1 * (pstar - prght) * tmp1);
    } else {
      tmp2 = pow(pstar / prght, C3);
      frght = C4 * crght * (tmp2 - 1.);
      dfrght = tmp2 * crght * invgamma / pstar;
    }
    pstar -= (flft + frght + udiff) / (dflft + dfrght);
    pstar = (SMALLP > pstar) ? SMALLP : pstar;
    relpstar = fabs(pstar - prevpstar) / (.5 * (prevpstar + pstar));
    prevpstar = pstar;
  }
  if (pstar > plft) flft = (pstar - plft) * sqrt(2. * rhol_inv / (gp1 * pstar + gm1 * plft));
  else flft = C4 * clft * (pow(pstar / plft, C3) - 1.);
  if (pstar > prght) frght = (pstar - prght) * sqrt(2. * rhor_inv / (gp1 * pstar + gm1 * prght));
  else frght = C4 * crght * (pow(pstar / prght, C3) - 1.);
  ustar = (ulft + urght + frght - flft) * 0.5;
  if (ustar >= 0) {
    ps = plft; us = ulft; *vav = vlft; *wav = wlft; rhos = rhol; cs = clft; scrch1 = 1.;
  } else {
    ps = prght; us = urght; *vav = vrght; *wav = wrght; rhos = rhor; cs = crght; scrch1 = -1.;
  }
  if (pstar >= ps) {
    double C = gm1 / gp1;
    tmp1 = pstar / ps;
    *rhoav = rhos * (tmp1 + C) / (C * tmp1 + 1.);
    *uav = ustar;
    *pav = pstar;
  } else {
    rhostar = rhos * pow(pstar / ps, invgamma);
    cstar = sqrt(gamma * pstar / rhostar);
    if ((ustar - scrch1 * cstar) * ustar <= 0.0) {
      *rhoav = rhostar; *uav = ustar; *pav = pstar;
    } else {
      double C = 2. / gp1;
      tmp1 = C + scrch1 * gm1 * us / (cs * gp1);
      *rhoav = rhos * pow(tmp1, C4);
      *uav = C * (gm1 * 0.5 * us + scrch1 * cs);
      *pav = ps * pow(tmp1, C4 * gamma);
    }
  }
}

static void riemann_flux(const or_solver* s, const double* n, const double* x, const double* u0,
                         const double* u1, double* flux) {
  const double g = s->gamma;
  switch (s->law) {
    case OR_SCALAR: { /* ScalarLaw::riemannSolver, ScalarLaw.cc:115-134 */
      const double* v = s->prm;
      double vn = (n[0] * v[0] + n[1] * v[1] + n[2] * v[2]);
      double u = (vn > 0) ? u0[0] : u1[0];
      double f[3] = {v[0] * u, v[1] * u, v[2] * u};
      flux[0] = dot3(f, n);
      break;
    }
    case OR_BURGERS2D: {
      if (s->flux == OR_FLUX_LLF) {
        double lam = fmax(fabs(u0[0]), fabs(u1[0])) * fabs(n[0] + n[1]);
        flux[0] = 0.5 * ((u0[0] * u0[0] + u1[0] * u1[0]) * (n[0] + n[1]) * 0.5 - lam * (u1[0] - u0[0]));
      } else { /* Burgers2D::riemannSolver, Burgers2D.cc:58-84: central, maxIV = 0 */
        double maxIV = 0;
        flux[0] = 0.5 * ((u0[0] * u0[0] + u1[0] * u1[0]) * (n[0] + n[1]) * 0.5 - maxIV * (u1[0] - u0[0]));
      }
      break;
    }
    case OR_EULER2D: {
      if (s->flux == OR_FLUX_ROE) { /* Euler2dRoe::riemannSolver, EulerLaw.cc:913-1010 */
        double rho_0 = u0[0], rho_1 = u1[0];
        double sqrt_rho_0 = sqrt(rho_0), sqrt_rho_1 = sqrt(rho_1);
        double inv_rho_0 = 1. / rho_0, inv_rho_1 = 1. / rho_1;
        double rho_A = sqrt_rho_0 * sqrt_rho_1;
        double inv_denom = 1. / (sqrt_rho_0 + sqrt_rho_1);
        double u_0 = u0[1] * inv_rho_0, u_1 = u1[1] * inv_rho_1;
        double u_A = (u_0 * sqrt_rho_0 + u_1 * sqrt_rho_1) * inv_denom;
        double v_0 = u0[2] * inv_rho_0, v_1 = u1[2] * inv_rho_1;
        double v_A = (v_0 * sqrt_rho_0 + v_1 * sqrt_rho_1) * inv_denom;
        double p_0 = (g - 1.) * (u0[3] - 0.5 * (u0[1] * u0[1] + u0[2] * u0[2]) * inv_rho_0);
        double p_1 = (g - 1.) * (u1[3] - 0.5 * (u1[1] * u1[1] + u1[2] * u1[2]) * inv_rho_1);
        double H_0 = (u0[3] + p_0) * inv_rho_0, H_1 = (u1[3] + p_1) * inv_rho_1;
        double H_A = (H_0 * sqrt_rho_0 + H_1 * sqrt_rho_1) * inv_denom;
        double qq = H_A - 0.5 * (u_A * u_A + v_A * v_A);
        double roe[4] = {0, 0, 0, 0};
        if (qq > 0.0) {
          double c_A = sqrt((g - 1.0) * qq);
          double vn = u_A * n[0] + v_A * n[1];
          double evec[4][4], eval[4];
          eval[0] = fabs(vn);
          eval[1] = fabs(vn);
          eval[2] = fabs(vn + c_A);
          eval[3] = fabs(vn - c_A);
          evec[0][0] = 1.; evec[0][1] = u_A; evec[0][2] = v_A; evec[0][3] = 0.5 * (u_A * u_A + v_A * v_A);
          evec[1][0] = 0.; evec[1][1] = n[1] * rho_A; evec[1][2] = -n[0] * rho_A;
          evec[1][3] = rho_A * (u_A * n[1] - v_A * n[0]);
          double k = 0.5 * rho_A / c_A;
          evec[2][0] = k; evec[2][1] = k * (u_A + c_A * n[0]); evec[2][2] = k * (v_A + c_A * n[1]);
          evec[2][3] = k * (H_A + c_A * vn);
          evec[3][0] = k; evec[3][1] = k * (u_A - c_A * n[0]); evec[3][2] = k * (v_A - c_A * n[1]);
          evec[3][3] = k * (H_A - c_A * vn);
          double charv[4];
          double inv_c_A = 1. / c_A;
          double drho = rho_1 - rho_0, dp = p_1 - p_0, du = u_1 - u_0, dv = v_1 - v_0;
          charv[0] = drho - dp * inv_c_A * inv_c_A;
          charv[1] = n[1] * du - n[0] * dv;
          charv[2] = n[0] * du + n[1] * dv + dp / rho_A * inv_c_A;
          charv[3] = -n[0] * du - n[1] * dv + dp / rho_A * inv_c_A;
          for (int i = 0; i < 4; i++)
            for (int j = 0; j < 4; j++) roe[j] += eval[i] * charv[i] * evec[i][j];
        }
        double f1[MAXM][3], f2[MAXM][3];
        law_flux(s, x, u0, f1);
        law_flux(s, x, u1, f2);
        for (int i = 0; i < 4; i++) {
          double sum[3] = {f1[i][0] + f2[i][0], f1[i][1] + f2[i][1], f1[i][2] + f2[i][2]};
          flux[i] = 0.5 * (dot3(sum, n) - roe[i]);
        }
      } else if (s->flux == OR_FLUX_LLF) {
        /* local Lax-Friedrichs with lambda = Euler2d::maximumEigenValue(n,UL,UR)
         * (EulerLaw.cc:1022-1034); not present in DG-Parallel */
        double rho_inv = 1. / u0[0];
        double p = (g - 1.) * (u0[3] - 0.5 * (u0[1] * u0[1] + u0[2] * u0[2]) * rho_inv);
        double c = sqrt(g * p * rho_inv);
        double l1 = c + fabs((u0[1] * n[0] + u0[2] * n[1]) * rho_inv);
        rho_inv = 1. / u1[0];
        p = (g - 1.) * (u1[3] - 0.5 * (u1[1] * u1[1] + u1[2] * u1[2]) * rho_inv);
        c = sqrt(g * p * rho_inv);
        double l2 = c + fabs((u1[1] * n[0] + u1[2] * n[1]) * rho_inv);
        double lam = l1 > l2 ? l1 : l2;
        double f1[MAXM][3], f2[MAXM][3];
        law_flux(s, x, u0, f1);
        law_flux(s, x, u1, f2);
        for (int i = 0; i < 4; i++)
          flux[i] = 0.5 * (dot3(f1[i], n) + dot3(f2[i], n)) - 0.5 * lam * (u1[i] - u0[i]);
      } else { /* Euler2d::riemannSolver, EulerLaw.cc:812-851 */
        double vn1 = n[0] * (u0[1] / u0[0]) + n[1] * (u0[2] / u0[0]);
        double vt1 = n[1] * (u0[1] / u0[0]) - n[0] * (u0[2] / u0[0]);
        double vn2 = n[0] * (u1[1] / u1[0]) + n[1] * (u1[2] / u1[0]);
        double vt2 = n[1] * (u1[1] / u1[0]) - n[0] * (u1[2] / u1[0]);
        double p1 = (g - 1) * u0[3] - 0.5 * (g - 1) * (u0[1] * u0[1] + u0[2] * u0[2]) / u0[0];
        double p2 = (g - 1) * u1[3] - 0.5 * (g - 1) * (u1[1] * u1[1] + u1[2] * u1[2]) / u1[0];
        double vnav, vtav, dummy, pav, ra[4];
        exact_riemann(g, u0[0], vn1, vt1, 0.0, p1, u1[0], vn2, vt2, 0.0, p2, &ra[0], &vnav, &vtav,
                      &dummy, &pav);
        ra[1] = ra[0] * (n[0] * vnav + n[1] * vtav);
        ra[2] = ra[0] * (n[1] * vnav - n[0] * vtav);
        ra[3] = (1. / (g - 1)) * (pav + 0.5 * (g - 1) * ra[0] * (vnav * vnav + vtav * vtav));
        double f[MAXM][3];
        law_flux(s, x, ra, f);
        for (int i = 0; i < 4; ++i) flux[i] = dot3(f[i], n);
      }
      break;
    }
    case OR_EULER3D: { /* Euler3d::riemannSolver, EulerLaw.cc:853-911 */
      const double n0 = n[0], n1 = n[1], n2 = n[2];
      double t[3] = {n1 + n2, -n0, -n0};
      double tl = sqrt(t[0] * t[0] + t[1] * t[1] + t[2] * t[2]);
      if (tl < 0.0000001) { t[0] = -n1; t[1] = n0 + n2; t[2] = -n1; }
      tl = sqrt(t[0] * t[0] + t[1] * t[1] + t[2] * t[2]);
      if (tl < 0.0000001) { t[0] = -n2; t[1] = -n2; t[2] = n0 + n1; }
      tl = sqrt(t[0] * t[0] + t[1] * t[1] + t[2] * t[2]);
      t[0] /= tl; t[1] /= tl; t[2] /= tl;
      double sv[3] = {n1 * t[2] - n2 * t[1], n2 * t[0] - n0 * t[2], n0 * t[1] - n1 * t[0]};
      double sl = sqrt(sv[0] * sv[0] + sv[1] * sv[1] + sv[2] * sv[2]);
      sv[0] /= sl; sv[1] /= sl; sv[2] /= sl;
      const double *Ql = u0, *Qr = u1;
      double vnl = (Ql[1] * n0 + Ql[2] * n1 + Ql[4] * n2) / Ql[0];
      double vtl = (Ql[1] * t[0] + Ql[2] * t[1] + Ql[4] * t[2]) / Ql[0];
      double vsl = (Ql[1] * sv[0] + Ql[2] * sv[1] + Ql[4] * sv[2]) / Ql[0];
      double vnr = (Qr[1] * n0 + Qr[2] * n1 + Qr[4] * n2) / Qr[0];
      double vtr = (Qr[1] * t[0] + Qr[2] * t[1] + Qr[4] * t[2]) / Qr[0];
      double vsr = (Qr[1] * sv[0] + Qr[2] * sv[1] + Qr[4] * sv[2]) / Qr[0];
      double pl = (g - 1.) * (Ql[3] - 0.5 * (Ql[1] * Ql[1] + Ql[2] * Ql[2] + Ql[4] * Ql[4]) / Ql[0]);
      double pr = (g - 1.) * (Qr[3] - 0.5 * (Qr[1] * Qr[1] + Qr[2] * Qr[2] + Qr[4] * Qr[4]) / Qr[0]);
      double rhoav, vnav, vtav, vsav, pav;
      exact_riemann(g, Ql[0], vnl, vtl, vsl, pl, Qr[0], vnr, vtr, vsr, pr, &rhoav, &vnav, &vtav, &vsav,
                    &pav);
      flux[0] = rhoav * vnav;
      flux[1] = flux[0] * (n0 * vnav + t[0] * vtav + sv[0] * vsav) + pav * n0;
      flux[2] = flux[0] * (n1 * vnav + t[1] * vtav + sv[1] * vsav) + pav * n1;
      flux[4] = flux[0] * (n2 * vnav + t[2] * vtav + sv[2] * vsav) + pav * n2;
      flux[3] = vnav * (pav / (g - 1.) + pav + 0.5 * rhoav * (vnav * vnav + vtav * vtav + vsav * vsav));
      break;
    }
    case OR_MAXWELL2D: {
      /* Maxwell2d::riemannSolver, MaxwellLaw.cc:137-195: the interface state of
       * its characteristic split in the reference's condensed form, then
       * Maxwell2d::Fi(uR2) . n */
      const double nx = n[0], ny = n[1];
      double uR2[3], F2[MAXM][3];
      uR2[0] = (u0[0] + u1[0]) * (nx * ny / 2 + ny * ny / 2) + (u0[1] + u1[1]) * (nx * nx / 2 - nx * ny / 2) +
               (u0[2] - u1[2]) * ny / 2;
      uR2[1] = (u0[0] + u1[0]) * (-nx * ny / 2 + ny * ny / 2) + (u0[1] + u1[1]) * (nx * nx / 2 + nx * ny / 2) +
               (u0[2] - u1[2]) * (-nx) / 2;
      uR2[2] = ny * (u0[0] - u1[0]) / 2 + nx * (u1[1] - u0[1]) / 2 + (u0[2] + u1[2]) / 2;
      law_flux(s, x, uR2, F2);
      for (int i = 0; i < 3; ++i) flux[i] = dot3(F2[i], n);
      break;
    }
    case OR_MAXWELL3D: {
      /* upwind flux (eps = mu = 1): F*_E = -n x {H} + 1/2 n x (n x [E]),
       *                             F*_H =  n x {E} + 1/2 n x (n x [H]),
       * {a} = (aL+aR)/2, [a] = aR-aL; |A| is the tangential projector. */
      double Ea[3], Ha[3], dE[3], dH[3];
      for (int i = 0; i < 3; ++i) {
        Ea[i] = 0.5 * (u0[i] + u1[i]);
        Ha[i] = 0.5 * (u0[3 + i] + u1[3 + i]);
        dE[i] = u1[i] - u0[i];
        dH[i] = u1[3 + i] - u0[3 + i];
      }
#define CROSS(a, b, o) do { o[0] = a[1] * b[2] - a[2] * b[1]; o[1] = a[2] * b[0] - a[0] * b[2]; \
                            o[2] = a[0] * b[1] - a[1] * b[0]; } while (0)
      double nH[3], nE[3], ndE[3], nndE[3], ndH[3], nndH[3];
      CROSS(n, Ha, nH);
      CROSS(n, Ea, nE);
      CROSS(n, dE, ndE);
      CROSS(n, ndE, nndE);
      CROSS(n, dH, ndH);
      CROSS(n, ndH, nndH);
#undef CROSS
      for (int i = 0; i < 3; ++i) {
        flux[i] = -nH[i] + 0.5 * nndE[i];
        flux[3 + i] = nE[i] + 0.5 * nndH[i];
      }
      break;
    }
  }
}

/* boundary flux for faces with no right cell (DGCell.cc:696-705 dispatch) */
static void boundary_flux(const or_solver* s, int bid, const double* n, const double* x, double T,
                          const double* Q, double* flux) {
  double f[MAXM];
  switch (s->law) {
    case OR_SCALAR: { /* ScalarLaw::boundaryFlux, ScalarLaw.cc:85-105 */
      const double* v = s->prm;
      double nv = (n[0] * v[0] + n[1] * v[1] + n[2] * v[2]);
      if (nv < 0) {
        or_field_eval(s, x, T, f);
        flux[0] = nv * f[0];
      } else {
        flux[0] = nv * Q[0];
      }
      return;
    }
    case OR_BURGERS2D: { /* Burgers2D::boundaryFlux, Burgers2D.cc:30-54 */
      if (s->flux == OR_FLUX_LLF) { /* LLF (no counterpart): far field as the ghost state */
        or_field_eval(s, x, T, f);
        riemann_flux(s, n, x, Q, f, flux);
        return;
      }
      double nvel = Q[0] * Q[0] * 0.5 * (n[0] + n[1]);
      if (nvel < 0) {
        or_field_eval(s, x, T, f);
        flux[0] = f[0] * f[0] * 0.5 * (n[0] + n[1]);
      } else {
        flux[0] = nvel;
      }
      return;
    }
    case OR_EULER2D:
      if (bid == 40000) { /* slip wall mirror state, EulerLaw.cc:280-291 */
        double vn = -(Q[1] * n[0] + Q[2] * n[1]);
        double vt = Q[1] * n[1] - Q[2] * n[0];
        f[0] = Q[0];
        f[1] = vn * n[0] + vt * n[1];
        f[2] = vn * n[1] - vt * n[0];
        f[3] = Q[3];
        riemann_flux(s, n, x, Q, f, flux);
        return;
      }
      or_field_eval(s, x, T, f); /* far field, EulerLaw.cc:293-295 */
      riemann_flux(s, n, x, Q, f, flux);
      return;
    case OR_EULER3D:
      or_field_eval(s, x, T, f);
      riemann_flux(s, n, x, Q, f, flux);
      return;
    case OR_MAXWELL2D:
      if (bid == 40000) { /* Maxwell2d::boundaryFlux reflection, MaxwellLaw.cc:113-125 */
        double Hdotn = Q[0] * n[0] + Q[1] * n[1];
        f[0] = -Q[0] + 2 * n[0] * Hdotn;
        f[1] = -Q[1] + 2 * n[1] * Hdotn;
        f[2] = Q[2];
      } else { /* far field, MaxwellLaw.cc:126-131 */
        or_field_eval(s, x, T, f);
      }
      riemann_flux(s, n, x, Q, f, flux);
      return;
    case OR_MAXWELL3D:
      if (bid == 40000) { /* perfect electric conductor: ghost E = -E, H = H */
        for (int i = 0; i < 3; ++i) {
          f[i] = -Q[i];
          f[3 + i] = Q[3 + i];
        }
      } else {
        or_field_eval(s, x, T, f);
      }
      riemann_flux(s, n, x, Q, f, flux);
      return;
  }
}

static double max_eigen(const or_solver* s, const double* Q) {
  const double g = s->gamma;
  switch (s->law) {
    case OR_SCALAR: return fabs(s->prm[0]) + fabs(s->prm[1]) + fabs(s->prm[2]);
    case OR_BURGERS2D: return 1.0;
    case OR_EULER2D: { /* EulerLaw.cc:1012-1020 */
      double rho_inv = 1. / Q[0];
      double v2 = (Q[1] * Q[1] + Q[2] * Q[2]) * rho_inv;
      double p = (g - 1.) * (Q[3] - 0.5 * v2);
      v2 *= rho_inv;
      double c = sqrt(g * p * rho_inv);
      return c + sqrt(v2);
    }
    case OR_EULER3D: { /* EulerLaw.cc:1160-1168 */
      double v2 = (Q[1] * Q[1] + Q[2] * Q[2] + Q[4] * Q[4]) / (Q[0] * Q[0]);
      double p = (g - 1.) * (Q[3] - 0.5 * (Q[1] * Q[1] + Q[2] * Q[2] + Q[4] * Q[4]) / Q[0]);
      double c = sqrt(g * p / Q[0]);
      return c + sqrt(v2);
    }
    case OR_MAXWELL3D: return 1.0;
    case OR_MAXWELL2D: return 1.0; /* Maxwell2d::maximumEigenValue, MaxwellLaw.cc:197-200 */
  }
  return 1.0;
}

/* ------------------------------------------------------------------------ */
/* mesh import (Gmsh v1, mImportExport.cc:77-170) and connectivity            */
typedef struct { int v[3]; int cell, lf; } facekey;

static int cmp_facekey(const void* a, const void* b) {
  const facekey *x = a, *y = b;
  for (int i = 0; i < 3; ++i) {
    if (x->v[i] != y->v[i]) return x->v[i] < y->v[i] ? -1 : 1;
  }
  return 0;
}

static void sort_ints(int* a, int n) {
  for (int i = 1; i < n; ++i)
    for (int j = i; j > 0 && a[j - 1] > a[j]; --j) {
      int t = a[j]; a[j] = a[j - 1]; a[j - 1] = t;
    }
}

static const int kTriFace[3][2] = {{0, 1}, {1, 2}, {2, 0}};
static const int kTetFace[4][3] = {{0, 1, 2}, {0, 1, 3}, {0, 2, 3}, {1, 2, 3}};

/* DG-Parallel's order of two cells sharing a face: the cell with the smaller
 * (int) sum of rand(vertex id), then the smaller sorted vertex-id list, is the
 * left one (mEntity::lessthan, mEntity.cc:173-200). */
static int32_t cell_key(const or_solver* s, const uint32_t* rk, int e) {
  uint64_t sum = 0;
  for (int k = 0; k < s->nvc; ++k) sum += rk[s->cv[e * s->nvc + k]];
  return (int32_t)(uint32_t)sum;
}

static int cell_less(const or_solver* s, const uint32_t* rk, int a, int b) {
  int32_t ka = cell_key(s, rk, a), kb = cell_key(s, rk, b);
  if (ka != kb) return ka < kb;
  int va[4], vb[4];
  for (int k = 0; k < s->nvc; ++k) {
    va[k] = s->vid[s->cv[a * s->nvc + k]];
    vb[k] = s->vid[s->cv[b * s->nvc + k]];
  }
  sort_ints(va, s->nvc);
  sort_ints(vb, s->nvc);
  for (int k = 0; k < s->nvc; ++k)
    if (va[k] != vb[k]) return va[k] < vb[k];
  return 0;
}

static int read_msh(or_solver* s, const char* path) {
  FILE* f = fopen(path, "r");
  if (!f) return -1;
  char tok[256];
  int nb = 0, cap_b = 0, ncell = 0, cap_c = 0;
  int *bv = NULL, *btag = NULL, *cells = NULL, *ctype = NULL;
  int* id2idx = NULL;
  int maxid = 0;
  s->ctag = 0;
  while (fscanf(f, "%255s", tok) == 1) {
    if (!strcmp(tok, "$NOD")) {
      if (fscanf(f, "%d", &s->nv) != 1) return -2;
      s->X = calloc((size_t)s->nv * 3, sizeof(double));
      s->vid = calloc((size_t)s->nv, sizeof(int));
      for (int i = 0; i < s->nv; ++i) {
        if (fscanf(f, "%d %lf %lf %lf", &s->vid[i], &s->X[3 * i], &s->X[3 * i + 1], &s->X[3 * i + 2]) != 4)
          return -2;
        if (s->vid[i] > maxid) maxid = s->vid[i];
      }
      id2idx = malloc((size_t)(maxid + 1) * sizeof(int));
      for (int i = 0; i <= maxid; ++i) id2idx[i] = -1;
      for (int i = 0; i < s->nv; ++i) id2idx[s->vid[i]] = i;
    } else if (!strcmp(tok, "$ELM")) {
      int n;
      if (fscanf(f, "%d", &n) != 1) return -2;
      for (int i = 0; i < n; ++i) {
        int num, typ, phys, elem, nn, v[8];
        if (fscanf(f, "%d %d %d %d %d", &num, &typ, &phys, &elem, &nn) != 5 || nn > 8) return -2;
        for (int k = 0; k < nn; ++k)
          if (fscanf(f, "%d", &v[k]) != 1) return -2;
        if (typ == 2 || typ == 4) {
          if (ncell == cap_c) {
            cap_c = cap_c ? 2 * cap_c : 1024;
            cells = realloc(cells, (size_t)cap_c * 4 * sizeof(int));
            ctype = realloc(ctype, (size_t)cap_c * sizeof(int));
          }
          for (int k = 0; k < 4; ++k) cells[ncell * 4 + k] = (k < nn) ? v[k] : -1;
          ctype[ncell] = typ;
          s->ctag = phys;
          ncell++;
        }
        if (typ == 1 || typ == 2) {
          if (nb == cap_b) {
            cap_b = cap_b ? 2 * cap_b : 1024;
            bv = realloc(bv, (size_t)cap_b * 3 * sizeof(int));
            btag = realloc(btag, (size_t)cap_b * sizeof(int));
          }
          for (int k = 0; k < 3; ++k) bv[nb * 3 + k] = (k < nn) ? v[k] : -1;
          btag[nb] = phys;
          nb++;
        }
      }
    }
  }
  fclose(f);
  int has_tet = 0;
  for (int i = 0; i < ncell; ++i) has_tet |= (ctype[i] == 4);
  s->dim = has_tet ? 3 : 2;
  s->nvc = s->dim + 1;
  s->nfv = s->dim;
  s->nlf = s->dim + 1;
  int want = has_tet ? 4 : 2;
  s->E = 0;
  s->cv = malloc((size_t)ncell * s->nvc * sizeof(int));
  for (int i = 0; i < ncell; ++i) {
    if (ctype[i] != want) continue;
    for (int k = 0; k < s->nvc; ++k) s->cv[s->E * s->nvc + k] = id2idx[cells[i * 4 + k]];
    s->E++;
  }
  /* boundary facets of the file: keep those of dimension dim-1 */
  facekey* bk = malloc((size_t)(nb + 1) * sizeof(facekey));
  int nbk = 0;
  for (int i = 0; i < nb; ++i) {
    int nvf = (bv[i * 3 + 2] < 0) ? 2 : 3;
    if (nvf != s->nfv) continue;
    facekey k = {{INT32_MAX, INT32_MAX, INT32_MAX}, btag[i], 0};
    for (int j = 0; j < nvf; ++j) k.v[j] = bv[i * 3 + j];
    sort_ints(k.v, nvf);
    bk[nbk++] = k;
  }
  qsort(bk, nbk, sizeof(facekey), cmp_facekey);

  /* faces from cell templates */
  size_t nk = (size_t)s->E * s->nlf;
  facekey* keys = malloc(nk * sizeof(facekey));
  for (int e = 0; e < s->E; ++e)
    for (int lf = 0; lf < s->nlf; ++lf) {
      facekey k = {{INT32_MAX, INT32_MAX, INT32_MAX}, e, lf};
      for (int j = 0; j < s->nfv; ++j) {
        int lv = (s->dim == 2) ? kTriFace[lf][j] : kTetFace[lf][j];
        k.v[j] = s->vid[s->cv[e * s->nvc + lv]];
      }
      sort_ints(k.v, s->nfv);
      keys[e * s->nlf + lf] = k;
    }
  qsort(keys, nk, sizeof(facekey), cmp_facekey);
  uint32_t* rk = malloc((size_t)s->nv * sizeof(uint32_t));
  for (int i = 0; i < s->nv; ++i) rk[i] = or_glibc_rand_first((unsigned)s->vid[i]);
  s->F = 0;
  s->fv = malloc(nk * s->nfv * sizeof(int));
  s->eL = malloc(nk * sizeof(int));
  s->eR = malloc(nk * sizeof(int));
  s->lfL = malloc(nk * sizeof(int));
  s->lfR = malloc(nk * sizeof(int));
  s->bid = malloc(nk * sizeof(int));
  for (size_t i = 0; i < nk;) {
    size_t j = i + 1;
    while (j < nk && cmp_facekey(&keys[i], &keys[j]) == 0) ++j;
    int f = s->F++;
    int a = keys[i].cell, la = keys[i].lf;
    if (j - i == 2) {
      int b = keys[i + 1].cell, lb = keys[i + 1].lf;
      if (cell_less(s, rk, b, a)) {
        int t = a; a = b; b = t;
        t = la; la = lb; lb = t;
      }
      s->eL[f] = a; s->lfL[f] = la; s->eR[f] = b; s->lfR[f] = lb;
      s->bid[f] = s->ctag;
    } else {
      s->eL[f] = a; s->lfL[f] = la; s->eR[f] = -1; s->lfR[f] = -1;
      facekey* hit = bsearch(&keys[i], bk, nbk, sizeof(facekey), cmp_facekey);
      s->bid[f] = hit ? hit->cell : s->ctag;
    }
    for (int k = 0; k < s->nfv; ++k) {
      int lv = (s->dim == 2) ? kTriFace[la][k] : kTetFace[la][k];
      s->fv[f * s->nfv + k] = s->cv[a * s->nvc + lv];
    }
    i = j;
  }
  free(rk);
  free(keys);
  free(bk);
  free(bv);
  free(btag);
  free(cells);
  free(ctype);
  free(id2idx);
  return 0;
}

/* ------------------------------------------------------------------------ */
/* geometry: affine map x = x0 + sum_r xi_r e_r with e_u = x1-x0, e_v = x2-x0  */
/* (triangle) and e_u = x3-x0, e_v = x2-x0, e_w = x1-x0 (tet, the node order  */
/* of MeshMapping::GeomShapeFunctionTet, Mapping.cc:40-71).                   */
static void cell_frame(const or_solver* s, int e, double* x0, double J[9]) {
  const int* c = s->cv + e * s->nvc;
  const double* p0 = s->X + 3 * c[0];
  int order3[3] = {3, 2, 1};
  for (int k = 0; k < 3; ++k) x0[k] = p0[k];
  for (int r = 0; r < 3; ++r)
    for (int k = 0; k < 3; ++k) J[r * 3 + k] = 0.0;
  for (int r = 0; r < s->dim; ++r) {
    int node = (s->dim == 2) ? r + 1 : order3[r];
    const double* p = s->X + 3 * c[node];
    for (int k = 0; k < 3; ++k) J[r * 3 + k] = p[k] - p0[k];
  }
  if (s->dim == 2) J[8] = 1.0;
}

static double inv3(const double* A, double* B) {
  double det = A[0] * (A[4] * A[8] - A[5] * A[7]) - A[1] * (A[3] * A[8] - A[5] * A[6]) +
               A[2] * (A[3] * A[7] - A[4] * A[6]);
  double id = 1.0 / det;
  B[0] = (A[4] * A[8] - A[5] * A[7]) * id;
  B[1] = (A[2] * A[7] - A[1] * A[8]) * id;
  B[2] = (A[1] * A[5] - A[2] * A[4]) * id;
  B[3] = (A[5] * A[6] - A[3] * A[8]) * id;
  B[4] = (A[0] * A[8] - A[2] * A[6]) * id;
  B[5] = (A[2] * A[3] - A[0] * A[5]) * id;
  B[6] = (A[3] * A[7] - A[4] * A[6]) * id;
  B[7] = (A[1] * A[6] - A[0] * A[7]) * id;
  B[8] = (A[0] * A[4] - A[1] * A[3]) * id;
  return det;
}

static double len3(const double* a, const double* b) {
  double d0 = b[0] - a[0], d1 = b[1] - a[1], d2 = b[2] - a[2];
  return sqrt(d0 * d0 + d1 * d1 + d2 * d2);
}

/* reference coordinates of physical point x in cell e (inverse affine map) */
static void to_ref(const or_solver* s, int e, const double* x, double* xi) {
  double x0[3], J[9];
  cell_frame(s, e, x0, J);
  const double* Ji = s->jinv + 9 * e;
  double d[3] = {x[0] - x0[0], x[1] - x0[1], x[2] - x0[2]};
  /* x - x0 = sum_r xi_r J[r][:]  ->  xi = (J^T)^{-1} d = Jinv^T d */
  for (int r = 0; r < 3; ++r) xi[r] = 0.0;
  for (int r = 0; r < s->dim; ++r) xi[r] = Ji[0 * 3 + r] * d[0] + Ji[1 * 3 + r] * d[1] + Ji[2 * 3 + r] * d[2];
  (void)J;
}

static void build_geometry(or_solver* s) {
  s->jac = malloc((size_t)s->E * 9 * sizeof(double));
  s->jinv = malloc((size_t)s->E * 9 * sizeof(double));
  s->det = malloc((size_t)s->E * sizeof(double));
  s->csize = malloc((size_t)s->E * sizeof(double));
  for (int e = 0; e < s->E; ++e) {
    double x0[3];
    cell_frame(s, e, x0, s->jac + 9 * e);
    double d = inv3(s->jac + 9 * e, s->jinv + 9 * e);
    s->det[e] = fabs(d);
    const int* c = s->cv + e * s->nvc;
    const double *p1 = s->X + 3 * c[0], *p2 = s->X + 3 * c[1], *p3 = s->X + 3 * c[2];
    if (s->dim == 2) { /* DGCell::computeCellSize, DGCell.cc:1211-1229 */
      double a = len3(p1, p2), b = len3(p2, p3), cc = len3(p3, p1);
      double halfP = 0.5 * (a + b + cc);
      s->csize[e] = sqrt(halfP * (halfP - a) * (halfP - b) * (halfP - cc)) / halfP * 2.;
    } else { /* minimum edge, DGCell.cc:1239-1256 */
      const double* p4 = s->X + 3 * c[3];
      double L[6] = {len3(p1, p2), len3(p2, p3), len3(p3, p1), len3(p1, p4), len3(p2, p4), len3(p3, p4)};
      double m = L[0];
      for (int k = 1; k < 6; ++k)
        if (m > L[k]) m = L[k];
      s->csize[e] = m;
    }
  }
  /* faces */
  s->fn = malloc((size_t)s->F * 3 * sizeof(double));
  s->fmeas = malloc((size_t)s->F * sizeof(double));
  s->fx = malloc((size_t)s->F * s->nqf * 3 * sizeof(double));
  s->fjw = malloc((size_t)s->F * s->nqf * sizeof(double));
  s->trL = malloc((size_t)s->F * s->nqf * s->Np * sizeof(double));
  s->trR = calloc((size_t)s->F * s->nqf * s->Np, sizeof(double));
  for (int f = 0; f < s->F; ++f) {
    const int* fv = s->fv + f * s->nfv;
    const double *a = s->X + 3 * fv[0], *b = s->X + 3 * fv[1];
    int eL = s->eL[f];
    /* vertex of the left cell off the face */
    int opp = -1;
    for (int k = 0; k < s->nvc; ++k) {
      int v = s->cv[eL * s->nvc + k], on = 0;
      for (int j = 0; j < s->nfv; ++j) on |= (fv[j] == v);
      if (!on) opp = v;
    }
    const double* po = s->X + 3 * opp;
    double n[3], meas, jf;
    if (s->dim == 2) {
      double t0 = b[0] - a[0], t1 = b[1] - a[1];
      meas = sqrt(t0 * t0 + t1 * t1);
      n[0] = t1 / meas; n[1] = -t0 / meas; n[2] = 0.0;
      jf = 0.5 * meas; /* edge map on [-1,1] */
    } else {
      const double* c = s->X + 3 * fv[2];
      double u[3] = {b[0] - a[0], b[1] - a[1], b[2] - a[2]}, v[3] = {c[0] - a[0], c[1] - a[1], c[2] - a[2]};
      double cr[3] = {u[1] * v[2] - u[2] * v[1], u[2] * v[0] - u[0] * v[2], u[0] * v[1] - u[1] * v[0]};
      double l = sqrt(cr[0] * cr[0] + cr[1] * cr[1] + cr[2] * cr[2]);
      n[0] = cr[0] / l; n[1] = cr[1] / l; n[2] = cr[2] / l;
      meas = 0.5 * l;
      jf = l; /* reference triangle map, weights carry the 1/2 */
    }
    double dop = (po[0] - a[0]) * n[0] + (po[1] - a[1]) * n[1] + (po[2] - a[2]) * n[2];
    if (dop > 0) { n[0] = -n[0]; n[1] = -n[1]; n[2] = -n[2]; }
    for (int k = 0; k < 3; ++k) s->fn[3 * f + k] = n[k];
    s->fmeas[f] = meas;
    for (int q = 0; q < s->nqf; ++q) {
      double x[3];
      if (s->dim == 2) {
        double sp = s->fqp[q][0];
        for (int k = 0; k < 3; ++k) x[k] = a[k] * (1 - sp) * 0.5 + b[k] * (1 + sp) * 0.5;
      } else {
        const double* c = s->X + 3 * fv[2];
        double u = s->fqp[q][0], v = s->fqp[q][1];
        for (int k = 0; k < 3; ++k) x[k] = a[k] * (1 - u - v) + b[k] * u + c[k] * v;
      }
      for (int k = 0; k < 3; ++k) s->fx[(f * s->nqf + q) * 3 + k] = x[k];
      s->fjw[f * s->nqf + q] = jf * s->fqw[q];
      double xi[3];
      to_ref(s, eL, x, xi);
      basis_eval(s, xi, s->trL + ((size_t)f * s->nqf + q) * s->Np);
      if (s->eR[f] >= 0) {
        to_ref(s, s->eR[f], x, xi);
        basis_eval(s, xi, s->trR + ((size_t)f * s->nqf + q) * s->Np);
      }
    }
  }
}

/* Periodic pairs (mMesh::setPeriodicBC, mMesh.cc:457-524): a boundary face
 * tagged 510 pairs with the first other 510 face whose two vertices have the
 * same y coordinates (1e-10, either order), 610 likewise with x; the partner
 * trace is the partner face's left cell evaluated at the mirrored point
 * (-x, y) for 510, (x, -y) for 610 (DGBoundaryCell::setPeriodicBC,
 * DGCell.cc:557-577).  Triangles only, as in the reference. */
static void build_periodic(or_solver* s) {
  s->pcell = malloc((size_t)s->F * sizeof(int));
  for (int f = 0; f < s->F; ++f) s->pcell[f] = -1;
  if (s->dim != 2) return;
  const double SN = 1.0e-10;
  for (int f = 0; f < s->F; ++f) {
    const int id = s->bid[f];
    if (s->eR[f] >= 0 || (id != 510 && id != 610)) continue;
    const int c = (id == 510) ? 1 : 0; /* coordinate that must match */
    const double* v1 = s->X + 3 * s->fv[f * 2];
    const double* v2 = s->X + 3 * s->fv[f * 2 + 1];
    for (int g = 0; g < s->F; ++g) {
      if (g == f || s->eR[g] >= 0 || s->bid[g] != id) continue;
      const double* a1 = s->X + 3 * s->fv[g * 2];
      const double* a2 = s->X + 3 * s->fv[g * 2 + 1];
      if ((fabs(v1[c] - a1[c]) < SN && fabs(v2[c] - a2[c]) < SN) ||
          (fabs(v1[c] - a2[c]) < SN && fabs(v2[c] - a1[c]) < SN)) {
        const int pe = s->eL[g];
        s->pcell[f] = pe;
        for (int q = 0; q < s->nqf; ++q) {
          const double* x = s->fx + (f * s->nqf + q) * 3;
          double xm[3] = {x[0], x[1], x[2]}, xi[3];
          if (id == 510) xm[0] = -x[0];
          else xm[1] = -x[1];
          to_ref(s, pe, xm, xi);
          basis_eval(s, xi, s->trR + ((size_t)f * s->nqf + q) * s->Np);
        }
        break;
      }
    }
  }
}

static int np_of(int dim, int p) {
  return dim == 2 ? (p + 1) * (p + 2) / 2 : (p + 1) * (p + 2) * (p + 3) / 6;
}

static const dgp_q_rule* simplex_rule(int dim, int degree) {
  if (degree < 1) degree = 1;
  if (dim == 2) {
    for (unsigned i = 0; i < sizeof(dgp_q_tri_rules) / sizeof(dgp_q_tri_rules[0]); ++i)
      if (dgp_q_tri_rules[i].degree == degree) return &dgp_q_tri_rules[i];
  } else {
    for (unsigned i = 0; i < sizeof(dgp_q_tet_rules) / sizeof(dgp_q_tet_rules[0]); ++i)
      if (dgp_q_tet_rules[i].degree == degree) return &dgp_q_tet_rules[i];
  }
  return NULL;
}

or_solver* or_create(const char* msh_path, int law, int flux, int order, int field,
                     const double* params) {
  return or_create_rule(msh_path, law, flux, order, field, params, 0);
}

/* rule 1: at P2 the workloads' quadrature point counts -- triangles the
 * 7-point volume rule of degree 5, tets the 11-point volume rule and the
 * 6-point face rule of degree 4; every other order as rule 0 (DG-Parallel's) */
or_solver* or_create_rule(const char* msh_path, int law, int flux, int order, int field,
                          const double* params, int rule) {
  or_solver* s = calloc(1, sizeof(or_solver));
  s->law = law;
  s->flux = flux;
  s->order = order;
  s->field = field;
  for (int i = 0; i < 16; ++i) s->prm[i] = params ? params[i] : 0.0;
  s->gamma = (s->prm[7] > 0) ? s->prm[7] : 1.4;
  switch (law) {
    case OR_SCALAR: case OR_BURGERS2D: s->m = 1; break;
    case OR_EULER2D: s->m = 4; break;
    case OR_EULER3D: s->m = 5; break;
    case OR_MAXWELL2D: s->m = 3; break;
    default: s->m = 6;
  }
  /* rules need the dimension: read the mesh first */
  if (read_msh(s, msh_path) != 0) {
    free(s);
    return NULL;
  }
  s->Np = np_of(s->dim, order);
  if (s->Np > MAXNP) { or_destroy(s); return NULL; }
  build_basis(s);
  s->phi0 = s->G[0][0];
  const int alt = rule == 1 && order == 2;
  const dgp_q_rule* vr = !alt ? simplex_rule(s->dim, 2 * order)
                              : s->dim == 2 ? simplex_rule(2, 5) : &dgp_q_tet_alt_rules[0];
  if (!vr) { or_destroy(s); return NULL; }
  s->nq = vr->npts;
  double refm = (s->dim == 2) ? 0.5 : 1.0 / 6.0;
  for (int q = 0; q < s->nq; ++q) {
    for (int k = 0; k < 3; ++k) s->qp[q][k] = (k < s->dim) ? vr->data[q * (s->dim + 1) + k] : 0.0;
    s->qw[q] = refm * vr->data[q * (s->dim + 1) + s->dim];
    basis_eval(s, s->qp[q], s->phi[q]);
    basis_grad(s, s->qp[q], s->dphi[q]);
  }
  if (s->dim == 2) {
    s->nqf = order + 1; /* getNGQ1DPts(2p+1) */
    const double* gl = dgp_q_gauss_legendre[s->nqf];
    for (int q = 0; q < s->nqf; ++q) {
      s->fqp[q][0] = gl[2 * q];
      s->fqp[q][1] = 0.0;
      s->fqw[q] = gl[2 * q + 1];
    }
  } else {
    const dgp_q_rule* fr = simplex_rule(2, alt ? 4 : 2 * order + 1);
    s->nqf = fr->npts;
    for (int q = 0; q < s->nqf; ++q) {
      s->fqp[q][0] = fr->data[q * 3];
      s->fqp[q][1] = fr->data[q * 3 + 1];
      s->fqw[q] = 0.5 * fr->data[q * 3 + 2];
    }
  }
  build_geometry(s);
  build_periodic(s);
  size_t n = (size_t)s->E * s->m * s->Np;
  s->C = calloc(n, sizeof(double));
  s->R = calloc(n, sizeof(double));
  s->soln = calloc(n, sizeof(double));
  s->L = calloc(n, sizeof(double));
  s->trig = calloc((size_t)s->E, 1);
  s->bad = calloc((size_t)s->E, 1);
  if (s->dim == 2) {
    build_limiter_tables(s);
    build_limiter_geometry(s);
  }
  or_project(s, 0.0);
  return s;
}

void or_destroy(or_solver* s) {
  if (!s) return;
  free(s->lts_bin); free(s->lts_role); free(s->lts_fcls);
  free(s->lts_c1); free(s->lts_save); free(s->lts_r);
  free(s->X); free(s->vid); free(s->cv); free(s->fv); free(s->eL); free(s->eR);
  free(s->lfL); free(s->lfR); free(s->bid); free(s->jac); free(s->jinv); free(s->det);
  free(s->csize); free(s->fn); free(s->fmeas); free(s->trL); free(s->trR); free(s->fx);
  free(s->fjw); free(s->C); free(s->R); free(s->soln);
  free(s->nb); free(s->bbc); free(s->L); free(s->trig); free(s->bad); free(s->pcell);
  free(s);
}

int or_num_cells(const or_solver* s) { return s->E; }
int or_num_faces(const or_solver* s) { return s->F; }
int or_num_fields(const or_solver* s) { return s->m; }
int or_num_modes(const or_solver* s) { return s->Np; }

int or_connectivity(const or_solver* s, int* out) {
  int w = 0;
  for (int f = 0; f < s->F; ++f) {
    int v[3];
    for (int k = 0; k < s->nfv; ++k) v[k] = s->vid[s->fv[f * s->nfv + k]];
    sort_ints(v, s->nfv);
    for (int k = 0; k < s->nfv; ++k) out[w++] = v[k];
    out[w++] = s->eL[f];
    out[w++] = s->eR[f];
    out[w++] = s->lfL[f];
    out[w++] = s->lfR[f];
    out[w++] = s->bid[f];
  }
  return w;
}

void or_face_normals(const or_solver* s, double* out) {
  for (int f = 0; f < s->F; ++f) {
    for (int k = 0; k < 3; ++k) out[4 * f + k] = s->fn[3 * f + k];
    out[4 * f + 3] = s->fmeas[f];
  }
}

void or_get_state(const or_solver* s, double* out) {
  memcpy(out, s->C, (size_t)s->E * s->m * s->Np * sizeof(double));
}

void or_set_state(or_solver* s, const double* in) {
  memcpy(s->C, in, (size_t)s->E * s->m * s->Np * sizeof(double));
}

static void phys_point(const or_solver* s, int e, const double* xi, double* x) {
  double x0[3], J[9];
  cell_frame(s, e, x0, J);
  for (int k = 0; k < 3; ++k) {
    x[k] = x0[k];
    for (int r = 0; r < s->dim; ++r) x[k] += xi[r] * J[r * 3 + k];
  }
}

/* DGCell::L2ProjInitial + L2Proj, DGCell.cc:1411-1483 (orthogonal basis) */
void or_project(or_solver* s, double t) {
  const int m = s->m, Np = s->Np;
  for (int e = 0; e < s->E; ++e) {
    double* c = s->C + (size_t)e * m * Np;
    double proj[MAXM * MAXNP];
    for (int i = 0; i < m * Np; ++i) proj[i] = 0.0;
    for (int q = 0; q < s->nq; ++q) {
      double x[3], val[MAXM];
      phys_point(s, e, s->qp[q], x);
      or_field_eval(s, x, t, val);
      double jw = s->det[e] * s->qw[q];
      for (int j = 0; j < m; ++j)
        for (int k = 0; k < Np; ++k) proj[k + Np * j] += val[j] * s->phi[q][k] * jw;
    }
    double inv = 1. / s->det[e];
    for (int i = 0; i < m * Np; ++i) c[i] = proj[i] * inv;
  }
}

static void interp(const double* fct, const double* a, int m, int Np, double* field) {
  for (int i = 0; i < m; ++i) {
    double tmp = 0.0;
    for (int j = 0; j < Np; ++j) tmp += fct[j] * a[i * Np + j];
    field[i] = tmp;
  }
}

/* DGCell::computeVolumeContribution (DGCell.cc:184-249) of cell e, added to R */
static void vol_add(const or_solver* s, const double* C, int e, double* R) {
  const int m = s->m, Np = s->Np, d = s->dim;
  const double* c = C + (size_t)e * m * Np;
  double* r = R + (size_t)e * m * Np;
  const double* Ji = s->jinv + 9 * e;
  for (int q = 0; q < s->nq; ++q) {
    double U[MAXM], F[MAXM][3], x[3];
    interp(s->phi[q], c, m, Np, U);
    phys_point(s, e, s->qp[q], x);
    law_flux(s, x, U, F);
    double jw = s->det[e] * s->qw[q];
    for (int j = 0; j < m; ++j)
      for (int k = 0; k < Np; ++k) {
        double g[3];
        for (int i = 0; i < 3; ++i) {
          g[i] = 0.0;
          for (int jj = 0; jj < 3; ++jj) g[i] += Ji[i * 3 + jj] * (jj < d ? s->dphi[q][jj][k] : 0.0);
          g[i] *= jw;
        }
        r[j * Np + k] += F[j][0] * g[0] + F[j][1] * g[1] + F[j][2] * g[2];
      }
  }
}

/* DGBoundaryCell::computeBoundaryContributions (DGCell.cc:639-732) of face f
 * at time t, added to R of both sides */
static void face_add(const or_solver* s, const double* C, int f, double t, double* R) {
  const int m = s->m, Np = s->Np;
  int eL = s->eL[f], eR = s->eR[f];
  const double* n = s->fn + 3 * f;
  for (int q = 0; q < s->nqf; ++q) {
    const double* x = s->fx + (f * s->nqf + q) * 3;
    const double* pl = s->trL + ((size_t)f * s->nqf + q) * Np;
    const double* pr = s->trR + ((size_t)f * s->nqf + q) * Np;
    double UL[MAXM], UR[MAXM], flux[MAXM];
    interp(pl, C + (size_t)eL * m * Np, m, Np, UL);
    if (eR >= 0) {
      interp(pr, C + (size_t)eR * m * Np, m, Np, UR);
      riemann_flux(s, n, x, UL, UR, flux);
    } else if (s->pcell[f] >= 0) { /* periodic: the partner's trace (DGCell.cc:687-705) */
      interp(pr, C + (size_t)s->pcell[f] * m * Np, m, Np, UR);
      riemann_flux(s, n, x, UL, UR, flux);
    } else {
      boundary_flux(s, s->bid[f], n, x, t, UL, flux);
    }
    double jw = s->fjw[f * s->nqf + q];
    double* rl = R + (size_t)eL * m * Np;
    for (int j = 0; j < m; ++j)
      for (int k = 0; k < Np; ++k) rl[j * Np + k] -= flux[j] * pl[k] * jw;
    if (eR >= 0) {
      double* rr = R + (size_t)eR * m * Np;
      for (int j = 0; j < m; ++j)
        for (int k = 0; k < Np; ++k) rr[j * Np + k] += flux[j] * pr[k] * jw;
    }
  }
}

/* assembly: the volume terms of all cells, then the face terms of all faces,
 * accumulating into R (which is zeroed first). */
static void assemble(or_solver* s, const double* C, double t, double* R) {
  memset(R, 0, (size_t)s->E * s->m * s->Np * sizeof(double));
  for (int e = 0; e < s->E; ++e) vol_add(s, C, e, R);
  for (int f = 0; f < s->F; ++f) face_add(s, C, f, t, R);
}

void or_rhs(or_solver* s, double t, double* out) { assemble(s, s->C, t, out); }

/* DGCell::adaptTimeStep / computeMAXEV (DGCell.cc:1155-1207) minimised over
 * cells as in DGAnalysis.cc:514-548 */
double or_cfl_dt(const or_solver* s, double cfl) {
  const int m = s->m, Np = s->Np;
  double DT = 500;
  for (int e = 0; e < s->E; ++e) {
    const double* c = s->C + (size_t)e * m * Np;
    double mean[MAXM];
    for (int j = 0; j < m; ++j) mean[j] = c[j * Np] * s->phi0;
    double a = max_eigen(s, mean);
    if (s->dim == 2) {
      static const double vx[3][3] = {{0, 0, 0}, {1, 0, 0}, {0, 1, 0}};
      for (int k = 0; k < 3; ++k) {
        double fct[MAXNP], val[MAXM];
        basis_eval(s, vx[k], fct);
        interp(fct, c, m, Np, val);
        double b = max_eigen(s, val);
        a = (b > a ? b : a);
      }
    }
    double deltat = s->csize[e] * cfl / (a * (2. * s->order + 1.0));
    if (DT > deltat) DT = deltat;
  }
  return DT;
}

/* ------------------------------------------------------------------------ */
/* Triangle moment limiter.  DGMomentLimiter::limit (DGLimiter.cc:963-1133)   */
/* indexes the tensor Legendre basis of quads ((p+1)^2-1 ...) and reads past  */
/* a triangle's coefficient row, so the triangle limiter is defined here and  */
/* restated independently by the CUDA path.  It keeps the reference's shape:  */
/*  - neighbours left/right/bottom/top by bounding boxes (DGLimiter.cc:977-993,*/
/*    faces visited in local-face order, later faces overwrite);              */
/*  - all differences use the unlimited state (the reference reads slot 0 and */
/*    writes the copy slot, then TimeIntegrator::limit copies back);          */
/*  - per field, degrees are visited from p down to 1; a degree whose modes   */
/*    are all below 1e-10 in magnitude is skipped; a degree with no component */
/*    limited ends the descent; minmod/absmin as DGLimiter.cc:1424-1447.      */
/* The moments of degree n are the n+1 physical derivatives                   */
/* d^n/dx^(n-a)dy^a of the cell's degree-n modal block (constant on the cell);*/
/* component a is bounded in x by the differences of the degree-(n-1)         */
/* derivative d^(n-1)/dx^(n-1-a)dy^a of the left/right neighbours and in y by */
/* d^(n-1)/dx^(n-a)dy^(a-1) of the bottom/top neighbours, times the reciprocal */
/* (rounded once) of the distance of the bounding-box centres (the degree-0   */
/* moment is the mean).                                                       */
/* A limited degree is mapped back to its modal block exactly; the mean is    */
/* never changed.  Trigger of a cell = lowest limited degree over its fields  */
/* (0: untouched).  Products and sums are evaluated one rounding at a time,   */
/* in the order written, so that the CUDA path reproduces them bit for bit.   */
/* ------------------------------------------------------------------------ */
#define LIM_SMALL 1.0e-10
#define LSIGN(a) ((a) < 0.0 ? -1 : 1)

static double lim_minmod3(double a, double b, double c, int* lim) {
  if (LSIGN(a) == LSIGN(b) && LSIGN(b) == LSIGN(c)) {
    double aa = fabs(a), ab = fabs(b), ac = fabs(c);
    if (aa < ab && aa < ac) { *lim = 0; return a; }
    if (ab < ac) { *lim = 1; return b; }
    *lim = 1;
    return c;
  }
  *lim = 1;
  return 0.0;
}

static double lim_minmod2(double a, double b, int* lim) {
  if (LSIGN(a) == LSIGN(b)) {
    if (fabs(a) < fabs(b)) { *lim = 0; return a; }
    *lim = 1;
    return b;
  }
  *lim = 1;
  return 0.0;
}

static int blk_off(int n) { return n * (n + 1) * (2 * n + 1) / 6; }

/* Dn[i][m] = d^n phi_(n,m) / du^(n-i) dv^i (constant): (n-i)! i! G[base+m][base+i];
 * Dinv = Dn^{-1} (upper triangular, back substitution in long double) */
static void build_limiter_tables(or_solver* s) {
  for (int n = 0; n <= s->order; ++n) {
    int base = n * (n + 1) / 2, w = n + 1, o = blk_off(n);
    long double A[5][5], X[5][5];
    for (int i = 0; i <= n; ++i)
      for (int m = 0; m <= n; ++m) {
        double f = (double)(fact(n - i) * fact(i));
        s->Dn[o + i * w + m] = f * s->G[base + m][base + i];
        A[i][m] = (long double)s->Dn[o + i * w + m];
      }
    for (int k = 0; k <= n; ++k) /* column k of the inverse */
      for (int i = n; i >= 0; --i) {
        long double r = (i == k) ? 1.0L : 0.0L;
        for (int m = i + 1; m <= n; ++m) r -= A[i][m] * X[m][k];
        X[i][k] = r / A[i][i];
      }
    for (int m = 0; m <= n; ++m)
      for (int i = 0; i <= n; ++i) s->Dinv[o + m * w + i] = (double)X[m][i];
  }
}

/* neighbours by bounding boxes (DGLimiter.cc:970-993; DGCell.cc:76-86) */
static void build_limiter_geometry(or_solver* s) {
  const int E = s->E;
  double* bmin = malloc((size_t)E * 2 * sizeof(double));
  double* bmax = malloc((size_t)E * 2 * sizeof(double));
  s->bbc = malloc((size_t)E * 2 * sizeof(double));
  s->nb = malloc((size_t)E * 4 * sizeof(int));
  for (int e = 0; e < E; ++e) {
    const int* c = s->cv + e * s->nvc;
    for (int k = 0; k < 2; ++k) bmin[2 * e + k] = bmax[2 * e + k] = s->X[3 * c[0] + k];
    for (int v = 1; v < s->nvc; ++v)
      for (int k = 0; k < 2; ++k) {
        double x = s->X[3 * c[v] + k];
        if (x < bmin[2 * e + k]) bmin[2 * e + k] = x;
        if (x > bmax[2 * e + k]) bmax[2 * e + k] = x;
      }
    for (int k = 0; k < 2; ++k) s->bbc[2 * e + k] = (bmin[2 * e + k] + bmax[2 * e + k]) / 2.;
  }
  int* cf = malloc((size_t)E * 3 * sizeof(int)); /* face of local face lf, -1: none */
  for (int i = 0; i < E * 3; ++i) cf[i] = -1;
  for (int f = 0; f < s->F; ++f) {
    cf[s->eL[f] * 3 + s->lfL[f]] = f;
    if (s->eR[f] >= 0) cf[s->eR[f] * 3 + s->lfR[f]] = f;
  }
  for (int e = 0; e < E; ++e) {
    int* nb = s->nb + 4 * e;
    nb[0] = nb[1] = nb[2] = nb[3] = -1;
    const double px = s->bbc[2 * e], py = s->bbc[2 * e + 1];
    for (int lf = 0; lf < 3; ++lf) {
      int f = cf[e * 3 + lf];
      if (f < 0 || s->eR[f] < 0) continue;
      int o = (s->eL[f] == e) ? s->eR[f] : s->eL[f];
      if (px > bmax[2 * o]) nb[0] = o;     /* left */
      if (px < bmin[2 * o]) nb[1] = o;     /* right */
      if (py > bmax[2 * o + 1]) nb[2] = o; /* bottom */
      if (py < bmin[2 * o + 1]) nb[3] = o; /* top */
    }
  }
  free(cf);
  free(bmin);
  free(bmax);
}

/* P[a][i]: coefficient of s^(n-i) t^i in (A s + B t)^(n-a) (C s + D t)^a */
static void lim_transform(int n, double A, double B, double C, double D, double* P) {
  for (int a = 0; a <= n; ++a) {
    double poly[6] = {1.0, 0, 0, 0, 0, 0}, q[6];
    int deg = 0;
    for (int k = 0; k < n; ++k) {
      double u = (k < n - a) ? A : C, v = (k < n - a) ? B : D;
      for (int i = 0; i <= deg + 1; ++i) {
        double x = (i <= deg) ? poly[i] * u : 0.0;
        double y = (i >= 1) ? poly[i - 1] * v : 0.0;
        q[i] = x + y;
      }
      ++deg;
      for (int i = 0; i <= deg; ++i) poly[i] = q[i];
    }
    for (int i = 0; i <= n; ++i) P[a * (n + 1) + i] = poly[i];
  }
}

/* physical degree-n derivatives of the degree-n block of one coefficient row */
static void lim_moments(const or_solver* s, const double* row, int n, const double* P, double* g) {
  const int base = n * (n + 1) / 2, w = n + 1;
  const double* D = s->Dn + blk_off(n);
  double r[5];
  for (int i = 0; i <= n; ++i) {
    double acc = 0.0;
    for (int m = 0; m <= n; ++m) acc = acc + D[i * w + m] * row[base + m];
    r[i] = acc;
  }
  for (int a = 0; a <= n; ++a) {
    double acc = 0.0;
    for (int i = 0; i <= n; ++i) acc = acc + P[a * w + i] * r[i];
    g[a] = acc;
  }
}

static void cell_lower_moments(const or_solver* s, const double* C, int e, int j, int n, double* h) {
  const double* Ji = s->jinv + 9 * e;
  double P[25];
  lim_transform(n, Ji[0], Ji[1], Ji[3], Ji[4], P);
  lim_moments(s, C + ((size_t)e * s->m + j) * s->Np, n, P, h);
}

static int limit_cell(const or_solver* s, const double* C, int e, double* out) {
  const int m = s->m, Np = s->Np, p = s->order;
  const int* nb = s->nb + 4 * e;
  const double px = s->bbc[2 * e], py = s->bbc[2 * e + 1];
  const double* Ji = s->jinv + 9 * e;
  const double* J = s->jac + 9 * e;
  int trig = 0;
  /* reciprocals of the signed centre distances: left/bottom own - theirs,
   * right/top theirs - own, each rounded once */
  double rc[4] = {0.0, 0.0, 0.0, 0.0};
  if (nb[0] >= 0) rc[0] = 1.0 / (px - s->bbc[2 * nb[0]]);
  if (nb[1] >= 0) rc[1] = 1.0 / (s->bbc[2 * nb[1]] - px);
  if (nb[2] >= 0) rc[2] = 1.0 / (py - s->bbc[2 * nb[2] + 1]);
  if (nb[3] >= 0) rc[3] = 1.0 / (s->bbc[2 * nb[3] + 1] - py);
  for (int j = 0; j < m; ++j) {
    const double* row = C + ((size_t)e * m + j) * Np;
    double* orow = out + (size_t)j * Np;
    for (int n = p; n >= 1; --n) {
      const int base = n * (n + 1) / 2, w = n + 1;
      int big = 0;
      for (int k = 0; k <= n; ++k) big |= fabs(row[base + k]) > LIM_SMALL;
      if (!big) continue;
      double P[25], g[5], gl[5], he[5], hx[4][5];
      lim_transform(n, Ji[0], Ji[1], Ji[3], Ji[4], P);
      lim_moments(s, row, n, P, g);
      cell_lower_moments(s, C, e, j, n - 1, he);
      for (int d = 0; d < 4; ++d)
        if (nb[d] >= 0) cell_lower_moments(s, C, nb[d], j, n - 1, hx[d]);
      int any = 0;
      for (int a = 0; a <= n; ++a) {
        gl[a] = g[a];
        int hasx = a <= n - 1 && (nb[0] >= 0 || nb[1] >= 0);
        int hasy = a >= 1 && (nb[2] >= 0 || nb[3] >= 0);
        double t1 = 0.0, t2 = 0.0;
        int l1 = 0, l2 = 0;
        if (hasx) {
          double fwd = 0.0, bwd = 0.0;
          if (nb[1] >= 0) fwd = (hx[1][a] - he[a]) * rc[1];
          if (nb[0] >= 0) bwd = (he[a] - hx[0][a]) * rc[0];
          if (nb[0] >= 0 && nb[1] >= 0) t1 = lim_minmod3(g[a], fwd, bwd, &l1);
          else if (nb[0] >= 0) t1 = lim_minmod2(g[a], bwd, &l1);
          else t1 = lim_minmod2(g[a], fwd, &l1);
        }
        if (hasy) {
          double fwd = 0.0, bwd = 0.0;
          if (nb[3] >= 0) fwd = (hx[3][a - 1] - he[a - 1]) * rc[3];
          if (nb[2] >= 0) bwd = (he[a - 1] - hx[2][a - 1]) * rc[2];
          if (nb[2] >= 0 && nb[3] >= 0) t2 = lim_minmod3(g[a], fwd, bwd, &l2);
          else if (nb[2] >= 0) t2 = lim_minmod2(g[a], bwd, &l2);
          else t2 = lim_minmod2(g[a], fwd, &l2);
        }
        if (hasx && hasy) {
          if (l1 || l2) { gl[a] = fabs(t1) < fabs(t2) ? t1 : t2; any = 1; }
        } else if (hasx) {
          if (l1) { gl[a] = t1; any = 1; }
        } else if (hasy) {
          if (l2) { gl[a] = t2; any = 1; }
        }
      }
      if (!any) break;
      /* back to reference derivatives (d/du = J00 d/dx + J01 d/dy, ...) and modes */
      double Q[25], r[5];
      lim_transform(n, J[0], J[1], J[3], J[4], Q);
      for (int i = 0; i <= n; ++i) {
        double acc = 0.0;
        for (int a = 0; a <= n; ++a) acc = acc + Q[i * w + a] * gl[a];
        r[i] = acc;
      }
      const double* Di = s->Dinv + blk_off(n);
      for (int k = 0; k <= n; ++k) {
        double acc = 0.0;
        for (int i = 0; i <= n; ++i) acc = acc + Di[k * w + i] * r[i];
        orow[base + k] = acc;
      }
      if (trig == 0 || n < trig) trig = n;
    }
  }
  return trig;
}

/* Barth limiter (DGBarthLimiter::limit, DGLimiter.cc:184-287) on every cell,
 * in place (the reference's TimeIntegrator::limit would copy the second
 * coefficient slot, which Barth never writes, back over it).  Per cell and
 * field: bounds = max/min of the interior-face neighbours' means (the cell's
 * own mean excluded; no interior neighbour: the cell is left alone, where the
 * reference reads uninitialised bounds); at every point of every face of the
 * cell, the cell's coefficients against the face's LEFT-cell basis values
 * (pg->fctleft, whichever side the cell is on), phi = (bound - mean) /
 * (val - mean) outside the bounds, 1 inside, clamped at 0; slope = min phi;
 * modes of degree >= 2 zeroed when slope < 0.9, degree-1 modes times slope.
 * The means never change, so the cell order does not matter.  trig: 1 where
 * a slope is below 1. */
static int barth_apply(or_solver* s, unsigned char* trig) {
  const int m = s->m, Np = s->Np, E = s->E, nqf = s->nqf;
  const int s1 = s->dim == 2 ? 3 : 4; /* modes of degree <= 1 */
  double* mx = (double*)malloc(sizeof(double) * (size_t)E * m);
  double* mn = (double*)malloc(sizeof(double) * (size_t)E * m);
  double* slope = (double*)malloc(sizeof(double) * (size_t)E * m);
  int* kk = (int*)calloc((size_t)E, sizeof(int));
  for (int f = 0; f < s->F; ++f) {
    if (s->eR[f] < 0) continue;
    for (int side = 0; side < 2; ++side) {
      const int c = side ? s->eR[f] : s->eL[f], o = side ? s->eL[f] : s->eR[f];
      for (int j = 0; j < m; ++j) {
        const double mo = s->C[((size_t)o * m + j) * Np] * s->phi0;
        double* X = mx + (size_t)c * m + j;
        double* N = mn + (size_t)c * m + j;
        if (kk[c] == 0) {
          *X = mo;
          *N = mo;
        } else {
          *X = mo > *X ? mo : *X;
          *N = mo < *N ? mo : *N;
        }
      }
      kk[c]++;
    }
  }
  for (size_t i = 0; i < (size_t)E * m; ++i) slope[i] = 1.0;
  for (int f = 0; f < s->F; ++f)
    for (int side = 0; side < 2; ++side) {
      const int c = side ? s->eR[f] : s->eL[f];
      if (c < 0 || kk[c] == 0) continue;
      const double* a = s->C + (size_t)c * m * Np;
      for (int q = 0; q < nqf; ++q) {
        double val[MAXM];
        interp(s->trL + ((size_t)f * nqf + q) * Np, a, m, Np, val);
        for (int j = 0; j < m; ++j) {
          const double mean = a[j * Np] * s->phi0;
          const double X = mx[(size_t)c * m + j], N = mn[(size_t)c * m + j];
          double phin = 1.0;
          if (val[j] > X) phin = (X - mean) / (val[j] - mean);
          else if (val[j] < N) phin = (N - mean) / (val[j] - mean);
          if (phin < 0.0) phin = 0.0;
          double* sl = slope + (size_t)c * m + j;
          *sl = *sl < phin ? *sl : phin;
        }
      }
    }
  int count = 0;
  for (int e = 0; e < E; ++e) {
    int t = 0;
    if (kk[e] > 0)
      for (int j = 0; j < m; ++j) {
        const double sl = slope[(size_t)e * m + j];
        if (!(sl < 1.0)) continue;
        double* a = s->C + ((size_t)e * m + j) * Np;
        t = 1;
        if (sl < 0.9)
          for (int k = s1; k < Np; ++k) a[k] = 0.0;
        for (int k = 1; k < s1 && k < Np; ++k) a[k] = a[k] * sl;
      }
    s->trig[e] = (unsigned char)t;
    count += t;
  }
  if (trig) memcpy(trig, s->trig, (size_t)E);
  free(mx);
  free(mn);
  free(slope);
  free(kk);
  return count;
}

/* on: 1 triangle moment limiter (triangles), 2 Barth limiter, 0 off */
void or_set_limiter(or_solver* s, int on) {
  if (on == 2) s->limiter = s->order > 0 ? 2 : 0;
  else s->limiter = (on && s->dim == 2 && s->order > 0) ? 1 : 0;
}

void or_set_p0_fallback(or_solver* s, int on) { s->p0 = on ? 1 : 0; }

int or_limit(or_solver* s, unsigned char* trig) {
  const size_t dof = (size_t)s->m * s->Np;
  int count = 0;
  if (s->limiter == 2) return barth_apply(s, trig);
  if (s->dim != 2 || s->order < 1) {
    if (trig) memset(trig, 0, (size_t)s->E);
    return 0;
  }
  memcpy(s->L, s->C, (size_t)s->E * dof * sizeof(double));
  for (int e = 0; e < s->E; ++e) {
    int t = limit_cell(s, s->C, e, s->L + e * dof);
    s->trig[e] = (unsigned char)t;
    count += t != 0;
  }
  memcpy(s->C, s->L, (size_t)s->E * dof * sizeof(double));
  if (trig) memcpy(trig, s->trig, (size_t)s->E);
  return count;
}

/* Euler2d::isPhysical / Euler3d::isPhysical (EulerLaw.cc:1398-1421) */
static int or_is_physical(const or_solver* s, const double* Q) {
  if (s->law == OR_EULER2D) {
    if (Q[0] < 0) return 0;
    if ((s->gamma - 1.) * (Q[3] - 0.5 * (Q[1] * Q[1] + Q[2] * Q[2]) / Q[0]) < 0.0) return 0;
  } else if (s->law == OR_EULER3D) {
    if (Q[0] < 0) return 0;
    if ((s->gamma - 1.) * (Q[3] - 0.5 * (Q[1] * Q[1] + Q[2] * Q[2] + Q[4] * Q[4]) / Q[0]) < 0.0) return 0;
  }
  return 1;
}

/* assembly of one stage with the P0 fallback: a cell with a non-physical
 * value at a volume quadrature point (the correction inside
 * DGCell::computeVolumeContribution, DGCell.cc:197-221, which runs before the
 * faces) or with a non-physical trace at a face point (the code of
 * computeBoundaryContributions, DGCell.cc:639-732, then DGCell::setToZero,
 * DGCell.cc:785-811, in the serial order of DGAnalysis.cc:392-417) drops its
 * modes k >= 1, and the RHS is assembled again.  The volume correction leaves
 * the zeroed cells with physical means, so the face check sees the same
 * cells either way: all marked cells are zeroed before the second assembly. */
static int assemble_stage(or_solver* s, double t, double* R) {
  assemble(s, s->C, t, R);
  if (!s->p0) return 0;
  const int m = s->m, Np = s->Np;
  int nbad = 0;
  memset(s->bad, 0, (size_t)s->E);
  for (int e = 0; e < s->E; ++e)
    for (int q = 0; q < s->nq; ++q) {
      double U[MAXM];
      interp(s->phi[q], s->C + (size_t)e * m * Np, m, Np, U);
      if (!or_is_physical(s, U)) s->bad[e] = 1;
    }
  for (int f = 0; f < s->F; ++f)
    for (int q = 0; q < s->nqf; ++q) {
      double U[MAXM];
      interp(s->trL + ((size_t)f * s->nqf + q) * Np, s->C + (size_t)s->eL[f] * m * Np, m, Np, U);
      if (!or_is_physical(s, U)) s->bad[s->eL[f]] = 1;
      if (s->eR[f] >= 0) {
        interp(s->trR + ((size_t)f * s->nqf + q) * Np, s->C + (size_t)s->eR[f] * m * Np, m, Np, U);
        if (!or_is_physical(s, U)) s->bad[s->eR[f]] = 1;
      }
    }
  for (int e = 0; e < s->E; ++e)
    if (s->bad[e]) {
      ++nbad;
      for (int j = 0; j < m; ++j)
        for (int k = 1; k < Np; ++k) s->C[((size_t)e * m + j) * Np + k] = 0.0;
    }
  if (nbad) assemble(s, s->C, t, R);
  return nbad;
}

void or_bad_cells(const or_solver* s, unsigned char* out) { memcpy(out, s->bad, (size_t)s->E); }

/* the right-hand side of one assembly with the P0 fallback (when on): the
 * marked cells' modes k >= 1 are zeroed in the state, as setToZero does;
 * returns the number of marked cells */
int or_rhs_p0(or_solver* s, double t, double* out) { return assemble_stage(s, t, out); }

void or_triggers(const or_solver* s, unsigned char* out) { memcpy(out, s->trig, (size_t)s->E); }

/* RungeKuttaTVD3::advanceInTime, TimeIntegrator.cc:838-990 (orthogonal basis) */
double or_step(or_solver* s, double t, double dt) {
  const int m = s->m, Np = s->Np, dof = m * Np;
  size_t n = (size_t)s->E * dof;
  assemble_stage(s, t, s->R); /* may drop cells to P0 before u_n is saved */
  memcpy(s->soln, s->C, n * sizeof(double));
  for (int e = 0; e < s->E; ++e) {
    double dj = dt / s->det[e];
    double* c = s->C + (size_t)e * dof;
    const double* r = s->R + (size_t)e * dof;
    for (int i = 0; i < dof; ++i) c[i] += r[i] * dj;
  }
  if (s->limiter) or_limit(s, NULL);
  assemble_stage(s, t + dt, s->R);
  for (int e = 0; e < s->E; ++e) {
    double dj = dt / s->det[e];
    double* c = s->C + (size_t)e * dof;
    const double* r = s->R + (size_t)e * dof;
    const double* so = s->soln + (size_t)e * dof;
    for (int i = 0; i < dof; ++i) c[i] = 0.25 * (c[i] + r[i] * dj + 3. * so[i]);
  }
  if (s->limiter) or_limit(s, NULL);
  assemble_stage(s, t + dt * 0.5, s->R);
  double resid = 0.0;
  for (int e = 0; e < s->E; ++e) {
    double dj = dt / s->det[e];
    double* c = s->C + (size_t)e * dof;
    const double* r = s->R + (size_t)e * dof;
    const double* so = s->soln + (size_t)e * dof;
    for (int i = 0; i < dof; ++i) {
      c[i] = (2.0 * (c[i] + r[i] * dj) + so[i]) / 3.0;
      double tmp = c[i] - so[i];
      resid += tmp * tmp;
    }
  }
  if (s->limiter) or_limit(s, NULL);
  return resid;
}

/* time loop of DGAnalysis::run (DGAnalysis.cc:480-731, CFL mode 0): with
 * tend > 0 the step is stretched to land on tend; with nsteps > 0 at most
 * nsteps steps are taken.  Returns the final time. */
double or_run(or_solver* s, double t0, double tend, double cfl, int nsteps, int* steps_done) {
  double t = t0;
  int k = 0;
  while ((nsteps <= 0 || k < nsteps) && (tend <= 0 || t < tend)) {
    if (nsteps <= 0 && tend <= 0) break;
    double dt = or_cfl_dt(s, cfl);
    if (tend > 0) {
      int N = (int)ceil((tend - t) / dt);
      dt = (tend - t) / N;
    }
    or_step(s, t, dt);
    t += dt;
    ++k;
  }
  if (steps_done) *steps_done = k;
  return t;
}

/* sqrt(sum_e sum_q (u_h - u_exact)^2 |J| w) with the rule of degree 2(p+1)
 * (DGCell::densityErrorL2, DGError.cc:805-826) */
/* The error family of DGError.cc (DGCell::L1exact :549, LinfError :567,
 * L1exactPressure :601, entropyErrorL1_2D/3D :621-665, pressureErrorL2 :774,
 * densityErrorL2 :805, entropyErrorL2_2D :687) in one place.  quantity >= 0:
 * field `quantity`; -1: pressure (gamma - 1)(E - |m|^2 / 2 rho) with E at
 * index 3 (and the 3D w-momentum at index 4); -2: entropy deviation
 * (p / p_ex) / (rho / rho_ex)^gamma - 1.  gamma = 1.4 as those functions fix it.
 * rule 0: the cell's volume rule of degree 2p (the L1 / Linf functions);
 * rule 1: the rule of degree 2(p+1) (the L2 functions).  out: L1 = sum |d| |J| w,
 * L2 = sqrt(sum d^2 |J| w), Linf = max |d| over the rule's points. */
static double err_quantity(const or_solver* s, int quantity, const double* v) {
  const double gamma = 1.4;
  if (quantity >= 0) return v[quantity];
  double m2 = v[1] * v[1] + v[2] * v[2];
  if (s->dim == 3) m2 += v[4] * v[4];
  const double p = (gamma - 1.) * (v[3] - 0.5 * m2 / v[0]);
  return p; /* the entropy deviation needs both states: see or_error_norms */
}

int or_error_norms(const or_solver* s, double t, int quantity, int rule, double* out) {
  const double gamma = 1.4;
  if (quantity >= s->m || quantity < -2) return -1;
  if (quantity < 0 && !(s->law == OR_EULER2D || s->law == OR_EULER3D)) return -1;
  const double refm = (s->dim == 2) ? 0.5 : 1.0 / 6.0;
  const dgp_q_rule* r = rule ? simplex_rule(s->dim, 2 * (s->order + 1)) : NULL;
  if (rule && !r) return -1;
  const int npts = rule ? r->npts : s->nq;
  double l1 = 0.0, l2 = 0.0, li = 0.0;
  for (int e = 0; e < s->E; ++e) {
    const double* c = s->C + (size_t)e * s->m * s->Np;
    for (int q = 0; q < npts; ++q) {
      double xi[3] = {0, 0, 0}, x[3], fct[MAXNP], val[MAXM], ex[MAXM], w;
      if (rule) {
        for (int k = 0; k < s->dim; ++k) xi[k] = r->data[q * (s->dim + 1) + k];
        w = refm * r->data[q * (s->dim + 1) + s->dim];
        basis_eval(s, xi, fct);
      } else {
        for (int k = 0; k < s->dim; ++k) xi[k] = s->qp[q][k];
        w = s->qw[q];
        for (int k = 0; k < s->Np; ++k) fct[k] = s->phi[q][k];
      }
      interp(fct, c, s->m, s->Np, val);
      phys_point(s, e, xi, x);
      or_field_eval(s, x, t, ex);
      double d;
      if (quantity == -2) {
        const double p = err_quantity(s, -1, val), pe = err_quantity(s, -1, ex);
        d = (p / pe) / pow(val[0] / ex[0], gamma) - 1.;
      } else {
        d = err_quantity(s, quantity, val) - err_quantity(s, quantity, ex);
      }
      const double jw = s->det[e] * w;
      l1 += fabs(d) * jw;
      l2 += d * d * jw;
      if (fabs(d) > li) li = fabs(d);
    }
  }
  out[0] = l1;
  out[1] = sqrt(l2);
  out[2] = li;
  return 0;
}

double or_l2_error(const or_solver* s, double t, int fi) {
  const dgp_q_rule* r = simplex_rule(s->dim, 2 * (s->order + 1));
  if (!r) return -1.0;
  double refm = (s->dim == 2) ? 0.5 : 1.0 / 6.0, acc = 0.0;
  for (int e = 0; e < s->E; ++e) {
    const double* c = s->C + (size_t)e * s->m * s->Np;
    for (int q = 0; q < r->npts; ++q) {
      double xi[3] = {0, 0, 0}, x[3], fct[MAXNP], val[MAXM], ex[MAXM];
      for (int k = 0; k < s->dim; ++k) xi[k] = r->data[q * (s->dim + 1) + k];
      double w = refm * r->data[q * (s->dim + 1) + s->dim];
      basis_eval(s, xi, fct);
      interp(fct, c, s->m, s->Np, val);
      phys_point(s, e, xi, x);
      or_field_eval(s, x, t, ex);
      double d = val[fi] - ex[fi];
      acc += d * d * s->det[e] * w;
    }
  }
  return sqrt(acc);
}

/* ------------------------------------------------------------------------ */
/* Local time stepping: RungeKuttaTVD2adaptive (TimeIntegrator.cc:442-836)   */
/* on the size bins of DGAnalysis::sortCellsBySize (DGAnalysis.cc:749-890).  */
/* The reference's range helpers TimeIntegrator::assembleVolume/             */
/* assembleBoundary(begin, end, t) (TimeIntegrator.cc:1438-1487) ship with   */
/* their bodies commented out, which leaves its local time stepping without  */
/* a right-hand side; here they do what the whole-mesh versions do           */
/* (TimeIntegrator.cc:1332-1412) on their range.  The right-hand side of a   */
/* cell accumulates across calls and is zeroed where the integrator calls   */
/* ZeroRHS, as in the reference.  Roles: 0 inner cell of bin b, 1 large cell */
/* on interface b (bin b), 2 small cell on interface b (bin b + 1).  Face   */
/* classes: b for the faces of bin b (both cells in bin b, or a boundary    */
/* face of a bin-b cell), nb + b for the faces between bins b and b + 1.    */
/* No limiter and no P0 fallback on this path.                              */
/* ------------------------------------------------------------------------ */
#define LTS_MAXBINS 10 /* the integrator's per-bin arrays (TimeIntegrator.h:47-50) */

int or_lts_setup(or_solver* s) {
  const int E = s->E, F = s->F;
  double maxS = 0.0, minS = 1.0; /* DGAnalysis.cc:756-766 (the minimum starts at 1) */
  for (int e = 0; e < E; ++e) {
    if (maxS < s->csize[e]) maxS = s->csize[e];
    if (minS > s->csize[e]) minS = s->csize[e];
  }
  int nb = (int)ceil(log(maxS / minS) / log(2.));
  if (nb < 2) return -1; /* no cell is binned: the reference stops ("cells were lost") */
  if (nb > LTS_MAXBINS) return -2;
  double B[LTS_MAXBINS + 1];
  B[0] = maxS;
  for (int i = 1; i <= nb; ++i) B[i] = B[i - 1] * 0.5;
  int* bin = (int*)malloc(sizeof(int) * (size_t)E);
  int* role = (int*)malloc(sizeof(int) * (size_t)E);
  int* fcls = (int*)malloc(sizeof(int) * (size_t)(F > 0 ? F : 1));
  int rc = 0;
  for (int e = 0; e < E && !rc; ++e) {
    bin[e] = -1;
    role[e] = 0;
    for (int i = 1; i <= nb; ++i)
      if (s->csize[e] <= B[i - 1] * 1.0001 && s->csize[e] > B[i] * 1.0001) bin[e] = i - 1;
    if (bin[e] < 0) rc = -3; /* below B_nb * 1.0001: lost */
  }
  for (int f = 0; f < F && !rc; ++f) {
    const int eL = s->eL[f], eR = s->eR[f];
    const int lb = bin[eL], rb = eR >= 0 ? bin[eR] : 0;
    if (eR < 0 || lb == rb) {
      fcls[f] = lb;
    } else if (lb - rb == 1 || rb - lb == 1) {
      const int lo = lb < rb ? lb : rb;
      const int large = lb < rb ? eL : eR, small = lb < rb ? eR : eL;
      fcls[f] = nb + lo;
      if (role[large] == 2 || role[small] == 1) rc = -4; /* on two interfaces: counted twice */
      role[large] = 1;
      role[small] = 2;
    } else {
      rc = -5; /* "Too big a difference between elements" */
    }
  }
  if (rc) {
    free(bin); free(role); free(fcls);
    return rc;
  }
  free(s->lts_bin); free(s->lts_role); free(s->lts_fcls);
  free(s->lts_c1); free(s->lts_save); free(s->lts_r);
  const size_t n = (size_t)E * s->m * s->Np;
  s->lts_bin = bin;
  s->lts_role = role;
  s->lts_fcls = fcls;
  s->lts_c1 = (double*)calloc(n, sizeof(double));
  s->lts_save = (double*)calloc(n, sizeof(double));
  s->lts_r = (double*)calloc(n, sizeof(double));
  s->lts_nb = nb;
  return nb;
}

void or_lts_bins(const or_solver* s, int* bin, int* role) {
  memcpy(bin, s->lts_bin, sizeof(int) * (size_t)s->E);
  memcpy(role, s->lts_role, sizeof(int) * (size_t)s->E);
}

/* group g of interface/bin index b: 0 inner cells of bin b, 1 large on
 * interface b, 2 small on interface b */
static int lts_in(const or_solver* s, int e, int g, int b) {
  const int r = s->lts_role[e], bb = s->lts_bin[e];
  return r == g && (g == 2 ? bb == b + 1 : bb == b);
}

static void lts_vol(or_solver* s, int g, int b) {
  for (int e = 0; e < s->E; ++e)
    if (lts_in(s, e, g, b)) vol_add(s, s->C, e, s->lts_r);
}

static void lts_bnd(or_solver* s, int cls, double t) {
  for (int f = 0; f < s->F; ++f)
    if (s->lts_fcls[f] == cls) face_add(s, s->C, f, t, s->lts_r);
}

/* the integrator's coefficient operations on one group (arithmetic in the
 * reference's order, one rounding per operation) */
enum { LU_EULER_IN, LU_TWO_HALF, LU_EULER, LU_SECOND, LU_SECOND_SWAP, LU_COPYBACK_ZERO, LU_LI_HALF,
       LU_RESTORE, LU_FINAL_RESET };

static void lts_update(or_solver* s, int g, int b, int op, double dt) {
  const int dof = s->m * s->Np;
  for (int e = 0; e < s->E; ++e) {
    if (!lts_in(s, e, g, b)) continue;
    const double det = s->det[e];
    double* c = s->C + (size_t)e * dof;
    double* c1 = s->lts_c1 + (size_t)e * dof;
    double* sv = s->lts_save + (size_t)e * dof;
    double* r = s->lts_r + (size_t)e * dof;
    for (int i = 0; i < dof; ++i) {
      switch (op) {
        case LU_EULER_IN: /* TimeIntegrator.cc:486-490 */
          sv[i] = c[i];
          c[i] += r[i] / det * dt;
          break;
        case LU_TWO_HALF: /* :508-518, :560-571 */
          sv[i] = c[i];
          c[i] += r[i] * dt / det;
          c1[i] = c[i];
          c[i] += r[i] * dt / det;
          break;
        case LU_EULER: /* :537-541 */
          sv[i] = c[i];
          c[i] += r[i] * dt / det;
          break;
        case LU_SECOND: /* :647-653, :697-704 */
        case LU_SECOND_SWAP: { /* :670-678, then DG_Dofs::swap */
          const double cn = (c[i] + r[i] * dt / det + sv[i]) * 0.5;
          if (op == LU_SECOND) {
            c[i] = cn;
          } else {
            c[i] = c1[i];
            c1[i] = cn;
          }
          break;
        }
        case LU_COPYBACK_ZERO: /* :615-621 */
          c[i] = c1[i];
          break;
        case LU_LI_HALF: { /* :735-738 */
          const double cn = sv[i] + (c[i] - sv[i]) + 0.25 * (c1[i] - 2. * c[i] + sv[i]);
          c[i] = cn;
          sv[i] = cn + 0.5 * (c1[i] - sv[i]);
          break;
        }
        case LU_RESTORE: /* :759-760 */
          c[i] = sv[i];
          break;
        case LU_FINAL_RESET: /* :777 */
          c[i] = c1[i];
          break;
      }
      if (op != LU_SECOND_SWAP && op != LU_LI_HALF && op != LU_RESTORE) r[i] = 0.0;
    }
  }
}

/* RungeKuttaTVD2adaptive::firstStage (TimeIntegrator.cc:442-591) */
static void lts_first(or_solver* s, int from, int to, double t, double DT) {
  const int nb = s->lts_nb;
  double dt = DT / pow(2., from);
  if (from) lts_vol(s, 2, from - 1);
  for (int b = from; b < to; ++b) {
    lts_vol(s, 0, b);
    lts_vol(s, 1, b);
    lts_vol(s, 2, b);
    lts_bnd(s, b, t + dt);
    lts_bnd(s, nb + b, t + dt);
    dt *= 0.5;
  }
  if (from) lts_bnd(s, nb + from - 1, t + dt);
  dt = DT / pow(2., from);
  for (int b = from; b < to; ++b) {
    lts_update(s, 0, b, LU_EULER_IN, dt);
    dt *= 0.5;
  }
  dt = DT / pow(2., from);
  for (int b = from; b < to - 1; ++b) {
    dt *= 0.5;
    lts_update(s, 1, b, LU_TWO_HALF, dt);
  }
  dt = DT / pow(2., from);
  if (from) lts_update(s, 2, from - 1, LU_EULER, dt);
  for (int b = from; b < to - 1; ++b) {
    dt *= 0.5;
    lts_update(s, 2, b, LU_TWO_HALF, dt);
  }
}

/* RungeKuttaTVD2adaptive::secondStage (TimeIntegrator.cc:594-715) */
static void lts_second(or_solver* s, int from, int to, double t, double DT) {
  const int nb = s->lts_nb;
  double dt = DT / pow(2., from);
  for (int b = from; b < to; ++b) {
    if (b > from) lts_update(s, 2, b - 1, LU_COPYBACK_ZERO, dt);
    lts_vol(s, 0, b);
    lts_vol(s, 1, b);
    if (b > 0) lts_vol(s, 2, b - 1);
    lts_bnd(s, b, t + dt);
    lts_bnd(s, nb + b, t + dt);
    if (b > 0) lts_bnd(s, nb + b - 1, t + dt);
    lts_update(s, 0, b, LU_SECOND, dt);
    lts_update(s, 1, b, LU_SECOND_SWAP, dt);
    if (b > 0) lts_update(s, 2, b - 1, LU_SECOND, dt);
    dt *= 0.5;
  }
}

/* RungeKuttaTVD2adaptive::advanceInTime (TimeIntegrator.cc:784-836): one
 * step of DT for bin 0, sub-cycled down to DT / 2^(nb-1) for the last bin.
 * Returns 0 as the reference does. */
double or_lts_step(or_solver* s, double t, double DT) {
  const int nb = s->lts_nb;
  int flat[LTS_MAXBINS];
  if (nb < 2) return -1.0;
  for (int i = 0; i < nb; ++i) flat[i] = 1;
  lts_first(s, 0, nb, t, DT);
  lts_second(s, 0, nb, t, DT);
  for (int i = 1; i < nb; ++i) flat[i] = 0;
  int i = nb - 1;
  while (i > 0) {
    for (i = nb - 1; i >= 1; i--)
      if (!flat[i]) {
        lts_update(s, 1, i - 1, LU_LI_HALF, 0.0);
        lts_first(s, i, nb, t, DT);
        lts_update(s, 1, i - 1, LU_RESTORE, 0.0);
        lts_second(s, i, nb, t, DT);
        lts_update(s, 1, i - 1, LU_FINAL_RESET, 0.0);
        flat[i] = 1;
        if (i != nb - 1)
          for (int j = i + 1; j < nb; ++j) flat[j] = 0;
        break;
      }
  }
  return 0.0;
}

/* time step of DGAnalysis::run mode 5 (DGAnalysis.cc:514-593): the CFL
 * minimum times 2^(bins - 1) */
double or_lts_dt(const or_solver* s, double cfl) { return or_cfl_dt(s, cfl) * pow(2., s->lts_nb - 1); }
