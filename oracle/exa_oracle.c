/*
 * CPU oracle -- TEST INFRASTRUCTURE ONLY (see exa_oracle.h).
 *
 * Plain-C FP64 restatement of ExaHyPE's generic ADER-DG and FV kernels.
 * Every function cites the reference file:line it follows.  Loop orders
 * follow the reference so that rounding stays close to it; the DG tables
 * come from the project's generated dg_tables.h (derived from the
 * mathematics and pinned against the reference's tables by
 * tests/test_dg_tables.py).
 */
#include "exa_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>
#include <float.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#include "../exahype_b200/csrc/dg_tables.h"

#define GAMMA 1.4
#define W(N, i) (exa_gl_weights[(N)][(i)])

/* ------------------------------------------------------------------ */
/* PDE: GenericEulerKernelTest3D.cpp:26-82, GenericEulerKernelTest2D.cpp:28-79 */
void orc_euler_flux(int dim, int planar, const double* Q, double* F) {
  const double irho = 1.0 / Q[0];
  const double j2 = planar ? (Q[1] * Q[1] + Q[2] * Q[2])
                           : (Q[1] * Q[1] + Q[2] * Q[2] + Q[3] * Q[3]);
  const double p = (GAMMA - 1) * (Q[4] - 0.5 * j2 * irho);
  for (int d = 0; d < dim; d++) {
    double* f = F + 5 * d;
    const double jn = Q[d + 1];
    f[0] = jn;
    f[1] = irho * jn * Q[1];
    f[2] = irho * jn * Q[2];
    f[3] = irho * jn * Q[3];
    f[d + 1] += p;
    f[4] = irho * jn * (Q[4] + p);
  }
}

void orc_euler_eigenvalues(int planar, const double* Q, int d, double* lambda) {
  const double irho = 1.0 / Q[0];
  const double j2 = planar ? (Q[1] * Q[1] + Q[2] * Q[2])
                           : (Q[1] * Q[1] + Q[2] * Q[2] + Q[3] * Q[3]);
  const double p = (GAMMA - 1) * (Q[4] - 0.5 * j2 * irho);
  const double un = Q[d + 1] * irho;
  const double c = sqrt(GAMMA * p * irho);
  lambda[0] = un - c;
  lambda[1] = un;
  lambda[2] = un;
  lambda[3] = un;
  lambda[4] = un + c;
}

/* ------------------------------------------------------------------ */
/* 3D space-time predictor:
 * kernels/aderdg/generic/c/3d/spaceTimePredictorNonlinear.cpph
 *   Picard loop :43-317, time averaging :325-397, extrapolation :399-519,
 *   driver :523-577.  Flux only (the Euler PDE has no source / NCP). */
static int stp3d(int N, int V, int P, int planar, double* lQhbnd, double* lFhbnd,
                 double* lQi, double* lQi_old, double* rhs, double* lFi,
                 double* lQhi, double* lFhi, const double* luh,
                 const double* dx, double dt) {
  const int B = N + 1, D = V + P, B2 = B * B, B3 = B2 * B, B4 = B3 * B;
#define LUH(z, y, x, m) luh[(((z) * B + (y)) * B + (x)) * D + (m)]
#define LQI(z, y, x, t, m) lQi[((((z) * B + (y)) * B + (x)) * B + (t)) * D + (m)]
#define LFI(t, z, y, x, d, m) lFi[(((((t) * B + (z)) * B + (y)) * B + (x)) * 4 + (d)) * V + (m)]
#define RHS(t, z, y, x, m) rhs[((((t) * B + (z)) * B + (y)) * B + (x)) * V + (m)]
  /* trivial initial guess :65-79 */
  for (int z = 0; z < B; z++)
    for (int y = 0; y < B; y++)
      for (int x = 0; x < B; x++)
        for (int t = 0; t < B; t++)
          for (int m = 0; m < D; m++) LQI(z, y, x, t, m) = LUH(z, y, x, m);

  const int maxit = 2 * (N + 1); /* :82 */
  int it;
  for (it = 0; it < maxit; it++) {
    memcpy(lQi_old, lQi, sizeof(double) * B4 * D);
    for (int t = 0; t < B; t++) {
      /* fluxes :93-115 */
      for (int z = 0; z < B; z++)
        for (int y = 0; y < B; y++)
          for (int x = 0; x < B; x++) {
            double F[15];
            orc_euler_flux(3, planar, &LQI(z, y, x, t, 0), F);
            for (int d = 0; d < 3; d++)
              for (int m = 0; m < V; m++) LFI(t, z, y, x, d, m) = F[5 * d + m];
            for (int m = 0; m < V; m++) LFI(t, z, y, x, 3, m) = 0.0;
          }
      /* rhs0 :117-133 */
      for (int z = 0; z < B; z++)
        for (int y = 0; y < B; y++)
          for (int x = 0; x < B; x++) {
            const double w = W(N, z) * W(N, y) * W(N, x);
            for (int m = 0; m < V; m++)
              RHS(t, z, y, x, m) = w * exa_f0[N][t] * LUH(z, y, x, m);
          }
      /* x derivative :141-169 */
      for (int z = 0; z < B; z++)
        for (int y = 0; y < B; y++) {
          const double us = W(N, t) * W(N, z) * W(N, y) * dt / dx[0];
          for (int l = 0; l < B; l++)
            for (int m = 0; m < V; m++)
              for (int n = 0; n < B; n++)
                RHS(t, z, y, l, m) -= us * LFI(t, z, y, n, 0, m) * exa_kxi[N][n][l];
        }
      /* y derivative :171-197 */
      for (int z = 0; z < B; z++)
        for (int x = 0; x < B; x++) {
          const double us = W(N, t) * W(N, z) * W(N, x) * dt / dx[1];
          for (int l = 0; l < B; l++)
            for (int m = 0; m < V; m++)
              for (int n = 0; n < B; n++)
                RHS(t, z, l, x, m) -= us * LFI(t, z, n, x, 1, m) * exa_kxi[N][n][l];
        }
      /* z derivative :199-225 */
      for (int y = 0; y < B; y++)
        for (int x = 0; x < B; x++) {
          const double us = W(N, t) * W(N, y) * W(N, x) * dt / dx[2];
          for (int l = 0; l < B; l++)
            for (int m = 0; m < V; m++)
              for (int n = 0; n < B; n++)
                RHS(t, l, y, x, m) -= us * LFI(t, n, y, x, 2, m) * exa_kxi[N][n][l];
        }
    }
    /* zero the variables (not the parameters) :255-268 */
    for (int s = 0; s < B4; s++)
      for (int m = 0; m < V; m++) lQi[s * D + m] = 0.0;
    /* discrete time integral with iK1 :270-296 */
    for (int z = 0; z < B; z++)
      for (int y = 0; y < B; y++)
        for (int x = 0; x < B; x++) {
          const double iw = 1.0 / (W(N, z) * W(N, y) * W(N, x));
          for (int l = 0; l < B; l++)
            for (int m = 0; m < V; m++)
              for (int n = 0; n < B; n++)
                LQI(z, y, x, l, m) += iw * RHS(n, z, y, x, m) * exa_ik1[N][l][n];
        }
    /* exit condition :298-306 */
    double sq = 0.0;
    for (int i = 0; i < B4 * D; i++) sq += (lQi_old[i] - lQi[i]) * (lQi_old[i] - lQi[i]);
    if (sq < 1e-7 * 1e-7) { it++; break; }
  }
  /* time averaging :325-397 */
  double* fx = lFhi;
  double* fy = lFhi + B3 * V;
  double* fz = lFhi + 2 * B3 * V;
  double* sh = lFhi + 3 * B3 * V;
  memset(lQhi, 0, sizeof(double) * B3 * D);
  memset(lFhi, 0, sizeof(double) * 4 * B3 * V);
  for (int z = 0; z < B; z++)
    for (int y = 0; y < B; y++)
      for (int x = 0; x < B; x++) {
        for (int m = 0; m < V; m++)
          for (int t = 0; t < B; t++) {
            fx[((z * B + y) * B + x) * V + m] += LFI(t, z, y, x, 0, m) * W(N, t);
            fy[((z * B + x) * B + y) * V + m] += LFI(t, z, y, x, 1, m) * W(N, t);
            fz[((y * B + x) * B + z) * V + m] += LFI(t, z, y, x, 2, m) * W(N, t);
          }
        for (int m = 0; m < D; m++)
          for (int t = 0; t < B; t++)
            lQhi[((z * B + y) * B + x) * D + m] += LQI(z, y, x, t, m) * W(N, t);
      }
  (void)sh;
  /* extrapolation :399-519 */
  memset(lQhbnd, 0, sizeof(double) * 6 * B2 * D);
  memset(lFhbnd, 0, sizeof(double) * 6 * B2 * V);
#define QB(f, i, j, m) lQhbnd[(((f) * B + (i)) * B + (j)) * D + (m)]
#define FB(f, i, j, m) lFhbnd[(((f) * B + (i)) * B + (j)) * V + (m)]
  for (int i = 0; i < B; i++)
    for (int j = 0; j < B; j++) {
      for (int k = 0; k < V; k++)
        for (int l = 0; l < B; l++) {
          FB(0, i, j, k) += fx[((i * B + j) * B + l) * V + k] * exa_flcoeff[N][l];
          FB(1, i, j, k) += fx[((i * B + j) * B + l) * V + k] * exa_frcoeff[N][l];
          FB(2, i, j, k) += fy[((i * B + j) * B + l) * V + k] * exa_flcoeff[N][l];
          FB(3, i, j, k) += fy[((i * B + j) * B + l) * V + k] * exa_frcoeff[N][l];
          FB(4, i, j, k) += fz[((i * B + j) * B + l) * V + k] * exa_flcoeff[N][l];
          FB(5, i, j, k) += fz[((i * B + j) * B + l) * V + k] * exa_frcoeff[N][l];
        }
      for (int k = 0; k < D; k++)
        for (int l = 0; l < B; l++) {
          QB(0, i, j, k) += lQhi[((i * B + j) * B + l) * D + k] * exa_flcoeff[N][l];
          QB(1, i, j, k) += lQhi[((i * B + j) * B + l) * D + k] * exa_frcoeff[N][l];
          QB(2, i, j, k) += lQhi[((i * B + l) * B + j) * D + k] * exa_flcoeff[N][l];
          QB(3, i, j, k) += lQhi[((i * B + l) * B + j) * D + k] * exa_frcoeff[N][l];
          QB(4, i, j, k) += lQhi[((l * B + i) * B + j) * D + k] * exa_flcoeff[N][l];
          QB(5, i, j, k) += lQhi[((l * B + i) * B + j) * D + k] * exa_frcoeff[N][l];
        }
    }
#undef QB
#undef FB
#undef LUH
#undef LQI
#undef LFI
#undef RHS
  return it;
}

/* 2D space-time predictor:
 * kernels/aderdg/generic/c/2d/spaceTimePredictorNonlinear.cpph
 *   Picard :43-266, averaging :274-330, extrapolation :332-409,
 *   driver :586-634. */
static int stp2d(int N, int V, int P, int planar, double* lQhbnd, double* lFhbnd,
                 double* lQi, double* lQi_old, double* rhs, double* lFi,
                 double* lQhi, double* lFhi, const double* luh,
                 const double* dx, double dt) {
  const int B = N + 1, D = V + P, B2 = B * B, B3 = B2 * B;
#define LUH(y, x, m) luh[((y) * B + (x)) * D + (m)]
#define LQI(y, x, t, m) lQi[(((y) * B + (x)) * B + (t)) * D + (m)]
#define LFI(t, y, x, d, m) lFi[((((t) * B + (y)) * B + (x)) * 3 + (d)) * V + (m)]
#define RHS(t, y, x, m) rhs[(((t) * B + (y)) * B + (x)) * V + (m)]
  for (int y = 0; y < B; y++)
    for (int x = 0; x < B; x++)
      for (int t = 0; t < B; t++)
        for (int m = 0; m < D; m++) LQI(y, x, t, m) = LUH(y, x, m);
  const int maxit = 2 * (N + 1);
  int it;
  for (it = 0; it < maxit; it++) {
    memcpy(lQi_old, lQi, sizeof(double) * B3 * D);
    for (int t = 0; t < B; t++) {
      for (int y = 0; y < B; y++)
        for (int x = 0; x < B; x++) {
          double F[10];
          orc_euler_flux(2, planar, &LQI(y, x, t, 0), F);
          for (int d = 0; d < 2; d++)
            for (int m = 0; m < V; m++) LFI(t, y, x, d, m) = F[5 * d + m];
          for (int m = 0; m < V; m++) LFI(t, y, x, 2, m) = 0.0;
        }
      for (int y = 0; y < B; y++)
        for (int x = 0; x < B; x++) {
          const double w = W(N, y) * W(N, x);
          for (int m = 0; m < V; m++) RHS(t, y, x, m) = w * exa_f0[N][t] * LUH(y, x, m);
        }
      for (int y = 0; y < B; y++) {
        const double us = W(N, t) * W(N, y) * dt / dx[0];
        for (int l = 0; l < B; l++)
          for (int m = 0; m < V; m++)
            for (int n = 0; n < B; n++)
              RHS(t, y, l, m) -= us * LFI(t, y, n, 0, m) * exa_kxi[N][n][l];
      }
      for (int x = 0; x < B; x++) {
        const double us = W(N, t) * W(N, x) * dt / dx[1];
        for (int l = 0; l < B; l++)
          for (int m = 0; m < V; m++)
            for (int n = 0; n < B; n++)
              RHS(t, l, x, m) -= us * LFI(t, n, x, 1, m) * exa_kxi[N][n][l];
      }
    }
    for (int s = 0; s < B3; s++)
      for (int m = 0; m < V; m++) lQi[s * D + m] = 0.0;
    for (int y = 0; y < B; y++)
      for (int x = 0; x < B; x++) {
        const double iw = 1.0 / (W(N, y) * W(N, x));
        for (int l = 0; l < B; l++)
          for (int m = 0; m < V; m++)
            for (int n = 0; n < B; n++)
              LQI(y, x, l, m) += iw * RHS(n, y, x, m) * exa_ik1[N][l][n];
      }
    double sq = 0.0;
    for (int i = 0; i < B3 * D; i++) sq += (lQi_old[i] - lQi[i]) * (lQi_old[i] - lQi[i]);
    if (sq < 1e-7 * 1e-7) { it++; break; }
  }
  double* fx = lFhi;
  double* fy = lFhi + B2 * V;
  memset(lQhi, 0, sizeof(double) * B2 * D);
  memset(lFhi, 0, sizeof(double) * 3 * B2 * V);
  for (int y = 0; y < B; y++)
    for (int x = 0; x < B; x++) {
      for (int m = 0; m < V; m++)
        for (int t = 0; t < B; t++) {
          fx[(y * B + x) * V + m] += LFI(t, y, x, 0, m) * W(N, t);
          fy[(x * B + y) * V + m] += LFI(t, y, x, 1, m) * W(N, t);
        }
      for (int m = 0; m < D; m++)
        for (int t = 0; t < B; t++) lQhi[(y * B + x) * D + m] += LQI(y, x, t, m) * W(N, t);
    }
  memset(lQhbnd, 0, sizeof(double) * 4 * B * D);
  memset(lFhbnd, 0, sizeof(double) * 4 * B * V);
  for (int j = 0; j < B; j++) {
    for (int k = 0; k < V; k++)
      for (int l = 0; l < B; l++) {
        lFhbnd[(0 * B + j) * V + k] += fx[(j * B + l) * V + k] * exa_flcoeff[N][l];
        lFhbnd[(1 * B + j) * V + k] += fx[(j * B + l) * V + k] * exa_frcoeff[N][l];
        lFhbnd[(2 * B + j) * V + k] += fy[(j * B + l) * V + k] * exa_flcoeff[N][l];
        lFhbnd[(3 * B + j) * V + k] += fy[(j * B + l) * V + k] * exa_frcoeff[N][l];
      }
    for (int k = 0; k < D; k++)
      for (int l = 0; l < B; l++) {
        lQhbnd[(0 * B + j) * D + k] += lQhi[(j * B + l) * D + k] * exa_flcoeff[N][l];
        lQhbnd[(1 * B + j) * D + k] += lQhi[(j * B + l) * D + k] * exa_frcoeff[N][l];
        lQhbnd[(2 * B + j) * D + k] += lQhi[(l * B + j) * D + k] * exa_flcoeff[N][l];
        lQhbnd[(3 * B + j) * D + k] += lQhi[(l * B + j) * D + k] * exa_frcoeff[N][l];
      }
  }
#undef LUH
#undef LQI
#undef LFI
#undef RHS
  return it;
}

int orc_stp_nonlinear(int dim, int order, int nvar, int npar, int planar,
                      double* lQhbnd, double* lFhbnd, double* lQi,
                      double* lQi_old, double* rhs, double* lFi, double* lQhi,
                      double* lFhi, const double* luh, const double* dx,
                      double dt) {
  if (dim == 3)
    return stp3d(order, nvar, npar, planar, lQhbnd, lFhbnd, lQi, lQi_old, rhs,
                 lFi, lQhi, lFhi, luh, dx, dt);
  return stp2d(order, nvar, npar, planar, lQhbnd, lFhbnd, lQi, lQi_old, rhs,
               lFi, lQhi, lFhi, luh, dx, dt);
}

/* ------------------------------------------------------------------ */
/* volume integral: c/3d/volumeIntegralNonlinear.cpph:26-125,
 *                  c/2d/volumeIntegralNonlinear.cpph:31-96 */
void orc_volume_integral(int dim, int order, int nvar, int use_source,
                         double* lduh, const double* lFhi, const double* dx) {
  const int N = order, B = N + 1, V = nvar;
  if (dim == 3) {
    const int B3 = B * B * B;
    const double* fx = lFhi;
    const double* fy = lFhi + B3 * V;
    const double* fz = lFhi + 2 * B3 * V;
    const double* sh = lFhi + 3 * B3 * V;
#define I4(a, b, c, m) ((((a) * B + (b)) * B + (c)) * V + (m))
    memset(lduh, 0, sizeof(double) * B3 * V);
    for (int i = 0; i < B; i++)
      for (int j = 0; j < B; j++) {
        const double us = W(N, i) * W(N, j) / dx[0];
        for (int k = 0; k < B; k++)
          for (int l = 0; l < V; l++)
            for (int m = 0; m < B; m++)
              lduh[I4(i, j, k, l)] += exa_kxi[N][k][m] * fx[I4(i, j, m, l)] * us;
      }
    for (int i = 0; i < B; i++)
      for (int j = 0; j < B; j++) {
        const double us = W(N, i) * W(N, j) / dx[1];
        for (int k = 0; k < B; k++)
          for (int l = 0; l < V; l++)
            for (int m = 0; m < B; m++)
              lduh[I4(i, k, j, l)] += exa_kxi[N][k][m] * fy[I4(i, j, m, l)] * us;
      }
    for (int i = 0; i < B; i++)
      for (int j = 0; j < B; j++) {
        const double us = W(N, i) * W(N, j) / dx[2];
        for (int k = 0; k < B; k++)
          for (int l = 0; l < V; l++)
            for (int m = 0; m < B; m++)
              lduh[I4(k, i, j, l)] += exa_kxi[N][k][m] * fz[I4(i, j, m, l)] * us;
      }
    if (use_source)
      for (int i = 0; i < B; i++)
        for (int j = 0; j < B; j++)
          for (int k = 0; k < B; k++) {
            const double w = W(N, i) * W(N, j) * W(N, k);
            for (int l = 0; l < V; l++) lduh[I4(i, j, k, l)] += w * sh[I4(i, j, k, l)];
          }
#undef I4
  } else {
    const int B2 = B * B;
    const double* fx = lFhi;
    const double* fy = lFhi + B2 * V;
    const double* sh = lFhi + 2 * B2 * V;
#define I3(a, b, m) (((a) * B + (b)) * V + (m))
    memset(lduh, 0, sizeof(double) * B2 * V);
    for (int j = 0; j < B; j++) {
      const double us = W(N, j) / dx[0];
      for (int k = 0; k < B; k++)
        for (int l = 0; l < V; l++)
          for (int m = 0; m < B; m++)
            lduh[I3(j, k, l)] += exa_kxi[N][k][m] * fx[I3(j, m, l)] * us;
    }
    for (int j = 0; j < B; j++) {
      const double us = W(N, j) / dx[1];
      for (int k = 0; k < B; k++)
        for (int l = 0; l < V; l++)
          for (int m = 0; m < B; m++)
            lduh[I3(k, j, l)] += exa_kxi[N][k][m] * fy[I3(j, m, l)] * us;
    }
    if (use_source)
      for (int j = 0; j < B; j++)
        for (int k = 0; k < B; k++) {
          const double w = W(N, j) * W(N, k);
          for (int l = 0; l < V; l++) lduh[I3(j, k, l)] += w * sh[I3(j, k, l)];
        }
#undef I3
  }
}

/* surface integral: c/3d/surfaceIntegralNonlinear.cpph:21-85,
 *                   c/2d/surfaceIntegralNonlinear.cpph:26-65 */
void orc_surface_integral(int dim, int order, int nvar, double* lduh,
                          const double* lF, const double* dx) {
  const int N = order, B = N + 1, V = nvar;
  if (dim == 3) {
#define I4(a, b, c, m) ((((a) * B + (b)) * B + (c)) * V + (m))
#define FB(f, a, b, m) ((((f) * B + (a)) * B + (b)) * V + (m))
    for (int i = 0; i < B; i++)
      for (int j = 0; j < B; j++) {
        const double us = W(N, i) * W(N, j) / dx[0];
        for (int k = 0; k < B; k++)
          for (int l = 0; l < V; l++)
            lduh[I4(i, j, k, l)] -= (lF[FB(1, i, j, l)] * exa_frcoeff[N][k] -
                                     lF[FB(0, i, j, l)] * exa_flcoeff[N][k]) * us;
      }
    for (int i = 0; i < B; i++)
      for (int j = 0; j < B; j++)
        for (int k = 0; k < B; k++) {
          const double us = W(N, i) * W(N, k) / dx[1];
          for (int l = 0; l < V; l++)
            lduh[I4(i, j, k, l)] -= (lF[FB(3, i, k, l)] * exa_frcoeff[N][j] -
                                     lF[FB(2, i, k, l)] * exa_flcoeff[N][j]) * us;
        }
    for (int i = 0; i < B; i++)
      for (int j = 0; j < B; j++)
        for (int k = 0; k < B; k++) {
          const double us = W(N, j) * W(N, k) / dx[2];
          for (int l = 0; l < V; l++)
            lduh[I4(i, j, k, l)] -= (lF[FB(5, j, k, l)] * exa_frcoeff[N][i] -
                                     lF[FB(4, j, k, l)] * exa_flcoeff[N][i]) * us;
        }
#undef I4
#undef FB
  } else {
#define I3(a, b, m) (((a) * B + (b)) * V + (m))
#define FB(f, a, m) ((((f) * B + (a))) * V + (m))
    for (int j = 0; j < B; j++) {
      const double us = W(N, j) / dx[0];
      for (int k = 0; k < B; k++)
        for (int l = 0; l < V; l++)
          lduh[I3(j, k, l)] -= (lF[FB(1, j, l)] * exa_frcoeff[N][k] -
                                lF[FB(0, j, l)] * exa_flcoeff[N][k]) * us;
    }
    for (int j = 0; j < B; j++)
      for (int k = 0; k < B; k++) {
        const double us = W(N, k) / dx[1];
        for (int l = 0; l < V; l++)
          lduh[I3(j, k, l)] -= (lF[FB(3, k, l)] * exa_frcoeff[N][j] -
                                lF[FB(2, k, l)] * exa_flcoeff[N][j]) * us;
      }
#undef I3
#undef FB
  }
}

/* Rusanov face flux: c/3d/riemannSolverNonlinear.cpph:37-120,
 *                    c/2d/riemannSolverNonlinear.cpph:37-114 */
void orc_riemann(int dim, int order, int nvar, int npar, int planar, double* FL,
                 double* FR, const double* QL, const double* QR, int direction) {
  const int N = order, B = N + 1, V = nvar, D = nvar + npar;
  const int nf = dim == 3 ? B * B : B;
  double QavL[16] = {0}, QavR[16] = {0};
  for (int i = 0; i < nf; i++) {
    const double w = dim == 3 ? W(N, i / B) * W(N, i % B) : W(N, i);
    for (int k = 0; k < D; k++) {
      QavL[k] += w * QL[i * D + k];
      QavR[k] += w * QR[i * D + k];
    }
  }
  double LL[5], LR[5];
  orc_euler_eigenvalues(planar, QavL, direction, LL);
  orc_euler_eigenvalues(planar, QavR, direction, LR);
  double sL = 0.0, sR = 0.0;
  for (int k = 0; k < 5; k++) {
    if (fabs(LL[k]) > sL) sL = fabs(LL[k]);
    if (fabs(LR[k]) > sR) sR = fabs(LR[k]);
  }
  const double smax = sL > sR ? sL : sR;
  for (int i = 0; i < nf; i++)
    for (int k = 0; k < V; k++) {
      const double f = 0.5 * (FR[i * V + k] + FL[i * V + k]) -
                       0.5 * smax * (QR[i * D + k] - QL[i * D + k]);
      FL[i * V + k] = f;
      FR[i * V + k] = f;
    }
}

/* c/3d/solutionUpdate.cpph:23-47, c/2d/solutionUpdate.cpph:23-45 */
void orc_solution_update(int dim, int order, int nvar, int npar, double* luh,
                         const double* lduh, double dt) {
  const int N = order, B = N + 1, V = nvar, D = nvar + npar;
  const int nn = dim == 3 ? B * B * B : B * B;
  for (int s = 0; s < nn; s++) {
    double w;
    if (dim == 3) w = W(N, s / (B * B)) * W(N, (s / B) % B) * W(N, s % B);
    else w = W(N, s / B) * W(N, s % B);
    const double us = dt / w;
    for (int l = 0; l < V; l++) luh[s * D + l] += lduh[s * V + l] * us;
  }
}

/* c/3d/stableTimeStepSize.cpph:21-61, c/2d/stableTimeStepSize.cpph:13-56 */
double orc_stable_dt(int dim, int order, int nvar, int npar, int planar,
                     const double* luh, const double* dx, double cfl) {
  const int B = order + 1, D = nvar + npar;
  const int nn = dim == 3 ? B * B * B : B * B;
  double dt = DBL_MAX;
  for (int s = 0; s < nn; s++) {
    double den = 0.0;
    for (int d = 0; d < dim; d++) {
      double lam[5];
      orc_euler_eigenvalues(planar, luh + s * D, d, lam);
      double mx = 0.0;
      for (int v = 0; v < nvar; v++) mx = fabs(lam[v]) > mx ? fabs(lam[v]) : mx;
      den += mx / dx[d];
    }
    const double c = cfl * exa_pnpm[order] / den;
    dt = c < dt ? c : dt;
  }
  return dt;
}

/* ------------------------------------------------------------------ */
/* Uniform periodic grid driver.  Step order of the reference's non-fused
 * time step (exahype/runners/Runner.cpp:1125-1160): dt (ADERDGSolver.cpp:
 * 1948-2000 + global min TimeStepSizeComputation.cpp:83-109), predictor +
 * volume integral (ADERDGSolver.cpp:1818-1946), Riemann on every face with
 * the left cell's face 2d+1 and the right cell's face 2d (ADERDGSolver.cpp:
 * 2744-2826), then surface integral + update (ADERDGSolver.cpp:2100-2170). */
static long ncells_of(int dim, const int* n) {
  return dim == 3 ? (long)n[0] * n[1] * n[2] : (long)n[0] * n[1];
}

/* dt of one cell: min over nodes of factor / sum_d(max|lambda_d|/dx_d) with
 * factor = CFL*PNPM[N] (policy 0, the reference rule) or CFL/(2N+1)
 * (policy 1). */
static double cell_dt(int dim, int order, int planar, const double* luh,
                      const double* dx, int policy, double cfl) {
  const int B = order + 1;
  const int nn = dim == 3 ? B * B * B : B * B;
  const double factor = policy == 0 ? cfl * exa_pnpm[order] : cfl / (2 * order + 1);
  double dt = DBL_MAX;
  for (int s = 0; s < nn; s++) {
    double den = 0.0;
    for (int d = 0; d < dim; d++) {
      double lam[5];
      orc_euler_eigenvalues(planar, luh + s * 5, d, lam);
      double mx = 0.0;
      for (int v = 0; v < 5; v++) mx = fabs(lam[v]) > mx ? fabs(lam[v]) : mx;
      den += mx / dx[d];
    }
    const double c = factor / den;
    dt = c < dt ? c : dt;
  }
  return dt;
}

double orc_aderdg_grid_dt(int dim, int order, int planar, const int* n,
                          const double* dx, const double* luh, int dt_policy,
                          double cfl) {
  const int B = order + 1;
  const int nn = dim == 3 ? B * B * B : B * B;
  const long nc = ncells_of(dim, n);
  double dt = DBL_MAX;
  for (long c = 0; c < nc; c++) {
    const double d = cell_dt(dim, order, planar, luh + c * nn * 5, dx, dt_policy, cfl);
    dt = d < dt ? d : dt;
  }
  return dt;
}

/* Outside state of a domain-boundary face node (the built-in stand-ins for
 * the reference's boundaryValues hook, boundaryConditions.cpph:24-85):
 * bc 1 = outflow (copy in -> out), bc 2 = reflecting wall (normal momentum
 * negated, normal flux of the reflected state). */
static void orc_boundary_values(int dim, int planar, int bc, int d, const double* qin,
                                const double* fin, double* qout, double* fout) {
  int m;
  if (bc == 1) {
    for (m = 0; m < 5; m++) {
      qout[m] = qin[m];
      fout[m] = fin[m];
    }
    return;
  }
  {
    double F[3 * 5];
    for (m = 0; m < 5; m++) qout[m] = qin[m];
    qout[d + 1] = -qout[d + 1];
    orc_euler_flux(dim, planar, qout, F);
    for (m = 0; m < 5; m++) fout[m] = F[d * 5 + m];
  }
}

double orc_aderdg_grid_step(int dim, int order, int planar, const int* n,
                            const double* dx, double* luh, int dt_policy,
                            double cfl, double dt_fixed, int* iters,
                            int nthreads) {
  return orc_aderdg_grid_step_bc(dim, order, planar, n, dx, luh, dt_policy, cfl, dt_fixed, iters,
                                 nthreads, NULL);
}

double orc_aderdg_grid_step_bc(int dim, int order, int planar, const int* n,
                               const double* dx, double* luh, int dt_policy,
                               double cfl, double dt_fixed, int* iters,
                               int nthreads, const int* bc) {
  const int B = order + 1, V = 5;
  const int nn = dim == 3 ? B * B * B : B * B;
  const int nst = nn * B;
  const int nfn = dim == 3 ? B * B : B;
  const long nc = ncells_of(dim, n);
  double dt;
  if (dt_policy == 2) dt = dt_fixed;
  else dt = orc_aderdg_grid_dt(dim, order, planar, n, dx, luh, dt_policy, cfl);
  double* lduh = (double*)malloc(sizeof(double) * nc * nn * V);
  double* qb = (double*)malloc(sizeof(double) * nc * 2 * dim * nfn * V);
  double* fb = (double*)malloc(sizeof(double) * nc * 2 * dim * nfn * V);
#ifdef _OPENMP
  if (nthreads > 0) omp_set_num_threads(nthreads);
#else
  (void)nthreads;
#endif
#pragma omp parallel
  {
    double* lQi = (double*)malloc(sizeof(double) * nst * V);
    double* lQo = (double*)malloc(sizeof(double) * nst * V);
    double* rhs = (double*)malloc(sizeof(double) * nst * V);
    double* lFi = (double*)malloc(sizeof(double) * nst * (dim + 1) * V);
    double* lQhi = (double*)malloc(sizeof(double) * nn * V);
    double* lFhi = (double*)malloc(sizeof(double) * nn * (dim + 1) * V);
#pragma omp for schedule(dynamic, 16)
    for (long c = 0; c < nc; c++) {
      int it = orc_stp_nonlinear(dim, order, V, 0, planar, qb + c * 2 * dim * nfn * V,
                                 fb + c * 2 * dim * nfn * V, lQi, lQo, rhs, lFi, lQhi,
                                 lFhi, luh + c * nn * V, dx, dt);
      if (iters) iters[c] = it;
      orc_volume_integral(dim, order, V, 0, lduh + c * nn * V, lFhi, dx);
    }
    free(lQi); free(lQo); free(rhs); free(lFi); free(lQhi); free(lFhi);
  }
  /* faces: for each cell and direction, the face towards the +d neighbour;
   * with a boundary rule in direction d, the faces on the domain ends are
   * solved against the outside state instead (applyBoundaryConditions,
   * ADERDGSolver.cpp:2854-2925: outside = left state on faces 2d, right
   * state on faces 2d+1) */
  const int fs = nfn * V;
  for (int d = 0; d < dim; d++) {
    const int bcd = bc ? bc[d] : 0;
#pragma omp parallel for schedule(static)
    for (long c = 0; c < nc; c++) {
      int cx = (int)(c % n[0]), cy = (int)((c / n[0]) % n[1]);
      int cz = dim == 3 ? (int)(c / ((long)n[0] * n[1])) : 0;
      int r[3] = {cx, cy, cz};
      if (bcd) {
        const int j0 = r[d];
        if (j0 == 0) {
          double* FR = fb + (c * 2 * dim + 2 * d) * fs;
          const double* QR = qb + (c * 2 * dim + 2 * d) * fs;
          double qo[125 * 5], fo[125 * 5];
          for (int j = 0; j < nfn; j++) orc_boundary_values(dim, planar, bcd, d, QR + j * V, FR + j * V, qo + j * V, fo + j * V);
          orc_riemann(dim, order, V, 0, planar, fo, FR, qo, QR, d);
        }
        if (j0 + 1 == n[d]) {
          double* FL = fb + (c * 2 * dim + 2 * d + 1) * fs;
          const double* QL = qb + (c * 2 * dim + 2 * d + 1) * fs;
          double qo[125 * 5], fo[125 * 5];
          for (int j = 0; j < nfn; j++) orc_boundary_values(dim, planar, bcd, d, QL + j * V, FL + j * V, qo + j * V, fo + j * V);
          orc_riemann(dim, order, V, 0, planar, FL, fo, QL, qo, d);
          continue;
        }
      }
      r[d] = (r[d] + 1) % n[d];
      long cr = dim == 3 ? ((long)r[2] * n[1] + r[1]) * n[0] + r[0]
                         : (long)r[1] * n[0] + r[0];
      orc_riemann(dim, order, V, 0, planar,
                  fb + (c * 2 * dim + 2 * d + 1) * fs, fb + (cr * 2 * dim + 2 * d) * fs,
                  qb + (c * 2 * dim + 2 * d + 1) * fs, qb + (cr * 2 * dim + 2 * d) * fs, d);
    }
  }
#pragma omp parallel for schedule(static)
  for (long c = 0; c < nc; c++) {
    orc_surface_integral(dim, order, V, lduh + c * nn * V, fb + c * 2 * dim * fs, dx);
    orc_solution_update(dim, order, V, 0, luh + c * nn * V, lduh + c * nn * V, dt);
  }
  free(lduh); free(qb); free(fb);
  return dt;
}

/* Slab decomposition (test oracle of the multi-GPU slab driver): the same
 * per-cell and per-face calls as orc_aderdg_grid_step, with the faces across
 * the ends of the last dimension solved against received face data. */
void orc_aderdg_slab_predict(int dim, int order, int planar, const int* n,
                             const double* dx, const double* luh, double dt,
                             double* lduh, double* qb, double* fb,
                             double* send_lo, double* send_hi) {
  const int B = order + 1, V = 5;
  const int nn = dim == 3 ? B * B * B : B * B;
  const int nst = nn * B;
  const int nfn = dim == 3 ? B * B : B;
  const int fs = nfn * V;
  const long nc = ncells_of(dim, n);
  const long layer = nc / n[dim - 1];
  double* lQi = (double*)malloc(sizeof(double) * nst * V);
  double* lQo = (double*)malloc(sizeof(double) * nst * V);
  double* rhs = (double*)malloc(sizeof(double) * nst * V);
  double* lFi = (double*)malloc(sizeof(double) * nst * (dim + 1) * V);
  double* lQhi = (double*)malloc(sizeof(double) * nn * V);
  double* lFhi = (double*)malloc(sizeof(double) * nn * (dim + 1) * V);
  for (long c = 0; c < nc; c++) {
    orc_stp_nonlinear(dim, order, V, 0, planar, qb + c * 2 * dim * fs, fb + c * 2 * dim * fs,
                      lQi, lQo, rhs, lFi, lQhi, lFhi, luh + c * nn * V, dx, dt);
    orc_volume_integral(dim, order, V, 0, lduh + c * nn * V, lFhi, dx);
  }
  free(lQi); free(lQo); free(rhs); free(lFi); free(lQhi); free(lFhi);
  const int d = dim - 1;
  for (long lc = 0; lc < layer; lc++) {
    const long lo = lc, hi = nc - layer + lc;
    memcpy(send_lo + lc * 2 * fs, qb + (lo * 2 * dim + 2 * d) * fs, sizeof(double) * fs);
    memcpy(send_lo + lc * 2 * fs + fs, fb + (lo * 2 * dim + 2 * d) * fs, sizeof(double) * fs);
    memcpy(send_hi + lc * 2 * fs, qb + (hi * 2 * dim + 2 * d + 1) * fs, sizeof(double) * fs);
    memcpy(send_hi + lc * 2 * fs + fs, fb + (hi * 2 * dim + 2 * d + 1) * fs, sizeof(double) * fs);
  }
}

void orc_aderdg_slab_correct(int dim, int order, int planar, const int* n,
                             const double* dx, double* luh, double* lduh,
                             double* qb, double* fb, const double* recv_lo,
                             const double* recv_hi, double dt) {
  const int B = order + 1, V = 5;
  const int nn = dim == 3 ? B * B * B : B * B;
  const int nfn = dim == 3 ? B * B : B;
  const int fs = nfn * V;
  const long nc = ncells_of(dim, n);
  const long layer = nc / n[dim - 1];
  double* tmp = (double*)malloc(sizeof(double) * fs);
  for (int d = 0; d < dim; d++) {
    for (long c = 0; c < nc; c++) {
      int r[3] = {(int)(c % n[0]), (int)((c / n[0]) % n[1]),
                  dim == 3 ? (int)(c / ((long)n[0] * n[1])) : 0};
      double* FLo = fb + (c * 2 * dim + 2 * d + 1) * fs;
      const double* QLo = qb + (c * 2 * dim + 2 * d + 1) * fs;
      if (d == dim - 1 && r[d] + 1 == n[d]) {
        /* upper slab end: the slab above's lowest-layer face */
        const double* h = recv_hi + (c - (nc - layer)) * 2 * fs;
        memcpy(tmp, h + fs, sizeof(double) * fs);
        orc_riemann(dim, order, V, 0, planar, FLo, tmp, QLo, h, d);
      } else {
        r[d] = (r[d] + 1) % n[d];
        long cr = dim == 3 ? ((long)r[2] * n[1] + r[1]) * n[0] + r[0] : (long)r[1] * n[0] + r[0];
        orc_riemann(dim, order, V, 0, planar, FLo, fb + (cr * 2 * dim + 2 * d) * fs, QLo,
                    qb + (cr * 2 * dim + 2 * d) * fs, d);
      }
    }
  }
  /* lower slab end: the slab below's highest-layer face against our own */
  {
    const int d = dim - 1;
    for (long lc = 0; lc < layer; lc++) {
      const double* h = recv_lo + lc * 2 * fs;
      memcpy(tmp, h + fs, sizeof(double) * fs);
      orc_riemann(dim, order, V, 0, planar, tmp, fb + (lc * 2 * dim + 2 * d) * fs, h,
                  qb + (lc * 2 * dim + 2 * d) * fs, d);
    }
  }
  free(tmp);
  for (long c = 0; c < nc; c++) {
    orc_surface_integral(dim, order, V, lduh + c * nn * V, fb + c * 2 * dim * fs, dx);
    orc_solution_update(dim, order, V, 0, luh + c * nn * V, lduh + c * nn * V, dt);
  }
}

/* One step's per-cell work on `ncells` independent cells (CPU-baseline
 * sample): predictor + volume integral, one Riemann solve per direction
 * (the cell's +d face against its own -d face, i.e. a one-cell periodic
 * domain), surface integral and update.  Same operation count per cell as
 * orc_aderdg_grid_step. */
void orc_aderdg_sample_step(int dim, int order, int planar, long ncells,
                            const double* dx, double* luh, double dt,
                            int nthreads) {
  const int B = order + 1, V = 5;
  const int nn = dim == 3 ? B * B * B : B * B;
  const int nst = nn * B, nfn = dim == 3 ? B * B : B, fs = nfn * V;
#ifdef _OPENMP
  if (nthreads > 0) omp_set_num_threads(nthreads);
#else
  (void)nthreads;
#endif
#pragma omp parallel
  {
    double* lQi = (double*)malloc(sizeof(double) * nst * V);
    double* lQo = (double*)malloc(sizeof(double) * nst * V);
    double* rhs = (double*)malloc(sizeof(double) * nst * V);
    double* lFi = (double*)malloc(sizeof(double) * nst * (dim + 1) * V);
    double* lQhi = (double*)malloc(sizeof(double) * nn * V);
    double* lFhi = (double*)malloc(sizeof(double) * nn * (dim + 1) * V);
    double* lduh = (double*)malloc(sizeof(double) * nn * V);
    double* qb = (double*)malloc(sizeof(double) * 2 * dim * fs);
    double* fb = (double*)malloc(sizeof(double) * 2 * dim * fs);
#pragma omp for schedule(dynamic, 16)
    for (long c = 0; c < ncells; c++) {
      double* u = luh + c * nn * V;
      orc_stp_nonlinear(dim, order, V, 0, planar, qb, fb, lQi, lQo, rhs, lFi, lQhi, lFhi, u, dx, dt);
      orc_volume_integral(dim, order, V, 0, lduh, lFhi, dx);
      for (int d = 0; d < dim; d++)
        orc_riemann(dim, order, V, 0, planar, fb + (2 * d + 1) * fs, fb + (2 * d) * fs,
                    qb + (2 * d + 1) * fs, qb + (2 * d) * fs, d);
      orc_surface_integral(dim, order, V, lduh, fb, dx);
      orc_solution_update(dim, order, V, 0, u, lduh, dt);
    }
    free(lQi); free(lQo); free(rhs); free(lFi); free(lQhi); free(lFhi);
    free(lduh); free(qb); free(fb);
  }
}

/* Grid of npx x npy periodic patches (back to back, x fastest), one step:
 * face ghost layers from the neighbouring patches' boundary layers
 * (ghostLayerFilling, kernels/finitevolumes/commons/c/commons.cpph:337-405),
 * dt = min over patches of the CFL rule, then every patch's solutionUpdate
 * with luh_new = luh beforehand (FiniteVolumesSolver.cpp:529-531).
 * dx = the patch extent.  Returns the dt used. */
void orc_fv_boundary_ghosts(int dim, int P, int g, double* luh, int face, int rule);

double orc_fv_patchgrid_step_2d(int scheme, int P, int npx, int npy, int planar,
                                double* luh, const double* dx) {
  return orc_fv_patchgrid_step_2d_bc(scheme, P, npx, npy, planar, luh, dx, NULL);
}

/* bc (nullable: periodic) = boundary rule per dimension; a domain-boundary
 * face of a patch takes its ghosts from the patch itself
 * (orc_fv_boundary_ghosts, FiniteVolumesSolver::mergeWithBoundaryData) */
double orc_fv_patchgrid_step_2d_bc(int scheme, int P, int npx, int npy, int planar,
                                   double* luh, const double* dx, const int* bc) {
  const int g = scheme == 0 ? 1 : 2, V = 5, S = P + 2 * g;
  const long per = (long)S * S * V, np = (long)npx * npy;
  long p;
  for (p = 0; p < np; p++) {
    const int px = (int)(p % npx), py = (int)(p / npx);
    double* u = luh + p * per;
    const double* L = luh + ((long)py * npx + (px + npx - 1) % npx) * per;
    const double* R = luh + ((long)py * npx + (px + 1) % npx) * per;
    const double* Bm = luh + ((long)((py + npy - 1) % npy) * npx + px) * per;
    const double* T = luh + ((long)((py + 1) % npy) * npx + px) * per;
    const int wl = bc && bc[0] && px == 0, wr = bc && bc[0] && px == npx - 1;
    const int wb = bc && bc[1] && py == 0, wt = bc && bc[1] && py == npy - 1;
    int i, k;
    for (i = g; i < g + P; i++)
      for (k = 0; k < g; k++) {
        if (!wl) memcpy(u + ((long)i * S + k) * V, L + ((long)i * S + P + k) * V, sizeof(double) * V);
        if (!wr) memcpy(u + ((long)i * S + g + P + k) * V, R + ((long)i * S + g + k) * V, sizeof(double) * V);
        if (!wb) memcpy(u + ((long)k * S + i) * V, Bm + ((long)(P + k) * S + i) * V, sizeof(double) * V);
        if (!wt) memcpy(u + ((long)(g + P + k) * S + i) * V, T + ((long)(g + k) * S + i) * V, sizeof(double) * V);
      }
    if (wl) orc_fv_boundary_ghosts(2, P, g, u, 0, bc[0]);
    if (wr) orc_fv_boundary_ghosts(2, P, g, u, 1, bc[0]);
    if (wb) orc_fv_boundary_ghosts(2, P, g, u, 2, bc[1]);
    if (wt) orc_fv_boundary_ghosts(2, P, g, u, 3, bc[1]);
  }
  double dt = DBL_MAX;
  for (p = 0; p < np; p++) {
    const double d = orc_fv_stable_dt_2d(P, g, V, 0, planar, luh + p * per, dx, 0.9);
    if (d < dt) dt = d;
  }
  double* old = (double*)malloc(sizeof(double) * per);
  for (p = 0; p < np; p++) {
    memcpy(old, luh + p * per, sizeof(double) * per);
    if (scheme == 0) orc_fv_godunov_2d(P, g, V, 0, planar, luh + p * per, old, dx, dt);
    else orc_fv_musclhancock_2d(P, g, V, 0, planar, luh + p * per, old, dx, dt);
  }
  free(old);
  return dt;
}

/* ---- AMR transfer operators (kernels/aderdg/generic/c/{2d,3d}/amrRoutines.cpph) ----
 * k-dimensional nodal arrays [n_{k-1}]...[n_0][var] (node index 0 fastest),
 * 3:1 refinement per level with the fine-grid projector
 * P[s][n][m] = phi_n((s + x_m) / 3) (DGMatrices.cpp fineGridProjector1d). */
static long ipow_l(long b, int e) { long r = 1; while (e-- > 0) r *= b; return r; }

/* single level: out[m] (+)= sum_n in[n] * prod_d P[s_d][n_d][m_d] */
static void amr_prolong1(int k, int order, int nvar, double* out, const double* in, const int* s) {
  const int B = order + 1;
  const long nn = ipow_l(B, k);
  long m, n;
  int v, d;
  for (m = 0; m < nn; m++)
    for (v = 0; v < nvar; v++) {
      double acc = 0.0;
      /* loop order of the reference: outer node index slowest */
      for (n = 0; n < nn; n++) {
        long mm = m, nr = n;
        double t = in[n * nvar + v];
        for (d = 0; d < k; d++) {
          t *= exa_fgp[order][s[d]][nr % B][mm % B];
          mm /= B;
          nr /= B;
        }
        acc += t;
      }
      out[m * nvar + v] += acc;
    }
}

/* single level: out[m] (+)= sum_n (prod w[n_d]) (prod P[s_d][m_d][n_d]) in[n]
 *                        / prod w[m_d] / 3^k */
static void amr_restrict1(int k, int order, int nvar, double* out, const double* in, const int* s) {
  const int B = order + 1;
  const long nn = ipow_l(B, k);
  const double* w = exa_gl_weights[order];
  long m, n;
  int v, d;
  for (m = 0; m < nn; m++)
    for (v = 0; v < nvar; v++) {
      double acc = 0.0;
      for (n = 0; n < nn; n++) {
        long mm, nr = n;
        double t = 1.0;
        for (d = 0; d < k; d++) { t *= w[nr % B]; nr /= B; }
        mm = m; nr = n;
        for (d = 0; d < k; d++) {
          t *= exa_fgp[order][s[d]][mm % B][nr % B];
          mm /= B;
          nr /= B;
        }
        t *= in[n * nvar + v];
        mm = m;
        for (d = 0; d < k; d++) { t /= w[mm % B]; mm /= B; }
        t /= (double)ipow_l(3, k);
        acc += t;
      }
      out[m * nvar + v] += acc;
    }
}

void orc_amr_prolongation(int k, int order, int nvar, double* fine, const double* coarse,
                          int level_delta, const int* index) {
  const int B = order + 1;
  const long nn = ipow_l(B, k) * nvar;
  double* a = (double*)malloc(sizeof(double) * nn);
  double* b = (double*)malloc(sizeof(double) * nn);
  int cur[3] = {0, 0, 0}, sub[3], d, l;
  memcpy(a, coarse, sizeof(double) * nn);
  for (d = 0; d < k; d++) cur[d] = index[d];
  for (l = 1; l <= level_delta; l++) {
    const long sig = ipow_l(3, level_delta - l);
    for (d = 0; d < k; d++) {
      sub[d] = (int)(cur[d] / sig);
      cur[d] = (int)(cur[d] % sig);
    }
    memset(b, 0, sizeof(double) * nn);
    amr_prolong1(k, order, nvar, b, a, sub);
    { double* t = a; a = b; b = t; }
  }
  memcpy(fine, a, sizeof(double) * nn);
  free(a);
  free(b);
}

void orc_amr_restriction(int k, int order, int nvar, double* coarse, const double* fine,
                         int level_delta, const int* index) {
  const int B = order + 1;
  const long nn = ipow_l(B, k) * nvar;
  double* a = (double*)malloc(sizeof(double) * nn);
  double* b = (double*)malloc(sizeof(double) * nn);
  int cur[3] = {0, 0, 0}, sub[3], d, l;
  long i;
  memcpy(a, fine, sizeof(double) * nn);
  for (d = 0; d < k; d++) cur[d] = index[d];
  for (l = 1; l <= level_delta; l++) {
    for (d = 0; d < k; d++) {
      sub[d] = cur[d] % 3;
      cur[d] /= 3;
    }
    memset(b, 0, sizeof(double) * nn);
    amr_restrict1(k, order, nvar, b, a, sub);
    { double* t = a; a = b; b = t; }
  }
  for (i = 0; i < nn; i++) coarse[i] += a[i];
  free(a);
  free(b);
}

/* ------------------------------------------------------------------ */
/* Counter-based noise: splitmix64 of (seed, index). */
double orc_noise_u01(unsigned long long seed, unsigned long long idx) {
  unsigned long long z = seed + 0x9E3779B97F4A7C15ULL * (idx + 1ULL);
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
  z = z ^ (z >> 31);
  return (double)(z >> 11) * (1.0 / 9007199254740992.0);
}

static void prim_to_cons(double rho, double u, double v, double w, double p, double* Q) {
  Q[0] = rho;
  Q[1] = rho * u;
  Q[2] = rho * v;
  Q[3] = rho * w;
  Q[4] = p / (GAMMA - 1) + 0.5 * rho * (u * u + v * v + w * w);
}

/* Point-wise initial state (the analogue of the user's adjustPointSolution,
 * kernels/aderdg/generic/c/3d/solutionAdjustment.cpph:18-52). */
static void ic_point(int kind, double param, double x, double y, double noise,
                     double* Q) {
  const double pi = 3.14159265358979323846;
  if (kind == 0) {
    /* isentropic vortex (Shu), centre (0.5,0.5), length scale 0.1 */
    const double eps = param, R = 0.1;
    const double xb = (x - 0.5) / R, yb = (y - 0.5) / R;
    const double r2 = xb * xb + yb * yb;
    const double e = exp(0.5 * (1.0 - r2));
    const double u = 1.0 - eps / (2 * pi) * yb * e;
    const double v = 1.0 + eps / (2 * pi) * xb * e;
    const double T = 1.0 - (GAMMA - 1) * eps * eps / (8 * GAMMA * pi * pi) * e * e;
    const double rho = pow(T, 1.0 / (GAMMA - 1));
    const double p = rho * T;
    prim_to_cons(rho * (1.0 + noise), u, v, 0.0, p, Q);
  } else {
    const double rho = 1.0 + param * sin(2 * pi * (x + y));
    prim_to_cons(rho * (1.0 + noise), 1.0, 1.0, 0.0, 1.0, Q);
  }
}

void orc_aderdg_grid_ic(int dim, int order, const int* n, const double* dx,
                        double* luh, int kind, double param,
                        unsigned long long seed, double noise_amp) {
  const int B = order + 1;
  const int nn = dim == 3 ? B * B * B : B * B;
  const long nc = ncells_of(dim, n);
#pragma omp parallel for schedule(static)
  for (long c = 0; c < nc; c++) {
    const int cx = (int)(c % n[0]), cy = (int)((c / n[0]) % n[1]);
    for (int s = 0; s < nn; s++) {
      const int ix = s % B, iy = (s / B) % B;
      const double x = (cx + exa_gl_nodes[order][ix]) * dx[0];
      const double y = (cy + exa_gl_nodes[order][iy]) * dx[1];
      const unsigned long long g = (unsigned long long)c * nn + s;
      const double nz = noise_amp != 0.0 ? noise_amp * (2.0 * orc_noise_u01(seed, g) - 1.0) : 0.0;
      ic_point(kind, param, x, y, nz, luh + (c * nn + s) * 5);
    }
  }
}

/* ------------------------------------------------------------------ */
/* FV Rusanov: kernels/finitevolumes/riemannsolvers/c/rusanov.cpph:24-83
 * (2D) / :98-156 (3D), without the non-conservative product: s_max over
 * the eigenvalues of both sides, fL = fR = 0.5 s_max (qL - qR) +
 * 0.5 (FL_d + FR_d), flux arrays zero before the PDE fills them.  The PDE
 * comes as callbacks (the reference's unit test drives the same kernel
 * with a mock solver, RusanovTest.cpp:33-90); nvar <= 16. */
double orc_rusanov_pde(int dim, int nvar, orc_flux_fn flux, orc_eig_fn eig, void* ctx,
                       double* fL, double* fR, const double* qL, const double* qR, int d) {
  double sL[16], sR[16];
  eig(ctx, qL, d, sL);
  eig(ctx, qR, d, sR);
  double smax = -1.0;
  for (int i = 0; i < nvar; i++) smax = fabs(sL[i]) > smax ? fabs(sL[i]) : smax;
  for (int i = 0; i < nvar; i++) smax = fabs(sR[i]) > smax ? fabs(sR[i]) : smax;
  double FL[3 * 16], FR[3 * 16];
  for (int i = 0; i < 3 * 16; i++) FL[i] = FR[i] = 0.0;
  flux(ctx, qL, FL);
  flux(ctx, qR, FR);
  for (int i = 0; i < nvar; i++) {
    double f = 0.5 * smax * (qL[i] - qR[i]);
    f += 0.5 * (FL[nvar * d + i] + FR[nvar * d + i]);
    fL[i] = f;
    fR[i] = f;
  }
  (void)dim;
  return smax;
}

struct euler_ctx { int dim, planar; };
static void euler_flux_cb(void* c, const double* q, double* F) {
  const struct euler_ctx* e = (const struct euler_ctx*)c;
  orc_euler_flux(e->dim, e->planar, q, F);
}
static void euler_eig_cb(void* c, const double* q, int d, double* lam) {
  orc_euler_eigenvalues(((const struct euler_ctx*)c)->planar, q, d, lam);
}

/* the Euler PDE's Rusanov flux (5 variables) */
double orc_rusanov(int dim, int nvar, int npar, int planar, double* fL,
                   double* fR, const double* qL, const double* qR, int d) {
  struct euler_ctx e = {dim, planar};
  (void)npar;
  return orc_rusanov_pde(dim, nvar, euler_flux_cb, euler_eig_cb, &e, fL, fR, qL, qR, d);
}

/* FV Godunov 2D: kernels/finitevolumes/godunov/c/2d/godunov.cpph:33-120 */
double orc_fv_godunov_2d(int P, int g, int V, int npar, int planar,
                         double* luh_new, const double* luh, const double* dx,
                         double dt) {
  const int D = V + npar, S = P + 2 * g, pb = g, pe = g + P;
  const double h[2] = {dx[0] / P, dx[1] / P};
  const double cfl = 0.9; /* AbstractGenericFiniteVolumesSolverHeader.template:34 */
#define IX(j, k, l) ((((long)(j)) * S + (k)) * D + (l))
  double fL[5], fR[5], dtmax = DBL_MAX;
  for (int j = pb; j < pe; j++)
    for (int k = pb - 1; k < pe; k++) {
      const double s = orc_rusanov(2, V, npar, planar, fL, fR, luh + IX(j, k, 0), luh + IX(j, k + 1, 0), 0);
      const double c = cfl / 2 * h[0] / s;
      dtmax = c < dtmax ? c : dtmax;
      for (int l = 0; l < V; l++) {
        luh_new[IX(j, k, l)] -= dt / h[0] * fL[l];
        luh_new[IX(j, k + 1, l)] += dt / h[0] * fR[l];
      }
    }
  for (int j = pb - 1; j < pe; j++)
    for (int k = pb; k < pe; k++) {
      const double s = orc_rusanov(2, V, npar, planar, fL, fR, luh + IX(j, k, 0), luh + IX(j + 1, k, 0), 1);
      const double c = cfl / 2 * h[1] / s;
      dtmax = c < dtmax ? c : dtmax;
      for (int l = 0; l < V; l++) {
        luh_new[IX(j, k, l)] -= dt / h[1] * fL[l];
        luh_new[IX(j + 1, k, l)] += dt / h[1] * fR[l];
      }
    }
#undef IX
  return dtmax;
}

/* minmod: kernels/finitevolumes/musclhancock/c/2d/musclhancock.cpph:27-40 */
static double minmod(double a, double b) {
  if (a * b < 0.0) return 0.0;
  return fabs(a) < fabs(b) ? a : b;
}

/* FV MUSCL-Hancock 2D: kernels/finitevolumes/musclhancock/c/2d/
 * musclhancock.cpph:50-240 (CFL 0.99 from musclhancock.h:29).  The ghost
 * cells next to the patch are extrapolated but not half-step evolved
 * (:132-170), exactly as in the reference. */
double orc_fv_musclhancock_2d(int P, int g, int V, int npar, int planar,
                              double* luh_new, const double* luh,
                              const double* dx, double dt) {
  const int D = V + npar, S = P + 2 * g, pb = g, pe = g + P;
  const double h[2] = {dx[0] / P, dx[1] / P};
  const double cfl = 0.99;
  const long nv = (long)S * S * V;
#define IX(j, k, l) ((((long)(j)) * S + (k)) * D + (l))
#define IW(j, k, l) ((((long)(j)) * S + (k)) * V + (l))
#define ISL(j, k, d, l) (((((long)(j)) * S + (k)) * 2 + (d)) * V + (l))
  double* slope = (double*)calloc(nv * 2, sizeof(double));
  double* wLx = (double*)calloc(nv, sizeof(double));
  double* wRx = (double*)calloc(nv, sizeof(double));
  double* wLy = (double*)calloc(nv, sizeof(double));
  double* wRy = (double*)calloc(nv, sizeof(double));
  double* slopet = (double*)calloc(nv, sizeof(double));
  /* slopes :79-98 */
  for (int j = pb; j < pe; j++)
    for (int k = pb - 1; k < pe + 1; k++)
      for (int l = 0; l < V; l++)
        slope[ISL(j, k, 0, l)] = minmod(luh[IX(j, k + 1, l)] - luh[IX(j, k, l)],
                                        luh[IX(j, k, l)] - luh[IX(j, k - 1, l)]) / h[0];
  for (int j = pb - 1; j < pe + 1; j++)
    for (int k = pb; k < pe; k++)
      for (int l = 0; l < V; l++)
        slope[ISL(j, k, 1, l)] = minmod(luh[IX(j + 1, k, l)] - luh[IX(j, k, l)],
                                        luh[IX(j, k, l)] - luh[IX(j - 1, k, l)]) / h[1];
  /* boundary extrapolation :100-124 */
  for (int j = pb; j < pe; j++)
    for (int k = pb - 1; k < pe + 1; k++)
      for (int l = 0; l < V; l++) {
        wLx[IW(j, k, l)] = luh[IX(j, k, l)] - 0.5 * h[0] * slope[ISL(j, k, 0, l)];
        wRx[IW(j, k, l)] = luh[IX(j, k, l)] + 0.5 * h[0] * slope[ISL(j, k, 0, l)];
      }
  for (int j = pb - 1; j < pe + 1; j++)
    for (int k = pb; k < pe; k++)
      for (int l = 0; l < V; l++) {
        wLy[IW(j, k, l)] = luh[IX(j, k, l)] - 0.5 * h[1] * slope[ISL(j, k, 1, l)];
        wRy[IW(j, k, l)] = luh[IX(j, k, l)] + 0.5 * h[1] * slope[ISL(j, k, 1, l)];
      }
  /* half-step evolution of the interior cells :126-170 (no source) */
  for (int j = pb; j < pe; j++)
    for (int k = pb; k < pe; k++) {
      double* Qt = slopet + IW(j, k, 0);
      double F[10];
      orc_euler_flux(2, planar, wLx + IW(j, k, 0), F);
      for (int l = 0; l < V; l++) Qt[l] += F[l] / h[0];
      orc_euler_flux(2, planar, wRx + IW(j, k, 0), F);
      for (int l = 0; l < V; l++) Qt[l] -= F[l] / h[0];
      orc_euler_flux(2, planar, wLy + IW(j, k, 0), F);
      for (int l = 0; l < V; l++) Qt[l] += F[5 + l] / h[1];
      orc_euler_flux(2, planar, wRy + IW(j, k, 0), F);
      for (int l = 0; l < V; l++) Qt[l] -= F[5 + l] / h[1];
      for (int l = 0; l < V; l++) {
        wLx[IW(j, k, l)] += 0.5 * dt * Qt[l];
        wRx[IW(j, k, l)] += 0.5 * dt * Qt[l];
        wLy[IW(j, k, l)] += 0.5 * dt * Qt[l];
        wRy[IW(j, k, l)] += 0.5 * dt * Qt[l];
      }
    }
  /* Riemann problems :172-214 */
  double fL[5], fR[5], dtmax = DBL_MAX;
  for (int j = pb; j < pe; j++)
    for (int k = pb - 1; k < pe; k++) {
      const double s = orc_rusanov(2, V, 0, planar, fL, fR, wRx + IW(j, k, 0), wLx + IW(j, k + 1, 0), 0);
      const double c = cfl / 2 * h[0] / s;
      dtmax = c < dtmax ? c : dtmax;
      for (int l = 0; l < V; l++) {
        luh_new[IX(j, k, l)] -= dt / h[0] * fL[l];
        luh_new[IX(j, k + 1, l)] += dt / h[0] * fR[l];
      }
    }
  for (int j = pb - 1; j < pe; j++)
    for (int k = pb; k < pe; k++) {
      const double s = orc_rusanov(2, V, 0, planar, fL, fR, wRy + IW(j, k, 0), wLy + IW(j + 1, k, 0), 1);
      const double c = cfl / 2 * h[1] / s;
      dtmax = c < dtmax ? c : dtmax;
      for (int l = 0; l < V; l++) {
        luh_new[IX(j, k, l)] -= dt / h[1] * fL[l];
        luh_new[IX(j + 1, k, l)] += dt / h[1] * fR[l];
      }
    }
  free(slope); free(wLx); free(wRx); free(wLy); free(wRy); free(slopet);
#undef IX
#undef IW
#undef ISL
  return dtmax;
}

/* FV CFL: kernels/finitevolumes/commons/c/commons.cpph:26-67 */
double orc_fv_stable_dt_2d(int P, int g, int V, int npar, int planar,
                           const double* luh, const double* dx, double cfl) {
  const int D = V + npar, S = P + 2 * g;
  double dtmax = DBL_MAX;
  for (int j = g; j < g + P; j++)
    for (int k = g; k < g + P; k++) {
      const double* q = luh + ((long)j * S + k) * D;
      for (int d = 0; d < 2; d++) {
        double lam[5], s = 0.0;
        orc_euler_eigenvalues(planar, q, d, lam);
        for (int v = 0; v < V; v++) s = fabs(lam[v]) > s ? fabs(lam[v]) : s;
        const double c = cfl / 2 * (dx[d] / P) / s;
        dtmax = c < dtmax ? c : dtmax;
      }
    }
  return dtmax;
}

/* Periodic ghost layers of a single patch (stands in for the neighbour
 * merging of commons.cpph:337-405 when the patch is its own neighbour). */
void orc_fv_periodic_ghosts_2d(int P, int g, int D, double* luh) {
  const int S = P + 2 * g;
  for (int j = 0; j < S; j++)
    for (int k = 0; k < S; k++) {
      if (j >= g && j < g + P && k >= g && k < g + P) continue;
      const int sj = g + ((j - g) % P + P) % P;
      const int sk = g + ((k - g) % P + P) % P;
      memcpy(luh + ((long)j * S + k) * D, luh + ((long)sj * S + sk) * D, sizeof(double) * D);
    }
}

double orc_fv_patch_step_2d(int scheme, int P, int planar, double* luh,
                            const double* dx, double dt_fixed,
                            double* max_admissible_dt) {
  const int g = scheme == 0 ? 1 : 2, V = 5, S = P + 2 * g;
  orc_fv_periodic_ghosts_2d(P, g, V, luh);
  const double dt = dt_fixed > 0 ? dt_fixed : orc_fv_stable_dt_2d(P, g, V, 0, planar, luh, dx, 0.9);
  double* old = (double*)malloc(sizeof(double) * S * S * V);
  memcpy(old, luh, sizeof(double) * S * S * V);
  double adm;
  if (scheme == 0) adm = orc_fv_godunov_2d(P, g, V, 0, planar, luh, old, dx, dt);
  else adm = orc_fv_musclhancock_2d(P, g, V, 0, planar, luh, old, dx, dt);
  if (max_admissible_dt) *max_admissible_dt = adm;
  free(old);
  return dt;
}

/* ------------------------------------------------------------------ */
/* A-posteriori subcell limiter (kernels/limiter/generic/c/Limiter.cpp).
 * Direct tensor sums in the reference's loop order; tables uh2lim, uh2lob,
 * lim2uh are the projections of LimiterProjectionMatrices.cpp:40-140 from
 * dg_tables.h. */
static int lim_subcells(int order) { return 2 * order + 1; }

/* projectOnFVLimiterSpace, Limiter.cpp:23-64 */
void orc_limiter_project_on_fv(int dim, int order, int nvar, int ghost, const double* luh,
                               double* lim) {
  const int B = order + 1, S = lim_subcells(order), SG = S + 2 * ghost;
  const int B3 = dim == 3 ? B : 1, S3 = dim == 3 ? S : 1, G3 = dim == 3 ? ghost : 0;
  const double(*U)[EXA_LIM_MAX_SUBCELLS] = exa_uh2lim[order];
  int x, y, z, v, ix, iy, iz;
  for (z = G3; z < S3 + G3; z++)
    for (y = ghost; y < S + ghost; y++)
      for (x = ghost; x < S + ghost; x++)
        for (v = 0; v < nvar; v++) {
          double acc = 0.0;
          for (iz = 0; iz < B3; iz++)
            for (iy = 0; iy < B; iy++)
              for (ix = 0; ix < B; ix++) {
                double t = luh[((iz * B + iy) * B + ix) * nvar + v];
                if (dim == 3) t *= U[iz][z - G3];
                acc += t * U[iy][y - ghost] * U[ix][x - ghost];
              }
          lim[(((long)z * SG + y) * SG + x) * nvar + v] = acc;
        }
}

/* projectOnDGSpace, Limiter.cpp:67-110 */
void orc_limiter_project_on_dg(int dim, int order, int nvar, int ghost, const double* lim,
                               double* luh) {
  const int B = order + 1, S = lim_subcells(order), SG = S + 2 * ghost;
  const int B3 = dim == 3 ? B : 1, S3 = dim == 3 ? S : 1, G3 = dim == 3 ? ghost : 0;
  const double(*L)[10] = exa_lim2uh[order];
  int x, y, z, v, ix, iy, iz;
  for (z = 0; z < B3; z++)
    for (y = 0; y < B; y++)
      for (x = 0; x < B; x++)
        for (v = 0; v < nvar; v++) {
          double acc = 0.0;
          for (iz = G3; iz < S3 + G3; iz++)
            for (iy = ghost; iy < S + ghost; iy++)
              for (ix = ghost; ix < S + ghost; ix++) {
                double t = lim[(((long)iz * SG + iy) * SG + ix) * nvar + v];
                if (dim == 3) t *= L[iz - G3][z];
                acc += t * L[iy - ghost][y] * L[ix - ghost][x];
              }
          luh[((z * B + y) * B + x) * nvar + v] = acc;
        }
}

/* min/max of the observables (= first nobs values) over a tensor-product
 * evaluation of luh with the 1D table T[k][i] (n points per direction) */
static void lim_eval_min_max(int dim, int order, int nvar, int nobs, const double* luh,
                             const double* T, int tstride, int n, double* mn, double* mx) {
  const int B = order + 1, B3 = dim == 3 ? B : 1, n3 = dim == 3 ? n : 1;
  int x, y, z, v, ix, iy, iz;
  for (z = 0; z < n3; z++)
    for (y = 0; y < n; y++)
      for (x = 0; x < n; x++)
        for (v = 0; v < nobs; v++) {
          double acc = 0.0;
          for (iz = 0; iz < B3; iz++)
            for (iy = 0; iy < B; iy++)
              for (ix = 0; ix < B; ix++) {
                double t = luh[((iz * B + iy) * B + ix) * nvar + v];
                if (dim == 3) t *= T[iz * tstride + z];
                acc += t * T[iy * tstride + y] * T[ix * tstride + x];
              }
          if (acc < mn[v]) mn[v] = acc;
          if (acc > mx[v]) mx[v] = acc;
        }
}

/* findCellLocalMinAndMax, Limiter.cpp:212-251, with
 * compareWithADERDGSolutionAtGaussLobattoNodes (:258-306) and
 * compareWithADERDGSolutionAtFVSubcellCenters (:312-368) */
static void lim_cell_local_min_max(int dim, int order, int nvar, int nobs, const double* luh,
                                   double* mn, double* mx) {
  const int B = order + 1, npts = dim == 3 ? B * B * B : B * B;
  int i, v;
  for (v = 0; v < nobs; v++) {
    mn[v] = DBL_MAX;
    mx[v] = -DBL_MAX;
  }
  for (i = 0; i < npts; i++)
    for (v = 0; v < nobs; v++) {
      const double q = luh[i * nvar + v];
      if (q < mn[v]) mn[v] = q;
      if (q > mx[v]) mx[v] = q;
    }
  lim_eval_min_max(dim, order, nvar, nobs, luh, &exa_uh2lob[order][0][0], 10, B, mn, mx);
  lim_eval_min_max(dim, order, nvar, nobs, luh, &exa_uh2lim[order][0][0],
                   EXA_LIM_MAX_SUBCELLS, lim_subcells(order), mn, mx);
}

static void lim_copy_to_faces(int dim, int nobs, double* obs_min, double* obs_max) {
  int f, v;
  for (f = 1; f < 2 * dim; f++)
    for (v = 0; v < nobs; v++) {
      obs_min[f * nobs + v] = obs_min[v];
      obs_max[f * nobs + v] = obs_max[v];
    }
}

void orc_limiter_local_min_max(int dim, int order, int nvar, int nobs, const double* luh,
                               double* obs_min, double* obs_max) {
  lim_cell_local_min_max(dim, order, nvar, nobs, luh, obs_min, obs_max);
  lim_copy_to_faces(dim, nobs, obs_min, obs_max);
}

/* findCellLocalLimiterMinAndMax, Limiter.cpp:170-207 */
void orc_limiter_fv_min_max(int dim, int order, int nvar, int nobs, int ghost,
                            const double* lim, double* obs_min, double* obs_max) {
  const int S = lim_subcells(order), SG = S + 2 * ghost;
  const int S3 = dim == 3 ? S : 1, G3 = dim == 3 ? ghost : 0;
  int x, y, z, v;
  for (v = 0; v < nobs; v++) {
    obs_min[v] = DBL_MAX;
    obs_max[v] = -DBL_MAX;
  }
  for (z = G3; z < S3 + G3; z++)
    for (y = ghost; y < S + ghost; y++)
      for (x = ghost; x < S + ghost; x++)
        for (v = 0; v < nobs; v++) {
          const double q = lim[(((long)z * SG + y) * SG + x) * nvar + v];
          if (q < obs_min[v]) obs_min[v] = q;
          if (q > obs_max[v]) obs_max[v] = q;
        }
  lim_copy_to_faces(dim, nobs, obs_min, obs_max);
}

/* discreteMaximumPrincipleAndMinAndMaxSearch, Limiter.cpp:113-167 */
int orc_limiter_dmp(int dim, int order, int nvar, int nobs, const double* luh, double relaxation,
                    double difference_scaling, double* obs_min, double* obs_max) {
  double mn[64], mx[64];
  int ok = 1, v, i;
  if (nobs > 64) return 0;
  lim_cell_local_min_max(dim, order, nvar, nobs, luh, mn, mx);
  for (v = 0; v < nobs; v++) {
    double bmin = obs_min[v], bmax = obs_max[v], sd;
    for (i = 1; i < 2 * dim; i++) {
      bmin = fmin(bmin, obs_min[i * nobs + v]);
      bmax = fmax(bmax, obs_max[i * nobs + v]);
    }
    sd = (bmax - bmin) * difference_scaling;
    sd = fmax(sd, relaxation);
    if (mn[v] < bmin - sd || mx[v] > bmax + sd) ok = 0;
    obs_min[v] = mn[v];
    obs_max[v] = mx[v];
    obs_min[v + nobs] = bmin;
    obs_max[v + nobs] = bmax;
  }
  return ok;
}

/* ------------------------------------------------------------------ */
/* Limiting ADER-DG on a uniform 2D or 3D grid: LimitingADERDGSolver
 * (exahype/solvers/LimitingADERDGSolver.cpp) restated for a uniform mesh
 * with global time stepping, on top of the restated kernels above.  Cells
 * x fastest; n[2] is ignored in 2D.  bc (nullable: all periodic) holds the
 * boundary rule per dimension, 0 periodic, 1 outflow, 2 reflecting wall. */
static long lim_nb(int dim, const int* n, const int* bc, long c, int f) {
  int co[3];
  const int d = f >> 1, up = f & 1;
  co[0] = (int)(c % n[0]);
  co[1] = (int)((c / n[0]) % n[1]);
  co[2] = dim == 3 ? (int)(c / ((long)n[0] * n[1])) : 0;
  if (up ? co[d] == n[d] - 1 : co[d] == 0) {
    if (bc && bc[d]) return -1; /* the domain boundary */
    co[d] = up ? 0 : n[d] - 1;
  } else {
    co[d] += up ? 1 : -1;
  }
  return ((long)co[2] * n[1] + co[1]) * n[0] + co[0];
}

static long lim_ncells(int dim, const int* n) { return (long)n[0] * n[1] * (dim == 3 ? n[2] : 1); }

/* mergeSolutionMinMaxOnFace (:1792-1853): face f keeps the extrema of the
 * cell (face block 0) and of its neighbour across f; a domain-boundary face
 * is never merged and keeps the cell's own */
static void lim_merge_bounds(int dim, const int* n, const int* bc, int nobs, double* bmin, double* bmax) {
  const long nc = lim_ncells(dim, n);
  const int nf = 2 * dim;
  double* loc = (double*)malloc(sizeof(double) * nc * 2 * nobs);
  long c;
  int f, v;
  for (c = 0; c < nc; c++)
    for (v = 0; v < nobs; v++) {
      loc[(c * 2) * nobs + v] = bmin[c * nf * nobs + v];
      loc[(c * 2 + 1) * nobs + v] = bmax[c * nf * nobs + v];
    }
  for (c = 0; c < nc; c++)
    for (f = 0; f < nf; f++) {
      const long nb0 = lim_nb(dim, n, bc, c, f), nb = nb0 < 0 ? c : nb0;
      for (v = 0; v < nobs; v++) {
        const double mo = loc[(c * 2) * nobs + v], mn = loc[(nb * 2) * nobs + v];
        const double xo = loc[(c * 2 + 1) * nobs + v], xn = loc[(nb * 2 + 1) * nobs + v];
        bmin[(c * nf + f) * nobs + v] = mn < mo ? mn : mo;
        bmax[(c * nf + f) * nobs + v] = xo < xn ? xn : xo;
      }
    }
  free(loc);
}

void orc_limiting_initial_bounds(int dim, int order, const int* n, const double* luh, int nobs, double* bmin,
                                 double* bmax, const int* bc) {
  const long nc = lim_ncells(dim, n);
  const int B = order + 1, npc = dim == 3 ? B * B * B : B * B;
  long c;
  for (c = 0; c < nc; c++)
    orc_limiter_local_min_max(dim, order, 5, nobs, luh + c * npc * 5, bmin + c * 2 * dim * nobs,
                              bmax + c * 2 * dim * nobs);
  lim_merge_bounds(dim, n, bc, nobs, bmin, bmax);
}

/* point (z, y, x) of a [S]^dim patch */
static long lim_pt(int dim, int SG, int z, int y, int x) {
  return dim == 3 ? ((long)z * SG + y) * SG + x : (long)y * SG + x;
}

void orc_fv_boundary_ghosts(int dim, int P, int g, double* luh, int face, int rule) {
  const int SG = P + 2 * g, d = face >> 1, up = face & 1, amax = dim == 3 ? P : 1;
  int a, b, k, m;
  for (a = 0; a < amax; a++)
    for (b = 0; b < P; b++)
      for (k = 0; k < g; k++) {
        /* ghost layer k and the interior layer it mirrors, along d; (a, b)
         * run over the other axes */
        const int gh = up ? g + P + k : k;
        /* 3D lower y and z faces: the reference's boundaryLayerExtraction
         * copies the first interior layer into every extracted layer
         * (commons.cpph:561 and 591 index patchBegin without + k),
         * so all those ghost layers repeat the layer next to the face */
        const int src = up ? g + P - 1 - k : (dim == 3 && d > 0 ? g : 2 * g - 1 - k);
        int dz, dy, dxx, sz, sy, sx;
        if (d == 0) {
          dz = sz = dim == 3 ? g + a : 0; dy = sy = g + b; dxx = gh; sx = src;
        } else if (d == 1) {
          dz = sz = dim == 3 ? g + a : 0; dxx = sx = g + b; dy = gh; sy = src;
        } else {
          dy = sy = g + a; dxx = sx = g + b; dz = gh; sz = src;
        }
        {
          double* o = luh + lim_pt(dim, SG, dz, dy, dxx) * 5;
          const double* q = luh + lim_pt(dim, SG, sz, sy, sx) * 5;
          for (m = 0; m < 5; m++) o[m] = rule == 2 && m == d + 1 ? -q[m] : q[m];
        }
      }
}

/* positive density and pressure at every node */
static int lim_admissible(int npc, int planar, const double* q) {
  int i;
  for (i = 0; i < npc; i++, q += 5) {
    const double j2 = planar ? q[1] * q[1] + q[2] * q[2] : q[1] * q[1] + q[2] * q[2] + q[3] * q[3];
    const double p = (GAMMA - 1) * (q[4] - 0.5 * j2 / q[0]);
    if (!(q[0] > 0.0 && p > 0.0 && isfinite(p))) return 0;
  }
  return 1;
}

double orc_limiting_grid_step(int dim, int order, const int* n, const double* dx, int planar, double* luh,
                              int* status, int* cure, double* bmin, double* bmax, int scheme, int nobs,
                              double relaxation, double difference_scaling, int steps_till_cured, int admissibility,
                              double dt, int dt_policy, double cfl, int* counts, const int* bc) {
  const int B = order + 1, npc = dim == 3 ? B * B * B : B * B, V = 5, S = 2 * order + 1;
  const int g = scheme == 0 ? 1 : 2, SG = S + 2 * g, nf = 2 * dim;
  const long nc = lim_ncells(dim, n), cell_d = (long)npc * V;
  const long patch_d = (long)(dim == 3 ? SG * SG * SG : SG * SG) * V;
  double* prev = (double*)malloc(sizeof(double) * nc * cell_d);
  double* patch = (double*)calloc(nc * patch_d, sizeof(double));
  double* old = (double*)malloc(sizeof(double) * patch_d);
  int* tmp = (int*)malloc(sizeof(int) * nc);
  int cnt[3] = {0, 0, 0};
  long c;
  int h, f, a, b, k, m;
  memcpy(prev, luh, sizeof(double) * nc * cell_d);
  /* 1. unlimited DG candidate */
  orc_aderdg_grid_step_bc(dim, order, planar, n, dx, luh, 2, cfl, dt, NULL, 0, bc);
  /* 2. DMP + admissibility -> status (determineLimiterStatusAfterSolutionUpdate) */
  for (c = 0; c < nc; c++) {
    int ok = orc_limiter_dmp(dim, order, V, nobs, luh + c * cell_d, relaxation, difference_scaling,
                             bmin + c * nf * nobs, bmax + c * nf * nobs);
    if (admissibility && !lim_admissible(npc, planar, luh + c * cell_d)) ok = 0;
    if (!ok) {
      cure[c] = steps_till_cured + 1;
      tmp[c] = 5;
    } else if (status[c] == 5) {
      if (cure[c] - 1 <= 0) {
        tmp[c] = 4;
        cure[c] = steps_till_cured;
      } else {
        tmp[c] = 5;
        cure[c] -= 1;
      }
    } else {
      tmp[c] = 0;
    }
  }
  /* spreading: four face-neighbour hops, status = max(own, neighbour - 1);
   * a domain-boundary face contributes status 0
   * (ADERDGSolver::mergeWithBoundaryOrEmptyCellMetadata :2933-2947) */
  for (h = 0; h < 4; h++) {
    for (c = 0; c < nc; c++) {
      int s = tmp[c];
      for (f = 0; f < nf; f++) {
        const long o = lim_nb(dim, n, bc, c, f);
        const int t = (o < 0 ? 0 : tmp[o]) - 1;
        if (t > s) s = t;
      }
      status[c] = s;
    }
    memcpy(tmp, status, sizeof(int) * nc);
  }
  /* 3. subcell patches of the previous solution (status >= NeighbourOfTroubled3) */
  for (c = 0; c < nc; c++) {
    if (status[c] >= 2) {
      orc_limiter_project_on_fv(dim, order, V, g, prev + c * cell_d, patch + c * patch_d);
      cnt[0]++;
    }
    if (status[c] >= 3) cnt[1]++;
    if (status[c] == 5) cnt[2]++;
  }
  /* 4. face ghosts of the FV cells' patches from the neighbours' patches
   * (FiniteVolumesSolver::mergeNeighbours / ghostLayerFilling), at a domain
   * boundary from the patch itself (orc_fv_boundary_ghosts) */
  for (c = 0; c < nc; c++) {
    if (status[c] < 3) continue;
    double* P = patch + c * patch_d;
    for (f = 0; f < nf; f++) {
      const int d = f >> 1, up = f & 1;
      const long o = lim_nb(dim, n, bc, c, f);
      const double* N = patch + o * patch_d;
      if (o < 0) {
        orc_fv_boundary_ghosts(dim, S, g, P, f, bc[d]);
        continue;
      }
      const int zmax = dim == 3 ? S : 1;
      for (a = 0; a < zmax; a++)
        for (b = 0; b < S; b++)
          for (k = 0; k < g; k++) {
            /* coordinates along the face: (a, b) over the two other axes */
            int dz, dy, dxx, sz, sy, sx;
            const int gh = up ? g + S + k : k, src = up ? g + k : S + k;
            if (d == 0) {
              dz = sz = dim == 3 ? g + a : 0; dy = sy = g + b; dxx = gh; sx = src;
            } else if (d == 1) {
              dz = sz = dim == 3 ? g + a : 0; dxx = sx = g + b; dy = gh; sy = src;
            } else {
              dy = sy = g + a; dxx = sx = g + b; dz = gh; sz = src;
            }
            for (m = 0; m < V; m++)
              P[lim_pt(dim, SG, dz, dy, dxx) * V + m] = N[lim_pt(dim, SG, sz, sy, sx) * V + m];
          }
    }
  }
  /* 5. FV step on those patches, projection back, limiter extrema
   * (recomputeSolution :1378-1441, determineLimiterMinAndMax :1118-1150) */
  for (c = 0; c < nc; c++) {
    if (status[c] < 3) continue;
    double* P = patch + c * patch_d;
    memcpy(old, P, sizeof(double) * patch_d);
    if (dim == 2) {
      if (scheme == 0) orc_fv_godunov_2d(S, g, V, 0, planar, P, old, dx, dt);
      else orc_fv_musclhancock_2d(S, g, V, 0, planar, P, old, dx, dt);
    } else {
      if (scheme == 0) orc_fv_godunov_3d(S, g, V, 0, P, old, dx, dt);
      else orc_fv_musclhancock_3d(S, g, V, 0, P, old, dx, dt);
    }
    orc_limiter_project_on_dg(dim, order, V, g, P, luh + c * cell_d);
    orc_limiter_fv_min_max(dim, order, V, nobs, g, P, bmin + c * nf * nobs, bmax + c * nf * nobs);
  }
  /* 6. next bounds */
  lim_merge_bounds(dim, n, bc, nobs, bmin, bmax);
  if (counts) memcpy(counts, cnt, sizeof(cnt));
  free(prev);
  free(patch);
  free(old);
  free(tmp);
  return orc_aderdg_grid_dt(dim, order, planar, n, dx, luh, dt_policy, cfl);
}

/* ------------------------------------------------------------------ */
/* 3D finite volumes on one patch, [z][y][x][D] with S = P + 2g per axis. */
#define I3(S, D, i, j, k, l) (((((long)(i)) * (S) + (j)) * (S) + (k)) * (D) + (l))

/* godunov::c::solutionUpdate, 3D (godunov/c/3d/godunov.cpph:35-143): x, y,
 * then z faces; luh_new (a copy of luh) is updated in place */
double orc_fv_godunov_3d(int P, int g, int V, int npar, double* luh_new, const double* luh, const double* dx,
                         double dt) {
  const int D = V + npar, S = P + 2 * g, pb = g, pe = g + P;
  const double h[3] = {dx[0] / P, dx[1] / P, dx[2] / P};
  const double cfl = 0.9;
  double fL[5], fR[5], dtmax = DBL_MAX;
  int i, j, k, l, d;
  for (d = 0; d < 3; d++)
    for (i = pb - (d == 2); i < pe; i++)
      for (j = pb - (d == 1); j < pe; j++)
        for (k = pb - (d == 0); k < pe; k++) {
          const int i2 = i + (d == 2), j2 = j + (d == 1), k2 = k + (d == 0);
          const double s = orc_rusanov(3, V, npar, 0, fL, fR, luh + I3(S, D, i, j, k, 0), luh + I3(S, D, i2, j2, k2, 0), d);
          const double c = cfl / 3 * h[d] / s;
          dtmax = c < dtmax ? c : dtmax;
          for (l = 0; l < V; l++) {
            luh_new[I3(S, D, i, j, k, l)] -= dt / h[d] * fL[l];
            luh_new[I3(S, D, i2, j2, k2, l)] += dt / h[d] * fR[l];
          }
        }
  return dtmax;
}

/* musclhancock::c::solutionUpdate, 3D (musclhancock/c/3d/musclhancock.cpph:
 * 50-311): minmod slopes, face extrapolation, half-step evolution of the
 * interior cells only, Rusanov on the evolved face values; CFL 0.99 */
double orc_fv_musclhancock_3d(int P, int g, int V, int npar, double* luh_new, const double* luh, const double* dx,
                              double dt) {
  const int D = V + npar, S = P + 2 * g, pb = g, pe = g + P;
  const double h[3] = {dx[0] / P, dx[1] / P, dx[2] / P};
  const double cfl = 0.99;
  const long nv = (long)S * S * S * V;
  double* slope = (double*)calloc(nv * 3, sizeof(double));
  double* wL[3];
  double* wR[3];
  double* slopet = (double*)calloc(nv, sizeof(double));
  double fL[5], fR[5], dtmax = DBL_MAX;
  int i, j, k, l, d;
  for (d = 0; d < 3; d++) {
    wL[d] = (double*)calloc(nv, sizeof(double));
    wR[d] = (double*)calloc(nv, sizeof(double));
  }
#define ISL3(i, j, k, d, l) ((((((long)(i)) * S + (j)) * S + (k)) * 3 + (d)) * V + (l))
  /* slopes and face values: direction d over the interior, with one ring
   * cell on each side along d (:70-150) */
  for (d = 0; d < 3; d++)
    for (i = pb - (d == 2); i < pe + (d == 2); i++)
      for (j = pb - (d == 1); j < pe + (d == 1); j++)
        for (k = pb - (d == 0); k < pe + (d == 0); k++) {
          const int di = d == 2, dj = d == 1, dk = d == 0;
          for (l = 0; l < V; l++) {
            const double u = luh[I3(S, D, i, j, k, l)];
            const double sl = minmod(luh[I3(S, D, i + di, j + dj, k + dk, l)] - u,
                                     u - luh[I3(S, D, i - di, j - dj, k - dk, l)]) / h[d];
            slope[ISL3(i, j, k, d, l)] = sl;
            wL[d][I3(S, V, i, j, k, l)] = u - 0.5 * h[d] * sl;
            wR[d][I3(S, V, i, j, k, l)] = u + 0.5 * h[d] * sl;
          }
        }
  /* half-step evolution increment of the interior cells (:152-205) */
  for (i = pb; i < pe; i++)
    for (j = pb; j < pe; j++)
      for (k = pb; k < pe; k++) {
        double* Qt = slopet + I3(S, V, i, j, k, 0);
        double F[15];
        for (d = 0; d < 3; d++) {
          orc_euler_flux(3, 0, wL[d] + I3(S, V, i, j, k, 0), F);
          for (l = 0; l < V; l++) Qt[l] += F[5 * d + l] / h[d];
          orc_euler_flux(3, 0, wR[d] + I3(S, V, i, j, k, 0), F);
          for (l = 0; l < V; l++) Qt[l] -= F[5 * d + l] / h[d];
        }
        for (l = 0; l < V; l++)
          for (d = 0; d < 3; d++) {
            wL[d][I3(S, V, i, j, k, l)] += 0.5 * dt * Qt[l];
            wR[d][I3(S, V, i, j, k, l)] += 0.5 * dt * Qt[l];
          }
      }
  /* Riemann problems (:207-290) */
  for (d = 0; d < 3; d++)
    for (i = pb - (d == 2); i < pe; i++)
      for (j = pb - (d == 1); j < pe; j++)
        for (k = pb - (d == 0); k < pe; k++) {
          const int i2 = i + (d == 2), j2 = j + (d == 1), k2 = k + (d == 0);
          const double s = orc_rusanov(3, V, 0, 0, fL, fR, wR[d] + I3(S, V, i, j, k, 0), wL[d] + I3(S, V, i2, j2, k2, 0), d);
          const double c = cfl / 3 * h[d] / s;
          dtmax = c < dtmax ? c : dtmax;
          for (l = 0; l < V; l++) {
            luh_new[I3(S, D, i, j, k, l)] -= dt / h[d] * fL[l];
            luh_new[I3(S, D, i2, j2, k2, l)] += dt / h[d] * fR[l];
          }
        }
#undef ISL3
  free(slope);
  free(slopet);
  for (d = 0; d < 3; d++) {
    free(wL[d]);
    free(wR[d]);
  }
  return dtmax;
}

/* commons::c::stableTimeStepSize, 3D (commons.cpph:410-455) */
double orc_fv_stable_dt_3d(int P, int g, int V, int npar, const double* luh, const double* dx, double cfl) {
  const int D = V + npar, S = P + 2 * g;
  double dtmax = DBL_MAX, lam[5];
  int i, j, k, d, l;
  for (i = g; i < g + P; i++)
    for (j = g; j < g + P; j++)
      for (k = g; k < g + P; k++)
        for (d = 0; d < 3; d++) {
          double s = 0.0;
          orc_euler_eigenvalues(0, luh + I3(S, D, i, j, k, 0), d, lam);
          for (l = 0; l < 5; l++) s = fabs(lam[l]) > s ? fabs(lam[l]) : s;
          {
            const double c = cfl / 3 * (dx[d] / P) / s;
            dtmax = c < dtmax ? c : dtmax;
          }
        }
  return dtmax;
}

/* periodic ghost layers of a single patch (every ghost cell, corners too) */
void orc_fv_periodic_ghosts_3d(int P, int g, int D, double* luh) {
  const int S = P + 2 * g;
  int i, j, k;
  for (i = 0; i < S; i++)
    for (j = 0; j < S; j++)
      for (k = 0; k < S; k++) {
        const int si = g + ((i - g) % P + P) % P, sj = g + ((j - g) % P + P) % P, sk = g + ((k - g) % P + P) % P;
        if (si == i && sj == j && sk == k) continue;
        memcpy(luh + I3(S, D, i, j, k, 0), luh + I3(S, D, si, sj, sk, 0), sizeof(double) * D);
      }
}

/* ------------------------------------------------------------------ */
/* Solution adjustment (kernels/aderdg/generic/c/3d/solutionAdjustment.cpph:
 * 17-52, 2D c/2d/solutionAdjustment.cpph): the adjustPointSolution hook at
 * every Gauss-Legendre node x = center + dx (xi - 1/2), loops i (z), j (y),
 * k (x) in 3D and i (y), j (x) in 2D; the hook is one of the built-in forms
 * of the device library (kind 1 sine wave, 2 isentropic vortex, 3 heat
 * source; when 0 = only at t == 0). */
#include "adjust_hooks.h"

void orc_solution_adjustment(int dim, int order, double* luh, const double* center, const double* dx, double t,
                             double dt, int kind, int when, const double* param) {
  const int B = order + 1;
  int i, j, k;
  double x[3];
  if (kind == 0 || (when == 0 && t != 0.0)) return;
  if (dim == 3) {
    for (i = 0; i < B; i++)
      for (j = 0; j < B; j++)
        for (k = 0; k < B; k++) {
          x[2] = center[2] + dx[2] * (exa_gl_nodes[order][i] - 0.5);
          x[1] = center[1] + dx[1] * (exa_gl_nodes[order][j] - 0.5);
          x[0] = center[0] + dx[0] * (exa_gl_nodes[order][k] - 0.5);
          orc_adjust_point(kind, dim, param, x, t, dt, luh + ((i * B + j) * B + k) * 5);
        }
  } else {
    for (i = 0; i < B; i++)
      for (j = 0; j < B; j++) {
        x[0] = center[0] + dx[0] * (exa_gl_nodes[order][j] - 0.5);
        x[1] = center[1] + dx[1] * (exa_gl_nodes[order][i] - 0.5);
        orc_adjust_point(kind, dim, param, x, t, dt, luh + (i * B + j) * 5);
      }
  }
}
