/* The built-in adjustPointSolution forms of the device library
 * (exa_adjust_t): kind 1 sine wave, 2 isentropic vortex, 3 heat source.
 * Shared by the oracle's solutionAdjustment restatement and by the driver
 * of the reference's own solutionAdjustment kernel (test infrastructure;
 * C and C++). */
#pragma once
#include <math.h>

static inline void orc_adjust_point(int kind, int dim, const double* param, const double* x, double t, double dt,
                             double* Q) {
  const double pi = 3.14159265358979323846, gam = 1.4;
  if (kind == 1) {
    const double rho = 1.0 + param[0] * sin(2 * pi * (x[0] + x[1]));
    const double u = 1.0, v = 1.0, p = 1.0;
    Q[0] = rho;
    Q[1] = rho * u;
    Q[2] = rho * v;
    Q[3] = 0.0;
    Q[4] = p / (gam - 1) + 0.5 * rho * (u * u + v * v);
  } else if (kind == 2) {
    const double eps = param[0], R = 0.1;
    const double xb = (x[0] - 0.5) / R, yb = (x[1] - 0.5) / R;
    const double r2 = xb * xb + yb * yb;
    const double e = exp(0.5 * (1.0 - r2));
    const double u = 1.0 - eps / (2 * pi) * yb * e;
    const double v = 1.0 + eps / (2 * pi) * xb * e;
    const double Tm = 1.0 - (gam - 1) * eps * eps / (8 * gam * pi * pi) * e * e;
    const double rho = pow(Tm, 1.0 / (gam - 1));
    const double p = rho * Tm;
    Q[0] = rho;
    Q[1] = rho * u;
    Q[2] = rho * v;
    Q[3] = 0.0;
    Q[4] = p / (gam - 1) + 0.5 * rho * (u * u + v * v);
  } else if (kind == 3) {
    double r2 = 0.0;
    int d;
    for (d = 0; d < dim; d++) r2 += (x[d] - param[3 + d]) * (x[d] - param[3 + d]);
    Q[4] += dt * param[0] * exp(-r2 / (param[1] * param[1])) * (1.0 + sin(2 * pi * param[2] * t));
  }
}

