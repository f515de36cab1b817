/*
 * orc_p2p.c -- oracle restatement of the reference's direct kernels (test
 * infrastructure only).  These are the scalar (non-SIMD) branches of
 *   Laplace            laplace.h:261-275 (potential), 335-358 (gradient)
 *   modified Helmholtz modified_helmholtz.h:70-83, 149-171
 *   Helmholtz          helmholtz.h:257-270, 361-382
 * in FP64, skipping r == 0 exactly as the reference does.  OpenMP over targets.
 */
#include <complex.h>
#include <math.h>
#include <stddef.h>

#include "orc.h"

#define ORC_PI 3.14159265358979323846

void orc_gradient_p2p(int kernel, double k_re, double k_im, int ns, const double* sxyz, const double* sq, int nt,
                      const double* txyz, double* out) {
  const double c4 = 4 * ORC_PI;
#pragma omp parallel for schedule(dynamic, 64)
  for (int t = 0; t < nt; t++) {
    if (kernel == 2) {
      const double complex wk = k_re + I * k_im;
      double complex pot = 0, g[3] = {0, 0, 0};
      for (int s = 0; s < ns; s++) {
        double dx[3];
        for (int d = 0; d < 3; d++) dx[d] = txyz[3 * t + d] - sxyz[3 * s + d];
        double r2 = dx[0] * dx[0] + dx[1] * dx[1] + dx[2] * dx[2];
        if (r2 != 0) {
          double r = sqrt(r2);
          double complex q = sq[2 * s] + I * sq[2 * s + 1];
          double complex pij = cexp(I * r * wk) * q / r;
          double complex cg = (I * wk / r - 1 / r2) * pij;
          pot += pij;
          for (int d = 0; d < 3; d++) g[d] += cg * dx[d];
        }
      }
      double complex v[4] = {pot / c4, g[0] / c4, g[1] / c4, g[2] / c4};
      for (int c = 0; c < 4; c++) {
        out[2 * (4 * (size_t)t + c)] += creal(v[c]);
        out[2 * (4 * (size_t)t + c) + 1] += cimag(v[c]);
      }
    } else if (kernel == 1) {
      double pot = 0, g[3] = {0, 0, 0};
      for (int s = 0; s < ns; s++) {
        double dx[3];
        for (int d = 0; d < 3; d++) dx[d] = txyz[3 * t + d] - sxyz[3 * s + d];
        double r2 = dx[0] * dx[0] + dx[1] * dx[1] + dx[2] * dx[2];
        if (r2 != 0) {
          double r = sqrt(r2);
          double kern = exp(-k_re * r) / r * sq[s];
          pot += kern;
          double dpdr = -kern * (k_re * r + 1) / r;
          for (int d = 0; d < 3; d++) g[d] += dpdr / r * dx[d];
        }
      }
      out[4 * (size_t)t] += pot / c4;
      for (int d = 0; d < 3; d++) out[4 * (size_t)t + 1 + d] += g[d] / c4;
    } else {
      double pot = 0, g[3] = {0, 0, 0};
      for (int s = 0; s < ns; s++) {
        double dx[3];
        for (int d = 0; d < 3; d++) dx[d] = txyz[3 * t + d] - sxyz[3 * s + d];
        double r2 = dx[0] * dx[0] + dx[1] * dx[1] + dx[2] * dx[2];
        if (r2 != 0) {
          double invr2 = 1.0 / r2;
          double invr = sq[s] * sqrt(invr2);
          pot += invr;
          for (int d = 0; d < 3; d++) g[d] += dx[d] * (invr2 * invr);
        }
      }
      out[4 * (size_t)t] += pot / c4;
      for (int d = 0; d < 3; d++) out[4 * (size_t)t + 1 + d] -= g[d] / c4;
    }
  }
}

void orc_potential_p2p(int kernel, double k_re, double k_im, int ns, const double* sxyz, const double* sq, int nt,
                       const double* txyz, double* out) {
  const double c4 = 4 * ORC_PI;
#pragma omp parallel for schedule(dynamic, 64)
  for (int t = 0; t < nt; t++) {
    if (kernel == 2) {
      const double complex wk = k_re + I * k_im;
      double complex pot = 0;
      for (int s = 0; s < ns; s++) {
        double dx[3];
        for (int d = 0; d < 3; d++) dx[d] = txyz[3 * t + d] - sxyz[3 * s + d];
        double r2 = dx[0] * dx[0] + dx[1] * dx[1] + dx[2] * dx[2];
        if (r2 != 0) {
          double r = sqrt(r2);
          pot += cexp(I * r * wk) * (sq[2 * s] + I * sq[2 * s + 1]) / r;
        }
      }
      out[2 * (size_t)t] += creal(pot / c4);
      out[2 * (size_t)t + 1] += cimag(pot / c4);
    } else {
      double pot = 0;
      for (int s = 0; s < ns; s++) {
        double dx[3];
        for (int d = 0; d < 3; d++) dx[d] = txyz[3 * t + d] - sxyz[3 * s + d];
        double r2 = dx[0] * dx[0] + dx[1] * dx[1] + dx[2] * dx[2];
        if (r2 != 0) {
          double r = sqrt(r2);
          pot += kernel == 1 ? exp(-k_re * r) * sq[s] / r : sq[s] * (1 / r);
        }
      }
      out[t] += pot / c4;
    }
  }
}
