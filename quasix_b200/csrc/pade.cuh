// Complex FP64 helpers and the Thiele/Pade continued fraction, shared by the
// per-orbital QP kernels (k_qp.cu) and the Pade entry points (qx_pade.cu).
#pragma once
#include <cuda_runtime.h>

namespace qx {

struct cplx {
  double re, im;
};
__device__ inline cplx cmk(double r, double i) { return cplx{r, i}; }
__device__ inline cplx cadd(cplx a, cplx b) { return cplx{a.re + b.re, a.im + b.im}; }
__device__ inline cplx csub(cplx a, cplx b) { return cplx{a.re - b.re, a.im - b.im}; }
__device__ inline cplx cmul(cplx a, cplx b) {
  return cplx{a.re * b.re - a.im * b.im, a.re * b.im + a.im * b.re};
}
__device__ inline cplx cdiv(cplx a, cplx b) {
  const double n = b.re * b.re + b.im * b.im;
  return cplx{(a.re * b.re + a.im * b.im) / n, (a.im * b.re - a.re * b.im) / n};
}
__device__ inline double cabs_(cplx a) { return hypot(a.re, a.im); }

constexpr int MAX_FIT = 64;

// Pade continued fraction at real omega (correlation_ac.rs:530-566); zn and
// a are read with stride `step` (1: contiguous per orbital).
__device__ inline cplx pade_eval(double omega, const cplx* zn, const cplx* a, int nfit, int step = 1) {
  if (nfit == 0) return cmk(0, 0);
  if (nfit == 1) return a[0];
  const cplx z = cmk(omega, 0.0);
  cplx x = cmul(a[(nfit - 1) * step], csub(z, zn[(nfit - 2) * step]));
  for (int i = nfit - 2; i >= 1; --i) {
    cplx den = cadd(cmk(1.0, 0.0), x);
    if (cabs_(den) < 1e-14) x = cmk(1e10, 0.0);
    else x = cdiv(cmul(a[i * step], csub(z, zn[(i - 1) * step])), den);
  }
  cplx den = cadd(cmk(1.0, 0.0), x);
  if (cabs_(den) < 1e-14) return a[0];
  return cdiv(a[0], den);
}

// Reciprocal differences in place (correlation_ac.rs:470-509): a[j] holds the
// sampled values f(zn[j]) on entry and the Thiele coefficients g[j][j] on
// exit (after column j, a[i > j] = g[i][j]).  Guard: a denominator below 1e-14
// gives 1e10, as the reference does.
__device__ inline void thiele_fit(cplx* a, const cplx* zn, int nfit) {
  for (int j = 1; j < nfit; ++j) {
    const cplx gd = a[j - 1];
    for (int i = j; i < nfit; ++i) {
      const cplx den = cmul(csub(zn[i], zn[j - 1]), a[i]);
      if (cabs_(den) < 1e-14) a[i] = cmk(1e10, 0.0);
      else a[i] = cdiv(csub(gd, a[i]), den);
    }
  }
}

}  // namespace qx
