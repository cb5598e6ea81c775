// Per-orbital FP64 kernels: Thiele coefficients, Pade evaluation, linearized
// and Newton quasiparticle roots.  One thread per orbital; latency-bound by
// nature (O(nfit^2) complex work per orbital).
#include "pade.cuh"
#include "qx_internal.cuh"

namespace qx {

struct Orbital {
  const cplx* zn;
  const cplx* a;
  int nfit;
  double eps, sx, vxc, ef;
  __device__ double sig(double w) const { return pade_eval(w, zn, a, nfit).re; }
  // 5-point stencil (newton_solver.rs:282-303, use_richardson = true).
  __device__ double deriv(double w) const {
    const double de = 1e-6;
    const double p1 = sig(w + de), m1 = sig(w - de), p2 = sig(w + 2.0 * de), m2 = sig(w - 2.0 * de);
    return (8.0 * (p1 - m1) - (p2 - m2)) / (12.0 * de);
  }
  __device__ double residual(double e) const { return e - eps - sx - sig(e - ef) + vxc; }
};

__global__ void k_pade_qp(QPParams p) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= p.norbs) return;
  const int n = p.orbs[t];
  const double s = (n < p.nocc) ? -1.0 : 1.0;
  const int nfit = p.nfit;
  cplx zn[MAX_FIT], a[MAX_FIT];
  // Fit points and values; col holds the running Thiele column.
  for (int j = 0; j < nfit; ++j) {
    const int k = p.fit_idx[j];
    zn[j] = cmk(0.0, s * p.iw[k]);
    a[j] = cmk(p.sigma[((size_t)t * p.nws + k) * 2], p.sigma[((size_t)t * p.nws + k) * 2 + 1]);
  }
  thiele_fit(a, zn, nfit);
  for (int j = 0; j < nfit; ++j) {
    p.coeff[((size_t)j * p.norbs + t) * 2] = a[j].re;
    p.coeff[((size_t)j * p.norbs + t) * 2 + 1] = a[j].im;
  }
  Orbital o{zn, a, nfit, p.mo_energy[n], p.sigma_x[n], p.vxc[n], p.ef};
  const double de = 1e-6;
  double qp, z;
  cplx sc;
  if (!p.solved) {
    // Linearized QP (qp/evgw.rs:784-821).
    const double we = p.eval_energy[n] - p.ef;
    sc = pade_eval(we, zn, a, nfit);
    const double s1 = pade_eval(we + de, zn, a, nfit).re;
    z = 1.0 / (1.0 - (s1 - sc.re) / de);
    z = fmin(fmax(z, p.z_min), p.z_max);
    qp = o.eps + z * (o.sx + sc.re - o.vxc);
  } else {
    // Newton (qp/evgw.rs:713-783, newton_solver.rs:174-392).
    double guess;
    if (p.first_iteration) {
      const double we = o.eps - p.ef;
      const double s0 = o.sig(we), s1 = o.sig(we + de);
      double zz = fmin(fmax(1.0 / (1.0 - (s1 - s0) / de), p.z_min), p.z_max);
      guess = o.eps + zz * (o.sx + s0 - o.vxc);
    } else {
      guess = p.eval_energy[n];
    }
    bool ok = false;
    double energy = guess, damping = 1.0, prev = 1e300;
    for (int it = 0; it < p.newton_max_iter; ++it) {
      const double omega = energy - p.ef;
      const cplx sv = pade_eval(omega, zn, a, nfit);
      const double res = energy - o.eps - o.sx - sv.re + o.vxc;
      const double ares = fabs(res);
      if (ares < p.newton_tol) {
        qp = energy;
        sc = sv;
        z = fmin(fmax(1.0 / (1.0 - o.deriv(energy - p.ef)), p.z_min), p.z_max);
        ok = true;
        break;
      }
      const double fp = 1.0 - o.deriv(omega);
      double step = (fabs(fp) < 1e-10) ? -copysign(1.0, res) * fmin(1.0, ares) : -res / fp;
      step = fmin(fmax(step, -1.0), 1.0);
      if (ares > prev) damping = fmax(damping * 0.5, 0.1);
      else if (ares < 0.5 * prev && damping < 1.0) damping = fmin(damping * 1.2, 1.0);
      energy += damping * step;
      prev = ares;
    }
    if (!ok) {
      // Bisection fallback (newton_solver.rs:317-392).
      double lo = guess - 2.0, hi = guess + 2.0;
      if (o.residual(lo) * o.residual(hi) > 0.0) {
        for (int e = 1; e < 5; ++e) {
          const double wdt = 2.0 * (double)(1 << e);
          lo = guess - wdt;
          hi = guess + wdt;
          if (o.residual(lo) * o.residual(hi) <= 0.0) break;
        }
      }
      for (int it = 0; it < 30; ++it) {
        const double mid = 0.5 * (lo + hi);
        const double fm = o.residual(mid);
        if (fabs(fm) < p.newton_tol || 0.5 * (hi - lo) < p.newton_tol) {
          qp = mid;
          sc = pade_eval(mid - p.ef, zn, a, nfit);
          z = fmin(fmax(1.0 / (1.0 - o.deriv(mid - p.ef)), p.z_min), p.z_max);
          ok = true;
          break;
        }
        if (fm * o.residual(lo) < 0.0) hi = mid;
        else lo = mid;
      }
    }
    if (!ok) {
      // Linearized fallback at the guess (qp/evgw.rs:766-781).
      const double we = guess - p.ef;
      sc = pade_eval(we, zn, a, nfit);
      const double s1 = pade_eval(we + de, zn, a, nfit).re;
      z = fmin(fmax(1.0 / (1.0 - (s1 - sc.re) / de), p.z_min), p.z_max);
      qp = o.eps + z * (o.sx + sc.re - o.vxc);
    }
  }
  p.qp_out[t] = qp;
  p.z_out[t] = z;
  p.sc_out[2 * t] = sc.re;
  p.sc_out[2 * t + 1] = sc.im;
}

void launch_pade_qp(qx_ctx* ctx, const QPParams& p) {
  QX_REQUIRE(p.nfit <= MAX_FIT, QX_ERR_INVALID_INPUT, "nfit %d exceeds %d", p.nfit, MAX_FIT);
  k_pade_qp<<<ceil_div(p.norbs, 64), 64, 0, ctx->stream>>>(p);
  check_launch(ctx);
}

}  // namespace qx
