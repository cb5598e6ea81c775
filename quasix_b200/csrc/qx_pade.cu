// Analytic continuation and spectral functions on the device: the Thiele fit
// of Sigma_c(iw) and the Pade evaluation behind the exported entry points, and
// the real-axis spectral functions built from QP energies or from the Pade
// continuation of Sigma_c.
//
// All of these are latency- or transcendental-bound (O(nfit^2) complex work
// per orbital, one exp or division per (state, omega) pair); the kernels keep
// each orbital's coefficients, or a tile of states, in shared memory and run
// one thread per output element.
#include <algorithm>
#include <cfloat>

#include "pade.cuh"
#include "qx_internal.cuh"

namespace qx {

std::vector<int> pade_indices(int nws, int npade);

namespace {

// coeff[j][t] and ofit[t][j] (complex) from sigma[t][k], omega[t][k] at the
// fit indices idx[j] (thiele + ac_pade_thiele_diag, correlation_ac.rs:470-509,
// 587-654).  One thread per orbital.
__global__ void k_thiele_fit(const double* __restrict__ sigma, const double* __restrict__ omega, int nws,
                             const int* __restrict__ idx, int nfit, int norbs, double* __restrict__ coeff,
                             double* __restrict__ ofit) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= norbs) return;
  cplx zn[MAX_FIT], a[MAX_FIT];
  for (int j = 0; j < nfit; ++j) {
    const size_t q = ((size_t)t * nws + idx[j]) * 2;
    zn[j] = cmk(omega[q], omega[q + 1]);
    a[j] = cmk(sigma[q], sigma[q + 1]);
    ofit[((size_t)t * nfit + j) * 2] = zn[j].re;
    ofit[((size_t)t * nfit + j) * 2 + 1] = zn[j].im;
  }
  thiele_fit(a, zn, nfit);
  for (int j = 0; j < nfit; ++j) {
    coeff[((size_t)j * norbs + t) * 2] = a[j].re;
    coeff[((size_t)j * norbs + t) * 2 + 1] = a[j].im;
  }
}

// The fit of orbital t (zn = ofit[t][:], a = coeff[:][t]) into shared memory.
__device__ __forceinline__ void stage_fit(const double* __restrict__ coeff, const double* __restrict__ ofit,
                                          int nfit, int norbs, int t, cplx* zs, cplx* as) {
  for (int j = threadIdx.x; j < nfit; j += blockDim.x) {
    zs[j] = cmk(ofit[((size_t)t * nfit + j) * 2], ofit[((size_t)t * nfit + j) * 2 + 1]);
    as[j] = cmk(coeff[((size_t)j * norbs + t) * 2], coeff[((size_t)j * norbs + t) * 2 + 1]);
  }
  __syncthreads();
}

// out[t][q] = pade_thiele(omega[q]) of orbital t (correlation_ac.rs:530-566).
// grid (ceil(nomega / 256), norbs).
__global__ void k_pade_eval(const double* __restrict__ coeff, const double* __restrict__ ofit, int nfit, int norbs,
                            const double* __restrict__ omega, int nomega, double* __restrict__ out) {
  __shared__ cplx zs[MAX_FIT], as[MAX_FIT];
  const int t = blockIdx.y;
  stage_fit(coeff, ofit, nfit, norbs, t, zs, as);
  const int q = blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= nomega) return;
  const cplx r = pade_eval(omega[q], zs, as, nfit);
  out[((size_t)t * nomega + q) * 2] = r.re;
  out[((size_t)t * nomega + q) * 2 + 1] = r.im;
}

// A_t(w) = (1/pi) G / ((w - e_t - Sx_t + Vxc_t - Re S(w - ef))^2 + G^2),
// G = |Im S(w - ef)| + eta, with S the Pade continuation of Sigma_c of
// orbital t: the quasiparticle peak and its satellites with the lifetime
// broadening of the continued self-energy (time-ordered: |Im Sigma| adds to
// eta on both sides of the Fermi level).  grid (ceil(nomega / 256), norbs).
__global__ void k_spectral_pade(const double* __restrict__ coeff, const double* __restrict__ ofit, int nfit,
                                int norbs, const double* __restrict__ e_ref, const double* __restrict__ sx,
                                const double* __restrict__ vxc, double ef, const double* __restrict__ omega,
                                int nomega, double eta, double* __restrict__ A) {
  __shared__ cplx zs[MAX_FIT], as[MAX_FIT];
  const int t = blockIdx.y;
  stage_fit(coeff, ofit, nfit, norbs, t, zs, as);
  const int q = blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= nomega) return;
  const double w = omega[q];
  const cplx s = pade_eval(w - ef, zs, as, nfit);
  const double re = w - e_ref[t] - sx[t] + vxc[t] - s.re;
  const double g = fabs(s.im) + eta;
  A[(size_t)t * nomega + q] = g / (M_PI * (re * re + g * g));
}

// Broadening profile of SpectralAnalyzer::compute_spectral_function
// (quasix_core/src/analysis/spectral.rs:283-325, 327-545): 0 Gaussian,
// 1 Lorentzian, 2 Voigt mixture (1 - alpha) G + alpha L.
struct Broadening {
  int mode;
  double sigma, gamma, alpha;
};
__device__ __forceinline__ double profile(const Broadening& b, double d) {
  const double gauss = exp(-d * d / (2.0 * b.sigma * b.sigma)) / (b.sigma * sqrt(2.0 * M_PI));
  const double lor = (b.gamma / M_PI) / (d * d + b.gamma * b.gamma);
  if (b.mode == 0) return gauss;
  if (b.mode == 1) return lor;
  return (1.0 - b.alpha) * gauss + b.alpha * lor;
}

// weights[q] = sum_i Z_i profile(omega[q] - E_i) over the states of `kind`
// (0: all, energies E as given; 1: PES, states E <= ef at binding energy
// ef - E; 2: IPES, states E > ef at ef-relative energy E - ef;
// generate_pes_spectrum / generate_ipes_spectrum, spectral.rs:557-656).
// States are staged through shared memory 256 at a time; one thread per omega.
__global__ void __launch_bounds__(256) k_spectral_qp(const double* __restrict__ e, const double* __restrict__ z,
                                                     int n, double ef, int kind, Broadening b,
                                                     const double* __restrict__ omega, int nomega,
                                                     double* __restrict__ weights) {
  __shared__ double se[256], sz[256];
  const int q = blockIdx.x * blockDim.x + threadIdx.x;
  const double w = q < nomega ? omega[q] : 0.0;
  double sum = 0.0;
  for (int i0 = 0; i0 < n; i0 += 256) {
    __syncthreads();
    const int i = i0 + threadIdx.x;
    double ei = 0.0, zi = 0.0;
    if (i < n) {
      ei = e[i];
      zi = z[i];
      if (kind == 1) {
        zi = ei <= ef ? zi : 0.0;
        ei = ef - ei;
      } else if (kind == 2) {
        zi = ei > ef ? zi : 0.0;
        ei = ei - ef;
      }
    }
    se[threadIdx.x] = ei;
    sz[threadIdx.x] = zi;
    __syncthreads();
    const int m = min(256, n - i0);
    for (int k = 0; k < m; ++k)
      if (sz[k] != 0.0) sum += sz[k] * profile(b, w - se[k]);
  }
  if (q < nomega) weights[q] = sum;
}

// A[i][q] = Z_i eta / ((omega[q] - E_i)^2 + eta^2) / pi
// (EvGWResult.spectral_function, quasix/quasix/evgw.py:124-134).
__global__ void k_spectral_states(const double* __restrict__ e, const double* __restrict__ z, int n,
                                  const double* __restrict__ omega, int nomega, double eta, double* __restrict__ A) {
  const size_t total = (size_t)n * nomega;
  for (size_t k = (size_t)blockIdx.x * blockDim.x + threadIdx.x; k < total; k += (size_t)gridDim.x * blockDim.x) {
    const int i = (int)(k / nomega), q = (int)(k % nomega);
    const double d = omega[q] - e[i];
    A[k] = z[i] * eta / (d * d + eta * eta) / M_PI;
  }
}

// NewtonQPSolver::solve with the Pade-continued Sigma_c as its evaluator
// (quasix_core/src/qp/newton_solver.rs:174-280 Newton with adaptive damping,
// :282-315 derivative and Z, :317-392 bisection fallback, :394-401 residual),
// one thread per orbital.  method: 0 Newton, 1 bisection, -1 neither
// converged (the reference's ConvergenceError).
struct NewtonArgs {
  qx_newton_config cfg;
  int norbs, nfit;
  const cplx* coeff;  // [nfit][norbs]
  const cplx* zfit;   // [norbs][nfit]
  const double *eps, *sx, *vxc, *guess;
  double ef;
  double *qp, *res, *z;
  cplx* sc;
  int *iters, *method;
};

__global__ void k_newton_qp(NewtonArgs p) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= p.norbs) return;
  const int nfit = p.nfit;
  cplx zn[MAX_FIT], a[MAX_FIT];
  for (int j = 0; j < nfit; ++j) {
    zn[j] = p.zfit[(size_t)t * nfit + j];
    a[j] = p.coeff[(size_t)j * p.norbs + t];
  }
  const qx_newton_config& c = p.cfg;
  const double eps = p.eps[t], sx = p.sx[t], vxc = p.vxc[t], ef = p.ef, guess = p.guess[t];
  auto sig = [&](double w) { return pade_eval(w, zn, a, nfit); };
  auto deriv = [&](double w) {
    const double de = c.derivative_delta;
    if (c.use_richardson) {
      const double p1 = sig(w + de).re, m1 = sig(w - de).re, p2 = sig(w + 2.0 * de).re, m2 = sig(w - 2.0 * de).re;
      return (8.0 * (p1 - m1) - (p2 - m2)) / (12.0 * de);
    }
    return (sig(w + de).re - sig(w - de).re) / (2.0 * de);
  };
  auto zfac = [&](double e) { return fmin(fmax(1.0 / (1.0 - deriv(e - ef)), c.z_min), c.z_max); };
  auto resid = [&](double e) { return e - eps - sx - sig(e - ef).re + vxc; };
  double energy = guess, damping = c.initial_damping, prev = DBL_MAX, ares = 0.0;
  for (int it = 0; it < c.max_iterations; ++it) {
    const double omega = energy - ef;
    const cplx s = sig(omega);
    const double r = energy - eps - sx - s.re + vxc;
    ares = fabs(r);
    if (ares < c.energy_tolerance) {
      p.qp[t] = energy;
      p.res[t] = ares;
      p.iters[t] = it + 1;
      p.method[t] = 0;
      p.sc[t] = s;
      p.z[t] = zfac(energy);
      return;
    }
    const double fp = 1.0 - deriv(omega);
    const double step = fabs(fp) < 1e-10 ? -copysign(1.0, r) * fmin(c.max_step, ares) : -r / fp;
    const double clipped = fmin(fmax(step, -c.max_step), c.max_step);
    if (ares > prev) damping = fmax(damping * 0.5, c.min_damping);
    else if (ares < 0.5 * prev && damping < c.max_damping) damping = fmin(damping * 1.2, c.max_damping);
    energy += damping * clipped;
    prev = ares;
  }
  if (c.use_bisection_fallback) {
    const double width = 2.0;
    double lo = guess - width, hi = guess + width;
    if (resid(lo) * resid(hi) > 0.0) {
      for (int e = 1; e < 5; ++e) {
        const double wd = width * (double)(1 << e);
        lo = guess - wd;
        hi = guess + wd;
        if (resid(lo) * resid(hi) <= 0.0) break;
      }
    }
    for (int it = 0; it < c.max_bisection_iterations; ++it) {
      const double mid = 0.5 * (lo + hi);
      const double fm = resid(mid);
      if (fabs(fm) < c.energy_tolerance || 0.5 * (hi - lo) < c.energy_tolerance) {
        p.qp[t] = mid;
        p.res[t] = fabs(fm);
        p.iters[t] = it + 1;
        p.method[t] = 1;
        p.sc[t] = sig(mid - ef);
        p.z[t] = zfac(mid);
        return;
      }
      if (fm * resid(lo) < 0.0) hi = mid;
      else lo = mid;
    }
  }
  // Not converged: the last Newton iterate, its residual and Z.
  p.qp[t] = energy;
  p.res[t] = prev;
  p.iters[t] = c.max_iterations;
  p.method[t] = -1;
  p.sc[t] = sig(energy - ef);
  p.z[t] = zfac(energy);
}

// Device copies of small caller arrays, carved from one workspace slot.
struct Carve {
  char* base;
  size_t off = 0;
  template <class T>
  T* take(size_t n) {
    T* p = reinterpret_cast<T*>(base + off);
    off += (n * sizeof(T) + 255) & ~size_t(255);
    return p;
  }
};
inline size_t carve_bytes(std::initializer_list<size_t> sizes) {
  size_t s = 0;
  for (size_t b : sizes) s += (b + 255) & ~size_t(255);
  return s;
}

}  // namespace

}  // namespace qx

using namespace qx;

template <class F>
static qx_status run(qx_ctx* ctx, F&& f) {
  if (!ctx) return QX_ERR_INVALID_INPUT;
  try {
    reset_pending(ctx);
    ctx->launches = 0;
    QX_CUDA(cudaSetDevice(ctx->device));
    f();
    ctx->err.clear();
    return QX_OK;
  } catch (const Error& e) {
    ctx->err = e.what();
    return e.status;
  } catch (const std::exception& e) {
    ctx->err = e.what();
    return QX_ERR_INVALID_INPUT;
  }
}

extern "C" {

qx_status qx_ac_pade_thiele_diag(qx_ctx* ctx, int norbs, int nws, const double* sigma, const double* omega, int npade,
                                 double* coeff, double* omega_fit, int nfit_max, int* nfit) {
  return run(ctx, [&] {
    QX_REQUIRE(norbs > 0 && nws > 0 && sigma && omega && nfit, QX_ERR_INVALID_INPUT, "invalid arguments");
    const std::vector<int> idx = pade_indices(nws, npade);
    const int nf = (int)idx.size();
    *nfit = nf;
    if (nf == 0) return;
    QX_REQUIRE(nf <= MAX_FIT, QX_ERR_INVALID_INPUT, "nfit %d exceeds %d", nf, MAX_FIT);
    QX_REQUIRE(nfit_max >= nf && coeff && omega_fit, QX_ERR_INVALID_INPUT, "nfit_max %d < %d", nfit_max, nf);
    const size_t in_b = (size_t)norbs * nws * 2 * sizeof(double), out_b = (size_t)norbs * nf * 2 * sizeof(double);
    const double* d_s = (const double*)device_view(ctx, WS_LPQ, sigma, in_b);
    const double* d_o = (const double*)device_view(ctx, WS_HOSTIN, omega, in_b);
    DevBuf& wb = ctx->ws[WS_QPOUT];
    wb.reserve(carve_bytes({out_b, out_b, nf * sizeof(int)}));
    Carve cv{wb.as<char>()};
    double* d_c = cv.take<double>((size_t)norbs * nf * 2);
    double* d_f = cv.take<double>((size_t)norbs * nf * 2);
    int* d_idx = cv.take<int>(nf);
    QX_CUDA(cudaMemcpyAsync(d_idx, idx.data(), nf * sizeof(int), cudaMemcpyHostToDevice, ctx->stream));
    k_thiele_fit<<<ceil_div(norbs, 64), 64, 0, ctx->stream>>>(d_s, d_o, nws, d_idx, nf, norbs, d_c, d_f);
    check_launch(ctx);
    QX_CUDA(cudaMemcpyAsync(coeff, d_c, out_b, cudaMemcpyDefault, ctx->stream));
    QX_CUDA(cudaMemcpyAsync(omega_fit, d_f, out_b, cudaMemcpyDefault, ctx->stream));
    sync_and_check(ctx);
  });
}

qx_status qx_pade_thiele(qx_ctx* ctx, int nfit, const double* zn, const double* coeff, int nomega,
                         const double* omega, double* out) {
  return run(ctx, [&] {
    QX_REQUIRE(nfit >= 0 && nomega >= 0 && (nfit == 0 || (zn && coeff)) && (nomega == 0 || (omega && out)),
               QX_ERR_INVALID_INPUT, "invalid arguments to pade_thiele");
    QX_REQUIRE(nfit <= MAX_FIT, QX_ERR_INVALID_INPUT, "nfit %d exceeds %d", nfit, MAX_FIT);
    if (nomega == 0) return;
    const size_t fb = (size_t)std::max(nfit, 1) * 2 * sizeof(double);
    DevBuf& wb = ctx->ws[WS_QPOUT];
    wb.reserve(carve_bytes({fb, fb, nomega * sizeof(double), (size_t)nomega * 2 * sizeof(double)}));
    Carve cv{wb.as<char>()};
    double* d_z = cv.take<double>(std::max(nfit, 1) * 2);
    double* d_c = cv.take<double>(std::max(nfit, 1) * 2);
    double* d_w = cv.take<double>(nomega);
    double* d_out = cv.take<double>((size_t)nomega * 2);
    if (nfit > 0) {
      QX_CUDA(cudaMemcpyAsync(d_z, zn, (size_t)nfit * 2 * sizeof(double), cudaMemcpyDefault, ctx->stream));
      QX_CUDA(cudaMemcpyAsync(d_c, coeff, (size_t)nfit * 2 * sizeof(double), cudaMemcpyDefault, ctx->stream));
    }
    QX_CUDA(cudaMemcpyAsync(d_w, omega, nomega * sizeof(double), cudaMemcpyDefault, ctx->stream));
    k_pade_eval<<<dim3(ceil_div(nomega, 256), 1), 256, 0, ctx->stream>>>(d_c, d_z, nfit, 1, d_w, nomega, d_out);
    check_launch(ctx);
    QX_CUDA(cudaMemcpyAsync(out, d_out, (size_t)nomega * 2 * sizeof(double), cudaMemcpyDefault, ctx->stream));
    sync_and_check(ctx);
  });
}

qx_status qx_spectral_function(qx_ctx* ctx, const double* qp_energies, const double* z_factors, int n_states,
                               double fermi_energy, int kind, const double* omega, int n_omega,
                               double gaussian_width, double lorentzian_width, double voigt_mixing,
                               double* weights, double* total_weight) {
  return run(ctx, [&] {
    QX_REQUIRE(n_states >= 0 && (n_states == 0 || (qp_energies && z_factors)) && weights, QX_ERR_INVALID_INPUT,
               "invalid arguments to spectral_function");
    QX_REQUIRE(n_omega > 0 && omega, QX_ERR_INVALID_INPUT, "Invalid omega grid: Empty omega grid");
    QX_REQUIRE(kind >= 0 && kind <= 2, QX_ERR_INVALID_INPUT, "kind %d: 0 all states, 1 PES, 2 IPES", kind);
    QX_REQUIRE(gaussian_width > 0.0, QX_ERR_INVALID_INPUT, "Invalid broadening parameter gaussian_width: %g",
               gaussian_width);
    QX_REQUIRE(lorentzian_width > 0.0, QX_ERR_INVALID_INPUT, "Invalid broadening parameter lorentzian_width: %g",
               lorentzian_width);
    QX_REQUIRE(voigt_mixing >= 0.0 && voigt_mixing <= 1.0, QX_ERR_INVALID_INPUT,
               "Invalid broadening parameter voigt_mixing: %g", voigt_mixing);
    std::vector<double> hz(n_states), hw(std::min(n_omega, 2));
    if (n_states) QX_CUDA(cudaMemcpy(hz.data(), z_factors, n_states * sizeof(double), cudaMemcpyDefault));
    for (int i = 0; i < n_states; ++i)
      QX_REQUIRE(hz[i] >= 0.0 && hz[i] <= 1.0, QX_ERR_INVALID_INPUT,
                 "Invalid Z-factor %g at index %d: must be in range (0, 1)", hz[i], i);
    QX_CUDA(cudaMemcpy(hw.data(), omega, hw.size() * sizeof(double), cudaMemcpyDefault));
    DevBuf& wb = ctx->ws[WS_QPOUT];
    const size_t sb = (size_t)std::max(n_states, 1) * sizeof(double), ob = (size_t)n_omega * sizeof(double);
    wb.reserve(carve_bytes({sb, sb, ob, ob}));
    Carve cv{wb.as<char>()};
    double* d_e = cv.take<double>(std::max(n_states, 1));
    double* d_z = cv.take<double>(std::max(n_states, 1));
    double* d_w = cv.take<double>(n_omega);
    double* d_out = cv.take<double>(n_omega);
    if (n_states) {
      QX_CUDA(cudaMemcpyAsync(d_e, qp_energies, sb, cudaMemcpyDefault, ctx->stream));
      QX_CUDA(cudaMemcpyAsync(d_z, hz.data(), sb, cudaMemcpyHostToDevice, ctx->stream));
    }
    QX_CUDA(cudaMemcpyAsync(d_w, omega, ob, cudaMemcpyDefault, ctx->stream));
    // Profile choice of compute_spectral_function (spectral.rs:291-302).
    Broadening b{voigt_mixing < 0.01 ? 0 : (voigt_mixing > 0.99 ? 1 : 2), gaussian_width, lorentzian_width,
                 voigt_mixing};
    k_spectral_qp<<<ceil_div(n_omega, 256), 256, 0, ctx->stream>>>(d_e, d_z, n_states, fermi_energy, kind, b, d_w,
                                                                    n_omega, d_out);
    check_launch(ctx);
    std::vector<double> hout(n_omega);
    QX_CUDA(cudaMemcpyAsync(hout.data(), d_out, ob, cudaMemcpyDeviceToHost, ctx->stream));
    sync_and_check(ctx);
    QX_CUDA(cudaMemcpy(weights, hout.data(), ob, cudaMemcpyDefault));
    if (total_weight) {
      // Normalisation check of the reference (spectral.rs:304-310): sum * dw.
      double s = 0.0;
      for (double v : hout) s += v;
      *total_weight = s * (n_omega > 1 ? hw[1] - hw[0] : 1.0);
    }
  });
}

qx_status qx_spectral_function_states(qx_ctx* ctx, const double* qp_energies, const double* z_factors, int n_states,
                                      const double* omega, int n_omega, double eta, double* A) {
  return run(ctx, [&] {
    QX_REQUIRE(n_states > 0 && n_omega > 0 && qp_energies && z_factors && omega && A, QX_ERR_INVALID_INPUT,
               "invalid arguments to spectral_function_states");
    const size_t sb = (size_t)n_states * sizeof(double), ob = (size_t)n_omega * sizeof(double);
    const size_t ab = (size_t)n_states * n_omega * sizeof(double);
    DevBuf& wb = ctx->ws[WS_QPOUT];
    wb.reserve(carve_bytes({sb, sb, ob}));
    Carve cv{wb.as<char>()};
    double* d_e = cv.take<double>(n_states);
    double* d_z = cv.take<double>(n_states);
    double* d_w = cv.take<double>(n_omega);
    QX_CUDA(cudaMemcpyAsync(d_e, qp_energies, sb, cudaMemcpyDefault, ctx->stream));
    QX_CUDA(cudaMemcpyAsync(d_z, z_factors, sb, cudaMemcpyDefault, ctx->stream));
    QX_CUDA(cudaMemcpyAsync(d_w, omega, ob, cudaMemcpyDefault, ctx->stream));
    double* d_a = A;
    if (!is_device_ptr(A)) {
      ctx->ws[WS_HOSTIN].reserve(ab);
      d_a = ctx->ws[WS_HOSTIN].as<double>();
    }
    const int blocks = (int)std::min<size_t>((ab / sizeof(double) + 255) / 256, 8 * (size_t)ctx->sm_count);
    k_spectral_states<<<std::max(blocks, 1), 256, 0, ctx->stream>>>(d_e, d_z, n_states, d_w, n_omega, eta, d_a);
    check_launch(ctx);
    if (d_a != A) QX_CUDA(cudaMemcpyAsync(A, d_a, ab, cudaMemcpyDeviceToHost, ctx->stream));
    sync_and_check(ctx);
  });
}

qx_status qx_spectral_function_pade(qx_ctx* ctx, int norbs, int nfit, const double* coeff, const double* omega_fit,
                                    const double* e_ref, const double* sigma_x, const double* vxc, double ef,
                                    const double* omega, int n_omega, double eta, double* A) {
  return run(ctx, [&] {
    QX_REQUIRE(norbs > 0 && nfit >= 0 && n_omega > 0 && (nfit == 0 || (coeff && omega_fit)) && e_ref && sigma_x &&
                   omega && A && eta >= 0.0,
               QX_ERR_INVALID_INPUT, "invalid arguments to spectral_function_pade");
    QX_REQUIRE(nfit <= MAX_FIT, QX_ERR_INVALID_INPUT, "nfit %d exceeds %d", nfit, MAX_FIT);
    QX_REQUIRE(norbs <= 65535, QX_ERR_INVALID_INPUT, "norbs %d exceeds 65535", norbs);
    const size_t fb = (size_t)norbs * std::max(nfit, 1) * 2 * sizeof(double), nb = (size_t)norbs * sizeof(double);
    const size_t ob = (size_t)n_omega * sizeof(double), ab = (size_t)norbs * n_omega * sizeof(double);
    DevBuf& wb = ctx->ws[WS_QPOUT];
    wb.reserve(carve_bytes({fb, fb, nb, nb, nb, ob}));
    Carve cv{wb.as<char>()};
    double* d_c = cv.take<double>(fb / sizeof(double));
    double* d_f = cv.take<double>(fb / sizeof(double));
    double* d_e = cv.take<double>(norbs);
    double* d_sx = cv.take<double>(norbs);
    double* d_vx = cv.take<double>(norbs);
    double* d_w = cv.take<double>(n_omega);
    if (nfit > 0) {
      QX_CUDA(cudaMemcpyAsync(d_c, coeff, (size_t)norbs * nfit * 2 * sizeof(double), cudaMemcpyDefault, ctx->stream));
      QX_CUDA(cudaMemcpyAsync(d_f, omega_fit, (size_t)norbs * nfit * 2 * sizeof(double), cudaMemcpyDefault,
                              ctx->stream));
    }
    QX_CUDA(cudaMemcpyAsync(d_e, e_ref, nb, cudaMemcpyDefault, ctx->stream));
    QX_CUDA(cudaMemcpyAsync(d_sx, sigma_x, nb, cudaMemcpyDefault, ctx->stream));
    if (vxc) QX_CUDA(cudaMemcpyAsync(d_vx, vxc, nb, cudaMemcpyDefault, ctx->stream));
    else QX_CUDA(cudaMemsetAsync(d_vx, 0, nb, ctx->stream));
    QX_CUDA(cudaMemcpyAsync(d_w, omega, ob, cudaMemcpyDefault, ctx->stream));
    double* d_a = A;
    if (!is_device_ptr(A)) {
      ctx->ws[WS_HOSTIN].reserve(ab);
      d_a = ctx->ws[WS_HOSTIN].as<double>();
    }
    k_spectral_pade<<<dim3(ceil_div(n_omega, 256), norbs), 256, 0, ctx->stream>>>(d_c, d_f, nfit, norbs, d_e, d_sx,
                                                                                 d_vx, ef, d_w, n_omega, eta, d_a);
    check_launch(ctx);
    if (d_a != A) QX_CUDA(cudaMemcpyAsync(A, d_a, ab, cudaMemcpyDeviceToHost, ctx->stream));
    sync_and_check(ctx);
  });
}

qx_status qx_newton_qp_solve(qx_ctx* ctx, const qx_newton_config* cfg, int norbs, int nfit, const double* coeff,
                             const double* omega_fit, const double* epsilon_hf, const double* sigma_x,
                             const double* vxc, double fermi_level, const double* initial_guess, double* qp_energy,
                             double* residual, int* iterations, int* method, double* sigma_c, double* z_factor) {
  return run(ctx, [&] {
    QX_REQUIRE(cfg && norbs >= 0 && nfit >= 1, QX_ERR_INVALID_INPUT, "invalid arguments to newton_qp_solve");
    QX_REQUIRE(nfit <= MAX_FIT, QX_ERR_INVALID_INPUT, "nfit %d exceeds %d", nfit, MAX_FIT);
    QX_REQUIRE(cfg->max_iterations >= 0 && cfg->max_bisection_iterations >= 0 && cfg->derivative_delta > 0.0 &&
                   cfg->max_step > 0.0,
               QX_ERR_INVALID_INPUT, "invalid Newton configuration");
    if (norbs == 0) return;
    QX_REQUIRE(coeff && omega_fit && epsilon_hf && sigma_x && vxc && initial_guess && qp_energy && residual &&
                   iterations && method && sigma_c && z_factor,
               QX_ERR_INVALID_INPUT, "null argument to newton_qp_solve");
    const size_t cb = (size_t)nfit * norbs * 2 * sizeof(double), ob = (size_t)norbs * sizeof(double);
    DevBuf& wb = ctx->ws[WS_QPOUT];
    wb.reserve(carve_bytes({cb, cb, ob, ob, ob, ob, ob, ob, ob, 2 * ob, norbs * sizeof(int), norbs * sizeof(int)}));
    Carve cv{wb.as<char>()};
    NewtonArgs a;
    a.cfg = *cfg;
    a.norbs = norbs;
    a.nfit = nfit;
    auto in = [&](const double* src, size_t n) {
      double* d = cv.take<double>(n);
      QX_CUDA(cudaMemcpyAsync(d, src, n * sizeof(double), cudaMemcpyDefault, ctx->stream));
      return d;
    };
    a.coeff = reinterpret_cast<const cplx*>(in(coeff, (size_t)nfit * norbs * 2));
    a.zfit = reinterpret_cast<const cplx*>(in(omega_fit, (size_t)nfit * norbs * 2));
    a.eps = in(epsilon_hf, norbs);
    a.sx = in(sigma_x, norbs);
    a.vxc = in(vxc, norbs);
    a.guess = in(initial_guess, norbs);
    a.ef = fermi_level;
    a.qp = cv.take<double>(norbs);
    a.res = cv.take<double>(norbs);
    a.z = cv.take<double>(norbs);
    a.sc = cv.take<cplx>(norbs);
    a.iters = cv.take<int>(norbs);
    a.method = cv.take<int>(norbs);
    k_newton_qp<<<ceil_div(norbs, 64), 64, 0, ctx->stream>>>(a);
    check_launch(ctx);
    QX_CUDA(cudaMemcpyAsync(qp_energy, a.qp, ob, cudaMemcpyDefault, ctx->stream));
    QX_CUDA(cudaMemcpyAsync(residual, a.res, ob, cudaMemcpyDefault, ctx->stream));
    QX_CUDA(cudaMemcpyAsync(z_factor, a.z, ob, cudaMemcpyDefault, ctx->stream));
    QX_CUDA(cudaMemcpyAsync(sigma_c, a.sc, 2 * ob, cudaMemcpyDefault, ctx->stream));
    QX_CUDA(cudaMemcpyAsync(iterations, a.iters, norbs * sizeof(int), cudaMemcpyDefault, ctx->stream));
    QX_CUDA(cudaMemcpyAsync(method, a.method, norbs * sizeof(int), cudaMemcpyDefault, ctx->stream));
    sync_and_check(ctx);
  });
}

}  // extern "C"
