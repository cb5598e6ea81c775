// BSE optical post-processing on the device: transition dipoles in the MO
// basis, oscillator strengths of the Davidson roots and the broadened
// absorption spectrum (quasix_core/src/bse/optical.rs:121-388,
// quasix/quasix/bse_driver.py:249-298 and 938-959).
//
// The transition dipoles are two FP64 DMMA GEMMs per Cartesian component
// (mu = C_occ^T D C_vir); the root dipoles d = X^T mu are one block
// reduction per root (n_trans is up to ~10^5, n_roots ~10); the spectrum is
// one thread per grid point over the roots.
#include <algorithm>

#include "qx_blas.cuh"
#include "qx_internal.cuh"

namespace qx {
namespace {

// mu[(i * nvir + a) * 3 + c] = m[c][i][a]  (the three component blocks
// interleaved into the reference's [n_trans][3] layout).
__global__ void k_interleave3(const double* __restrict__ m, int nov, int ldm, double* __restrict__ mu) {
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < 3 * nov; k += gridDim.x * blockDim.x) {
    const int t = k / 3, c = k % 3;
    mu[k] = m[(size_t)c * ldm + t];
  }
}

// d[n][c] = sum_t X[t][n] mu[t][c]; f[n] = 2/3 E_n |d_n|^2 (optical.rs:215-240).
// One block per root; a fixed-order tree reduction (deterministic).
__global__ void __launch_bounds__(256) k_root_dipoles(const double* __restrict__ x, int ldx, int n_trans,
                                                      const double* __restrict__ mu, const double* __restrict__ e,
                                                      double* __restrict__ d, double* __restrict__ f) {
  const int n = blockIdx.x;
  double s0 = 0.0, s1 = 0.0, s2 = 0.0;
  for (int t = threadIdx.x; t < n_trans; t += blockDim.x) {
    const double xv = x[(size_t)t * ldx + n];
    s0 += xv * mu[(size_t)t * 3];
    s1 += xv * mu[(size_t)t * 3 + 1];
    s2 += xv * mu[(size_t)t * 3 + 2];
  }
  __shared__ double r[3][256];
  r[0][threadIdx.x] = s0;
  r[1][threadIdx.x] = s1;
  r[2][threadIdx.x] = s2;
  __syncthreads();
  for (int o = 128; o > 0; o >>= 1) {
    if (threadIdx.x < o)
      for (int c = 0; c < 3; ++c) r[c][threadIdx.x] += r[c][threadIdx.x + o];
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    const double d0 = r[0][0], d1 = r[1][0], d2 = r[2][0];
    d[n * 3] = d0;
    d[n * 3 + 1] = d1;
    d[n * 3 + 2] = d2;
    f[n] = (2.0 / 3.0) * e[n] * (d0 * d0 + d1 * d1 + d2 * d2);
  }
}

// intensity[q] = sum_n f_n L(E_q - E_n) with L = gamma / (x^2 + gamma^2)
// (lorentzian) or exp(-x^2 / (2 gamma^2)) (gaussian), E_q = e_min + q de
// (compute_absorption_spectrum, optical.rs:305-385).
__global__ void k_absorption(const double* __restrict__ e, const double* __restrict__ f, int n_roots, int gaussian,
                             double gamma, double e_min, double de, int n_points, double* __restrict__ energies,
                             double* __restrict__ out) {
  const int q = blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= n_points) return;
  const double E = e_min + q * de;
  double s = 0.0;
  for (int n = 0; n < n_roots; ++n) {
    const double x = E - e[n];
    s += f[n] * (gaussian ? exp(-0.5 * x * x / (gamma * gamma)) : gamma / (x * x + gamma * gamma));
  }
  energies[q] = E;
  out[q] = s;
}

size_t a256(size_t b) { return (b + 255) & ~size_t(255); }

}  // namespace
}  // namespace qx

using namespace qx;

template <class F>
static qx_status run_optical(qx_ctx* ctx, F&& f) {
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

qx_status qx_compute_transition_dipoles(qx_ctx* ctx, const double* mo_coeff, const double* ao_dipoles, int nao,
                                        int nmo, int nocc, double* mu) {
  return run_optical(ctx, [&] {
    QX_REQUIRE(mo_coeff && ao_dipoles && mu && nao > 0 && nmo > 0 && nocc > 0 && nocc < nmo && nmo <= nao,
               QX_ERR_INVALID_INPUT, "invalid arguments to compute_transition_dipoles (nao=%d nmo=%d nocc=%d)", nao,
               nmo, nocc);
    const int nvir = nmo - nocc, nov = nocc * nvir;
    const int lda = round_up(nao, 8), ldm = round_up(nov, 8);
    const double* d_c = (const double*)device_view(ctx, WS_LPQ, mo_coeff, (size_t)nao * nmo * sizeof(double));
    // AO dipoles re-pitched to [3][nao][lda] (the GEMM wants 16-byte rows).
    DevBuf& wb = ctx->ws[WS_BSE0];
    const size_t b_dip = a256((size_t)3 * nao * lda * 8), b_ct = a256((size_t)nmo * lda * 8),
                 b_t = a256((size_t)3 * nvir * lda * 8), b_m = a256((size_t)3 * ldm * 8), b_mu = a256((size_t)3 * nov * 8);
    wb.reserve(b_dip + b_ct + b_t + b_m + b_mu);
    char* p = wb.as<char>();
    double* dip = reinterpret_cast<double*>(p);
    double* ct = reinterpret_cast<double*>(p + b_dip);
    double* tt = reinterpret_cast<double*>(p + b_dip + b_ct);
    double* m = reinterpret_cast<double*>(p + b_dip + b_ct + b_t);
    double* dmu = reinterpret_cast<double*>(p + b_dip + b_ct + b_t + b_m);
    QX_CUDA(cudaMemcpy2DAsync(dip, lda * sizeof(double), ao_dipoles, nao * sizeof(double), nao * sizeof(double),
                              (size_t)3 * nao, cudaMemcpyDefault, ctx->stream));
    // C^T [nmo][lda]: rows 0..nocc are C_occ^T, the rest C_vir^T.
    QX_CUDA(cudaMemsetAsync(ct, 0, b_ct, ctx->stream));
    transpose(ctx, d_c, nao, nmo, nmo, 0, ct, lda, 0, 1);
    for (int c = 0; c < 3; ++c) {
      // T^T[a][mu] = sum_nu C_vir^T[a][nu] D[mu][nu]
      GemmNT g1{nvir, nao, nao, ct + (size_t)nocc * lda, lda, 0, dip + (size_t)c * nao * lda, lda, 0,
                tt + (size_t)c * nvir * lda, lda, 0, 1, 1.0, 0.0, 0};
      gemm_nt_f64(ctx, g1);
    }
    for (int c = 0; c < 3; ++c) {
      // m[c][i][a] = sum_mu C_occ^T[i][mu] T^T[a][mu]
      GemmNT g2{nocc, nvir, nao, ct, lda, 0, tt + (size_t)c * nvir * lda, lda, 0, m + (size_t)c * ldm, nvir, 0, 1,
                1.0, 0.0, 0};
      gemm_nt_f64(ctx, g2);
    }
    k_interleave3<<<std::min(ceil_div(3 * nov, 256), 4 * ctx->sm_count), 256, 0, ctx->stream>>>(m, nov, ldm, dmu);
    check_launch(ctx);
    QX_CUDA(cudaMemcpyAsync(mu, dmu, (size_t)3 * nov * sizeof(double), cudaMemcpyDefault, ctx->stream));
    sync_and_check(ctx);
  });
}

qx_status qx_compute_oscillator_strengths(qx_ctx* ctx, const double* eigenvalues, const double* eigenvectors,
                                          const double* transition_dipoles, int n_trans, int n_roots,
                                          double* oscillator_strengths, double* root_dipoles, double* f_sum) {
  return run_optical(ctx, [&] {
    QX_REQUIRE(eigenvalues && eigenvectors && transition_dipoles && oscillator_strengths && n_trans > 0 &&
                   n_roots > 0,
               QX_ERR_INVALID_INPUT, "invalid arguments to compute_oscillator_strengths");
    std::vector<double> he(n_roots);
    QX_CUDA(cudaMemcpy(he.data(), eigenvalues, n_roots * sizeof(double), cudaMemcpyDefault));
    for (int i = 0; i < n_roots; ++i) {
      QX_REQUIRE(std::isfinite(he[i]), QX_ERR_NUMERICAL, "Non-finite eigenvalue at index %d: %g", i, he[i]);
      QX_REQUIRE(he[i] >= 0.0, QX_ERR_NUMERICAL,
                 "Negative eigenvalue at index %d: %g (BSE-TDA should give positive energies)", i, he[i]);
    }
    const double* d_x = (const double*)device_view(ctx, WS_LPQ, eigenvectors, (size_t)n_trans * n_roots * 8);
    const double* d_mu = (const double*)device_view(ctx, WS_BSE2, transition_dipoles, (size_t)n_trans * 3 * 8);
    DevBuf& wb = ctx->ws[WS_BSE1];
    wb.reserve(a256(n_roots * 8) + a256((size_t)n_roots * 3 * 8) + a256(n_roots * 8));
    double* d_e = wb.as<double>();
    double* d_d = reinterpret_cast<double*>(wb.as<char>() + a256(n_roots * 8));
    double* d_f = reinterpret_cast<double*>(wb.as<char>() + a256(n_roots * 8) + a256((size_t)n_roots * 24));
    QX_CUDA(cudaMemcpyAsync(d_e, he.data(), n_roots * sizeof(double), cudaMemcpyHostToDevice, ctx->stream));
    k_root_dipoles<<<n_roots, 256, 0, ctx->stream>>>(d_x, n_roots, n_trans, d_mu, d_e, d_d, d_f);
    check_launch(ctx);
    std::vector<double> hf(n_roots), hd((size_t)n_roots * 3);
    QX_CUDA(cudaMemcpyAsync(hf.data(), d_f, n_roots * 8, cudaMemcpyDeviceToHost, ctx->stream));
    QX_CUDA(cudaMemcpyAsync(hd.data(), d_d, (size_t)n_roots * 24, cudaMemcpyDeviceToHost, ctx->stream));
    sync_and_check(ctx);
    QX_CUDA(cudaMemcpy(oscillator_strengths, hf.data(), n_roots * 8, cudaMemcpyDefault));
    if (root_dipoles) QX_CUDA(cudaMemcpy(root_dipoles, hd.data(), (size_t)n_roots * 24, cudaMemcpyDefault));
    if (f_sum) {
      double s = 0.0;
      for (double v : hf) s += v;
      *f_sum = s;
    }
  });
}

qx_status qx_compute_absorption_spectrum(qx_ctx* ctx, const double* eigenvalues, const double* oscillator_strengths,
                                         int n_roots, int broadening_type, double broadening, int has_range,
                                         double e_min, double e_max, int n_points, double* energies,
                                         double* intensities) {
  return run_optical(ctx, [&] {
    QX_REQUIRE(eigenvalues && oscillator_strengths && energies && intensities && n_roots > 0 && n_points > 0 &&
                   (broadening_type == 0 || broadening_type == 1),
               QX_ERR_INVALID_INPUT, "invalid arguments to compute_absorption_spectrum");
    std::vector<double> he(n_roots), hf(n_roots);
    QX_CUDA(cudaMemcpy(he.data(), eigenvalues, n_roots * 8, cudaMemcpyDefault));
    QX_CUDA(cudaMemcpy(hf.data(), oscillator_strengths, n_roots * 8, cudaMemcpyDefault));
    if (!has_range) {
      // Auto range (optical.rs:332-340): eigenvalue span padded by
      // max(0.2 span, 5 broadening), clipped at 0 below.
      const double lo = *std::min_element(he.begin(), he.end()), hi = *std::max_element(he.begin(), he.end());
      const double pad = std::max((hi - lo) * 0.2, broadening * 5.0);
      e_min = std::max(lo - pad, 0.0);
      e_max = hi + pad;
    }
    const double de = n_points > 1 ? (e_max - e_min) / (n_points - 1) : 0.0;
    DevBuf& wb = ctx->ws[WS_BSE1];
    wb.reserve(2 * a256(n_roots * 8) + 2 * a256((size_t)n_points * 8));
    char* p = wb.as<char>();
    double* d_e = reinterpret_cast<double*>(p);
    double* d_f = reinterpret_cast<double*>(p + a256(n_roots * 8));
    double* d_w = reinterpret_cast<double*>(p + 2 * a256(n_roots * 8));
    double* d_i = reinterpret_cast<double*>(p + 2 * a256(n_roots * 8) + a256((size_t)n_points * 8));
    QX_CUDA(cudaMemcpyAsync(d_e, he.data(), n_roots * 8, cudaMemcpyHostToDevice, ctx->stream));
    QX_CUDA(cudaMemcpyAsync(d_f, hf.data(), n_roots * 8, cudaMemcpyHostToDevice, ctx->stream));
    k_absorption<<<ceil_div(n_points, 256), 256, 0, ctx->stream>>>(d_e, d_f, n_roots, broadening_type, broadening,
                                                                    e_min, de, n_points, d_w, d_i);
    check_launch(ctx);
    QX_CUDA(cudaMemcpyAsync(energies, d_w, (size_t)n_points * 8, cudaMemcpyDefault, ctx->stream));
    QX_CUDA(cudaMemcpyAsync(intensities, d_i, (size_t)n_points * 8, cudaMemcpyDefault, ctx->stream));
    sync_and_check(ctx);
  });
}

}  // extern "C"
