// G0W0 by contour deformation on the GPU.
//
//   Sigma_n(w) = I_n(w) + R_n(w)
//   I_n(w) = -(1/pi) sum_k wts_k sum_m Wc_nm(i f_k) (w - e_m) / ((w - e_m)^2 + f_k^2)
//   R_n(w) = - sum_{m occ, e_m > w} Wc_nm(e_m - w) + sum_{m vir, e_m < w} Wc_nm(w - e_m)
//
// The imaginary-axis integrand is the one of compute_sigma_c_pyscf_cd
// (quasix_core/src/selfenergy/correlation_pyscf_cd.rs:164-259) evaluated at
// the real target energy; the residue term, which the reference leaves as a
// skeleton (freq/contour_deformation.rs:142-239), follows the full-frequency
// contour-deformation formulation.  Wc_nm at the real shifts comes from
// eps(w) = I - Pi(w) with chi_ia = e_ia / (e_ia^2 - w^2), inverted by the same
// block sweep as on the imaginary axis (eps is indefinite above the lowest
// transition; the sweep needs no positive pivots).  The QP root is a Newton
// iteration with the analytic derivative, all targets at once.
#include <algorithm>

#include "qx_blas.cuh"
#include "qx_gw_sys.cuh"
#include "qx_internal.cuh"

namespace qx {

// I_t and dI_t/dw at w = omega[t].
__global__ void k_cd_imag(const double* __restrict__ v, int ldv, int nw, const int* __restrict__ pidx, int nmo,
                          const double* __restrict__ en, const double* __restrict__ freqs,
                          const double* __restrict__ wts, const double* __restrict__ omega,
                          double* __restrict__ out) {
  const int t = blockIdx.x;
  const double w0 = omega[t];
  double s = 0.0, ds = 0.0;
  for (int idx = threadIdx.x; idx < nw * nmo; idx += blockDim.x) {
    const int w = idx / nmo, m = idx % nmo;
    const double x = w0 - en[m], f2 = freqs[w] * freqs[w];
    const double den = x * x + f2;
    const double val = v[(size_t)w * ldv + pidx[(size_t)t * nmo + m]] * wts[w];
    s += val * x / den;
    ds += val * (f2 - x * x) / (den * den);
  }
  __shared__ double r1[256], r2[256];
  r1[threadIdx.x] = s;
  r2[threadIdx.x] = ds;
  __syncthreads();
  for (int o = 128; o > 0; o >>= 1) {
    if (threadIdx.x < o) {
      r1[threadIdx.x] += r1[threadIdx.x + o];
      r2[threadIdx.x] += r2[threadIdx.x + o];
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    out[2 * t] = -r1[0] / M_PI;
    out[2 * t + 1] = -r2[0] / M_PI;
  }
}

// b[r][P] = lpq[P][n_r][m_r]
__global__ void k_cd_gather(const double* __restrict__ lpq, int naux, int nmo, const int2* __restrict__ nm, int R,
                            double* __restrict__ b, int ld) {
  const int r = blockIdx.y;
  const int2 p = nm[r];
  for (int P = blockIdx.x * blockDim.x + threadIdx.x; P < ld; P += gridDim.x * blockDim.x)
    b[(size_t)r * ld + P] = (P < naux) ? lpq[(size_t)P * nmo * nmo + (size_t)p.x * nmo + p.y] : 0.0;
}

// x[r] = b[r] + Wc[r] b[r] (= eps^-1 b);  wc[r] = b^T Wc b.  One warp per row.
__global__ void k_cd_quad(const double* __restrict__ wc, int ldn, size_t stride, const double* __restrict__ b, int n,
                          int ld, double* __restrict__ x, double* __restrict__ val) {
  const int r = blockIdx.x;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarp = blockDim.x >> 5;
  const double* W = wc + (size_t)r * stride;
  const double* br = b + (size_t)r * ld;
  double q = 0.0;
  for (int P = warp; P < n; P += nwarp) {
    double s = 0.0;
    for (int Q = lane; Q < n; Q += 32) s += W[(size_t)P * ldn + Q] * br[Q];
    for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    if (lane == 0) {
      x[(size_t)r * ld + P] = br[P] + s;
      q += br[P] * s;
    }
  }
  __shared__ double red[32];
  if (lane == 0) red[warp] = q;
  __syncthreads();
  if (threadIdx.x == 0) {
    double t = 0.0;
    for (int i = 0; i < nwarp; ++i) t += red[i];
    val[r] = t;
  }
}

// dwc[r] = 4 sum_ia e_ia 2 w_r / (e_ia^2 - w_r^2)^2 (B_ia^T x_r)^2
__global__ void k_cd_dres(const double* __restrict__ tmat, int ldt, const double* __restrict__ en, int nocc, int nvir,
                          const double* __restrict__ wr, double* __restrict__ out) {
  const int r = blockIdx.x;
  const double w = wr[r];
  double s = 0.0;
  for (int k = threadIdx.x; k < nocc * nvir; k += blockDim.x) {
    const int i = k / nvir, a = k % nvir;
    const double e = en[i] - en[nocc + a];
    const double d = e * e - w * w;
    const double t = tmat[(size_t)r * ldt + k];
    s += e * 2.0 * w / (d * d) * t * t;
  }
  __shared__ double red[256];
  red[threadIdx.x] = s;
  __syncthreads();
  for (int o = 128; o > 0; o >>= 1) {
    if (threadIdx.x < o) red[threadIdx.x] += red[threadIdx.x + o];
    __syncthreads();
  }
  if (threadIdx.x == 0) out[r] = 4.0 * red[0];
}

}  // namespace qx

using namespace qx;

extern "C" qx_status qx_g0w0_cd(qx_ctx* ctx, const double* mo_energy, const double* lpq, const double* vxc, int nmo,
                                int nocc, int naux, const int* targets, int ntarget, int nw, double x0, double tol,
                                int max_iter, int precision, double* qp_energies, double* z_factors, double* sigma_c,
                                double* sigma_x) {
  if (!ctx) return QX_ERR_INVALID_INPUT;
  try {
    ctx->pending.clear();
    ctx->launches = 0;
    for (double& v : ctx->stage_ms) v = 0.0;
    QX_CUDA(cudaSetDevice(ctx->device));
    QX_REQUIRE(mo_energy && lpq && targets && qp_energies && ntarget > 0 && nw > 0 && max_iter > 0,
               QX_ERR_INVALID_INPUT, "invalid arguments to g0w0_cd");
    validate_common(nmo, nocc, naux);
    const int nvir = nmo - nocc;
    std::vector<double> e(nmo), vx(nmo, 0.0);
    QX_CUDA(cudaMemcpy(e.data(), mo_energy, nmo * sizeof(double), cudaMemcpyDefault));
    if (vxc) QX_CUDA(cudaMemcpy(vx.data(), vxc, nmo * sizeof(double), cudaMemcpyDefault));
    std::vector<int> tg(ntarget);
    QX_CUDA(cudaMemcpy(tg.data(), targets, ntarget * sizeof(int), cudaMemcpyDefault));
    for (int t : tg) QX_REQUIRE(t >= 0 && t < nmo, QX_ERR_INVALID_INPUT, "target orbital %d out of range", t);
    const double* d_lpq = (const double*)device_view(ctx, WS_LPQ, lpq, (size_t)naux * nmo * nmo * sizeof(double));
    // Imaginary axis: Wc_nm(i f_k) for the target pairs (no cutoff: the sigma grid is unused).
    GWSystem S;
    gw_setup(ctx, S, d_lpq, nmo, nocc, naux, tg, nw, 1e300, x0, precision);
    gw_wc_pairs(ctx, S, e.data());
    // Exchange.
    DevBuf& cb = ctx->ws[WS_CD0];
    cb.reserve((size_t)(nmo + 4 * ntarget + 64) * sizeof(double));
    double* d_sx = cb.as<double>();
    double* d_om = d_sx + nmo;
    double* d_imag = d_om + ntarget;
    launch_exchange_diag(ctx, d_lpq, naux, nmo, nocc, d_sx);
    std::vector<double> sx(nmo);
    QX_CUDA(cudaMemcpyAsync(sx.data(), d_sx, nmo * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
    // B_ov^T [nov][ldn] for the residue derivatives.
    const int nov = nocc * nvir, ldn = S.ldn;
    DevBuf& bt = ctx->ws[WS_CD1];
    bt.reserve((size_t)nov * ldn * sizeof(double));
    double* bovT = bt.as<double>();
    QX_CUDA(cudaMemsetAsync(bovT, 0, (size_t)nov * ldn * sizeof(double), ctx->stream));
    transpose(ctx, S.bov, naux, nov, S.ldov, 0, bovT, ldn, 0, 1);
    std::vector<double> om(ntarget), sig(ntarget, 0.0), dsig(ntarget, 0.0);
    std::vector<int> done(ntarget, 0), iters(ntarget, 0);
    for (int t = 0; t < ntarget; ++t) om[t] = e[tg[t]];
    auto evaluate = [&](const std::vector<int>& act) {
      // Imaginary-axis part for every target.
      QX_CUDA(cudaMemcpyAsync(d_om, om.data(), ntarget * sizeof(double), cudaMemcpyHostToDevice, ctx->stream));
      k_cd_imag<<<ntarget, 256, 0, ctx->stream>>>(S.v, S.npair, nw, S.d_pidx, nmo, S.d_en, S.d_freqs, S.d_wts, d_om,
                                                   d_imag);
      check_launch(ctx);
      std::vector<double> hi(2 * ntarget);
      QX_CUDA(cudaMemcpyAsync(hi.data(), d_imag, 2 * ntarget * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
      // Residue list.
      std::vector<int2> nm;
      std::vector<double> wr, sgn;
      std::vector<int> owner;
      for (int t : act) {
        const int n = tg[t];
        for (int m = 0; m < nmo; ++m) {
          if (m < nocc && e[m] > om[t]) {
            nm.push_back(make_int2(n, m));
            wr.push_back(e[m] - om[t]);
            sgn.push_back(-1.0);
            owner.push_back(t);
          } else if (m >= nocc && e[m] < om[t]) {
            nm.push_back(make_int2(n, m));
            wr.push_back(om[t] - e[m]);
            sgn.push_back(1.0);
            owner.push_back(t);
          }
        }
      }
      const int R = (int)nm.size();
      std::vector<double> rv(R), rd(R);
      if (R > 0) {
        const size_t stride = (size_t)naux * ldn;
        DevBuf& rb = ctx->ws[WS_CD2];
        const size_t need = (size_t)R * (stride + 2 * ldn + S.ldov + 4) * sizeof(double) + R * sizeof(int2) + 1024;
        rb.reserve(need);
        double* eps = rb.as<double>();
        double* b = eps + (size_t)R * stride;
        double* x = b + (size_t)R * ldn;
        double* tm = x + (size_t)R * ldn;
        double* d_wr = tm + (size_t)R * S.ldov;
        double* d_val = d_wr + R;
        double* d_dv = d_val + R;
        int2* d_nm = reinterpret_cast<int2*>(d_dv + R + 1);
        QX_CUDA(cudaMemcpyAsync(d_wr, wr.data(), R * sizeof(double), cudaMemcpyHostToDevice, ctx->stream));
        QX_CUDA(cudaMemcpyAsync(d_nm, nm.data(), R * sizeof(int2), cudaMemcpyHostToDevice, ctx->stream));
        // eps(w_r) = I + B_ov diag(chi'(w_r)) B_ov^T, real axis (chi buffer reused).
        ctx->ws[WS_CD3].reserve((size_t)R * S.ldov * sizeof(double));
        double* chi = ctx->ws[WS_CD3].as<double>();
        launch_chi(ctx, S.d_en, nocc, nvir, d_wr, R, 1, chi, S.ldov);
        launch_eps_fp64(ctx, S.bov, S.ldov, naux, nov, chi, R, eps, ldn, stride);
        launch_invert_wc(ctx, eps, naux, ldn, stride, R);
        dim3 gg(ceil_div(ldn, 256), R);
        k_cd_gather<<<gg, 256, 0, ctx->stream>>>(d_lpq, naux, nmo, d_nm, R, b, ldn);
        check_launch(ctx);
        k_cd_quad<<<R, 256, 0, ctx->stream>>>(eps, ldn, stride, b, naux, ldn, x, d_val);
        check_launch(ctx);
        GemmNT g{};
        g.M = R;
        g.N = nov;
        g.K = naux;
        g.A = x;
        g.lda = ldn;
        g.B = bovT;
        g.ldb = ldn;
        g.C = tm;
        g.ldc = S.ldov;
        g.batch = 1;
        g.alpha = 1.0;
        g.splitk = 0;
        gemm_nt_f64(ctx, g);
        k_cd_dres<<<R, 256, 0, ctx->stream>>>(tm, S.ldov, S.d_en, nocc, nvir, d_wr, d_dv);
        check_launch(ctx);
        QX_CUDA(cudaMemcpyAsync(rv.data(), d_val, R * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
        QX_CUDA(cudaMemcpyAsync(rd.data(), d_dv, R * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
      }
      sync_and_check(ctx);
      for (int t : act) {
        sig[t] = hi[2 * t];
        dsig[t] = hi[2 * t + 1];
      }
      for (int r = 0; r < R; ++r) {
        sig[owner[r]] += sgn[r] * rv[r];
        dsig[owner[r]] += rd[r];
      }
    };
    std::vector<int> act;
    for (int t = 0; t < ntarget; ++t) act.push_back(t);
    for (int it = 0; it < max_iter && !act.empty(); ++it) {
      evaluate(act);
      std::vector<int> next;
      for (int t : act) {
        const int n = tg[t];
        const double f = om[t] - e[n] - sx[n] - sig[t] + vx[n];
        iters[t] = it + 1;
        if (std::fabs(f) < tol) continue;  // converged at om[t]
        double step = -f / (1.0 - dsig[t]);
        step = std::min(std::max(step, -1.0), 1.0);
        om[t] += step;
        next.push_back(t);
      }
      act.swap(next);
    }
    // Final self-energy and slope at the returned energies.
    std::vector<int> all;
    for (int t = 0; t < ntarget; ++t) all.push_back(t);
    evaluate(all);
    std::vector<double> zf(ntarget), sxo(ntarget);
    for (int t = 0; t < ntarget; ++t) {
      zf[t] = 1.0 / (1.0 - dsig[t]);
      sxo[t] = sx[tg[t]];
      QX_REQUIRE(std::isfinite(om[t]) && std::isfinite(sig[t]), QX_ERR_NUMERICAL, "non-finite CD result for target %d",
                 tg[t]);
    }
    QX_CUDA(cudaMemcpy(qp_energies, om.data(), ntarget * sizeof(double), cudaMemcpyDefault));
    if (z_factors) QX_CUDA(cudaMemcpy(z_factors, zf.data(), ntarget * sizeof(double), cudaMemcpyDefault));
    if (sigma_c) QX_CUDA(cudaMemcpy(sigma_c, sig.data(), ntarget * sizeof(double), cudaMemcpyDefault));
    if (sigma_x) QX_CUDA(cudaMemcpy(sigma_x, sxo.data(), ntarget * sizeof(double), cudaMemcpyDefault));
    ctx->err.clear();
    return QX_OK;
  } catch (const Error& ex) {
    ctx->err = ex.what();
    return ex.status;
  } catch (const std::exception& ex) {
    ctx->err = ex.what();
    return QX_ERR_INVALID_INPUT;
  }
}
