// Adjoint of the contour-deformation QP roots (qx_g0w0_cd_grad).
//
// For L = sum_t lambda_t E_t, with E_t the root of
//   f_t(E) = E - e_n - Sx_n - Sigma_n(E) + Vxc_n      (Vxc held fixed),
// implicit differentiation gives dL = sum_t mu_t (de_n + dSx_n + dSigma_n|_E),
// mu_t = lambda_t / (1 - dSigma_n/dE).  Sigma_n = I_n + R_n as in qx_cd.cu,
// with every Wc_nm = b^T (eps^-1 - I) b, eps = I + B_ov diag(chi') B_ov^T:
//   dL/db_nm  = 2 c (x - b),  x = eps^-1 b
//   dL/deps   = G = -sum c x x^T
//   dL/dB_ov  = 2 G B_ov diag(chi'),   dL/dchi'_ia = b_ia^T G b_ia
// where c is the coefficient of Wc_nm in mu_t Sigma_n: mu_t (-1/pi) wts_k
// g(E_t - e_m, f_k) on the imaginary axis, mu_t sgn_r at a residue.  The
// orbital energies enter through e_ia = e_i - e_a in chi', through
// g(E - e_m, f) on the imaginary axis and through the residue shifts
// w_r = sgn_r (E - e_m).  P0 and W are rebuilt per frequency (chunked), not
// stored.  The reference has no derivative code; this follows the
// mathematics of the forward path (correlation_pyscf_cd.rs:164-259 for the
// imaginary-axis integrand).
#include <algorithm>

#include "qx_cd.cuh"

namespace qx {

constexpr int GRAD_FCMAX = 32;  // frequencies per chunk (register arrays below)

// Per (pair p = (t, m), frequency f of the chunk): v = b_p^T Wc_f b_p from
// Y = Wc_f b_p; coefficient c and the direct orbital-energy term; X = b + Y
// (= eps^-1 b) and c X written transposed for the G product.
__global__ void k_grad_imag_pairs(const double* __restrict__ bp, int ldn, const double* __restrict__ Y, int Tn,
                                  int naux, int nmo, const double* __restrict__ qp, const double* __restrict__ mu,
                                  const double* __restrict__ en, const double* __restrict__ freqs,
                                  const double* __restrict__ wts, double* __restrict__ cbuf,
                                  double* __restrict__ gef, double* __restrict__ XT, double* __restrict__ XsT,
                                  int ldT) {
  const int p = blockIdx.x, f = blockIdx.y;
  const int t = p / nmo, m = p % nmo;
  const double* b = bp + (size_t)p * ldn;
  const double* y = Y + ((size_t)f * Tn + p) * ldn;
  double s = 0.0;
  for (int P = threadIdx.x; P < naux; P += blockDim.x) s += b[P] * y[P];
  __shared__ double red[256];
  red[threadIdx.x] = s;
  __syncthreads();
  for (int o = blockDim.x / 2; o > 0; o >>= 1) {
    if (threadIdx.x < o) red[threadIdx.x] += red[threadIdx.x + o];
    __syncthreads();
  }
  const double v = red[0];
  const double x = qp[t] - en[m], F = freqs[f];
  const double den = x * x + F * F;
  const double c = mu[t] * (-1.0 / M_PI) * wts[f] * x / den;
  if (threadIdx.x == 0) {
    cbuf[(size_t)f * Tn + p] = c;
    gef[(size_t)f * Tn + p] = mu[t] * (1.0 / M_PI) * wts[f] * v * (F * F - x * x) / (den * den);
  }
  for (int P = threadIdx.x; P < naux; P += blockDim.x) {
    const double X = b[P] + y[P];
    XT[((size_t)f * naux + P) * ldT + p] = X;
    XsT[((size_t)f * naux + P) * ldT + p] = c * X;
  }
}

// g_bp[p][P] += sum_f 2 c[f][p] Y[f][p][P];  ge[p] += sum_f gef[f][p]
__global__ void k_grad_bp_accum(const double* __restrict__ Y, int ldn, int Tn, int naux, int fc,
                                const double* __restrict__ cbuf, const double* __restrict__ gef,
                                double* __restrict__ g_bp, double* __restrict__ ge) {
  const int p = blockIdx.x;
  for (int P = blockIdx.y * blockDim.x + threadIdx.x; P < naux; P += gridDim.y * blockDim.x) {
    double acc = 0.0;
    for (int f = 0; f < fc; ++f) acc += 2.0 * cbuf[(size_t)f * Tn + p] * Y[((size_t)f * Tn + p) * ldn + P];
    g_bp[(size_t)p * ldn + P] += acc;
  }
  if (blockIdx.y == 0 && threadIdx.x == 0) {
    double a = 0.0;
    for (int f = 0; f < fc; ++f) a += gef[(size_t)f * Tn + p];
    ge[p] += a;
  }
}

// For columns ia and a range of 64 rows P:
//   g_bov[P][ia] += 2 sum_f chi'_f[ia] H_f[P][ia]
//   part[f][pb][ia] = sum_{P in range} B_ov[P][ia] H_f[P][ia]
__global__ void k_grad_ov_imag(const double* __restrict__ bov, int ldov, int naux, int nov,
                               const double* __restrict__ H, const double* __restrict__ chi, int fc,
                               double* __restrict__ g_bov, double* __restrict__ part, int npb) {
  const int ia = blockIdx.x * blockDim.x + threadIdx.x;
  const int pb = blockIdx.y;
  if (ia >= nov) return;
  const size_t hs = (size_t)naux * ldov;
  double s[GRAD_FCMAX];
#pragma unroll
  for (int f = 0; f < GRAD_FCMAX; ++f) s[f] = 0.0;
  const int P1 = min(naux, (pb + 1) * 64);
  for (int P = pb * 64; P < P1; ++P) {
    const double bv = bov[(size_t)P * ldov + ia];
    double acc = 0.0;
#pragma unroll
    for (int f = 0; f < GRAD_FCMAX; ++f) {
      if (f < fc) {
        const double h = H[f * hs + (size_t)P * ldov + ia];
        acc += chi[(size_t)f * ldov + ia] * h;
        s[f] += bv * h;
      }
    }
    g_bov[(size_t)P * ldov + ia] += 2.0 * acc;
  }
#pragma unroll
  for (int f = 0; f < GRAD_FCMAX; ++f)
    if (f < fc) part[((size_t)f * npb + pb) * ldov + ia] = s[f];
}

// g_eia[ia] += sum_f dchi'/de (i f_f) * sum_pb part[f][pb][ia],
// dchi'/de = -4 (f^2 - e^2) / (f^2 + e^2)^2 on the imaginary axis.
__global__ void k_grad_eia_imag(const double* __restrict__ part, int npb, int ldov, int nov, int fc,
                                const double* __restrict__ en, int nocc, int nvir,
                                const double* __restrict__ freqs, double* __restrict__ g_eia) {
  const int ia = blockIdx.x * blockDim.x + threadIdx.x;
  if (ia >= nov) return;
  const double e = en[ia / nvir] - en[nocc + ia % nvir];
  double acc = 0.0;
  for (int f = 0; f < fc; ++f) {
    double s = 0.0;
    for (int pb = 0; pb < npb; ++pb) s += part[((size_t)f * npb + pb) * ldov + ia];
    const double F2 = freqs[f] * freqs[f], e2 = e * e;
    acc += s * (-4.0 * (F2 - e2) / ((F2 + e2) * (F2 + e2)));
  }
  g_eia[ia] += acc;
}

// Residues: g_bp[row_r][P] += 2 c_r (x_r[P] - b_r[P])
__global__ void k_grad_res_bp(const double* __restrict__ x, const double* __restrict__ b, int ldn, int naux,
                              const int* __restrict__ row, const double* __restrict__ coef,
                              double* __restrict__ g_bp) {
  const int r = blockIdx.x;
  for (int P = threadIdx.x; P < naux; P += blockDim.x)
    g_bp[(size_t)row[r] * ldn + P] += 2.0 * coef[r] * (x[(size_t)r * ldn + P] - b[(size_t)r * ldn + P]);
}

// Residues: g_bov[P][ia] -= 2 sum_r c_r x_r[P] t_r[ia] chi'_r[ia];
// g_eia[ia] -= sum_r c_r t_r[ia]^2 dchi'/de(w_r), dchi'/de = 4 (e^2 + w^2) / (e^2 - w^2)^2.
__global__ void k_grad_res_ov(const double* __restrict__ x, int ldn, const double* __restrict__ tm,
                              const double* __restrict__ chi, int ldov, int naux, int nov, int rc,
                              const double* __restrict__ coef, const double* __restrict__ wr,
                              const double* __restrict__ en, int nocc, int nvir, double* __restrict__ g_bov,
                              double* __restrict__ g_eia) {
  const int ia = blockIdx.x * blockDim.x + threadIdx.x;
  const int pb = blockIdx.y;
  if (ia >= nov) return;
  const int P1 = min(naux, (pb + 1) * 64);
  for (int P = pb * 64; P < P1; ++P) {
    double acc = 0.0;
    for (int r = 0; r < rc; ++r)
      acc += coef[r] * x[(size_t)r * ldn + P] * tm[(size_t)r * ldov + ia] * chi[(size_t)r * ldov + ia];
    g_bov[(size_t)P * ldov + ia] -= 2.0 * acc;
  }
  if (pb == 0) {
    const double e = en[ia / nvir] - en[nocc + ia % nvir], e2 = e * e;
    double acc = 0.0;
    for (int r = 0; r < rc; ++r) {
      const double t = tm[(size_t)r * ldov + ia], w2 = wr[r] * wr[r];
      const double d = e2 - w2;
      acc += coef[r] * t * t * 4.0 * (e2 + w2) / (d * d);
    }
    g_eia[ia] -= acc;
  }
}

// grad_lpq[P][p][q] = (raw(p, q) + raw(q, p)) / 2 with raw from the B_ov
// block, the target rows and Sigma_x.
__device__ __forceinline__ double grad_raw(int P, int p, int q, int nmo, int nocc, int nvir, int ldn, int ldov,
                                           const double* g_bov, const double* g_bp, const int* tidx,
                                           const double* mu, const double* lpq) {
  double r = 0.0;
  if (p < nocc && q >= nocc) r += g_bov[(size_t)P * ldov + p * nvir + (q - nocc)];
  const int t = tidx[p];
  if (t >= 0) {
    r += g_bp[((size_t)t * nmo + q) * ldn + P];
    if (q < nocc) r -= 2.0 * mu[t] * lpq[((size_t)P * nmo + p) * nmo + q];
  }
  return r;
}

__global__ void k_grad_assemble_lpq(int nmo, int nocc, int ldn, int ldov, const double* __restrict__ g_bov,
                                    const double* __restrict__ g_bp, const int* __restrict__ tidx,
                                    const double* __restrict__ mu, const double* __restrict__ lpq,
                                    double* __restrict__ out) {
  const int P = blockIdx.y;
  const int nvir = nmo - nocc;
  for (int idx = blockIdx.x * blockDim.x + threadIdx.x; idx < nmo * nmo; idx += gridDim.x * blockDim.x) {
    const int p = idx / nmo, q = idx % nmo;
    out[(size_t)P * nmo * nmo + idx] =
        0.5 * (grad_raw(P, p, q, nmo, nocc, nvir, ldn, ldov, g_bov, g_bp, tidx, mu, lpq) +
               grad_raw(P, q, p, nmo, nocc, nvir, ldn, ldov, g_bov, g_bp, tidx, mu, lpq));
  }
}

static void gemm(qx_ctx* ctx, int M, int N, int K, const double* A, int lda, size_t sA, const double* B, int ldb,
                 size_t sB, double* C, int ldc, size_t sC, int batch, double alpha) {
  GemmNT g{};
  g.M = M;
  g.N = N;
  g.K = K;
  g.A = A;
  g.lda = lda;
  g.sA = sA;
  g.B = B;
  g.ldb = ldb;
  g.sB = sB;
  g.C = C;
  g.ldc = ldc;
  g.sC = sC;
  g.batch = batch;
  g.alpha = alpha;
  g.beta = 0.0;
  g.splitk = 0;
  gemm_nt_f64(ctx, g);
}

}  // namespace qx

using namespace qx;

extern "C" qx_status qx_g0w0_cd_grad(qx_ctx* ctx, const double* mo_energy, const double* lpq, int nmo, int nocc,
                                     int naux, const int* targets, int ntarget, const double* qp_energies,
                                     const double* dl_dqp, int nw, double x0, int precision, double* grad_energy,
                                     double* grad_lpq, double* z_raw) {
  if (!ctx) return QX_ERR_INVALID_INPUT;
  try {
    reset_pending(ctx);
    ctx->launches = 0;
    for (double& v : ctx->stage_ms) v = 0.0;
    QX_CUDA(cudaSetDevice(ctx->device));
    QX_REQUIRE(qp_energies && dl_dqp && (grad_energy || grad_lpq), QX_ERR_INVALID_INPUT,
               "invalid arguments to g0w0_cd_grad");
    CdEngine E;
    E.ctx = ctx;
    E.setup(mo_energy, lpq, targets, ntarget, nmo, nocc, naux, nw, x0, precision);
    {
      std::vector<int> seen(nmo, 0);
      for (int t : E.tg) {
        QX_REQUIRE(!seen[t], QX_ERR_INVALID_INPUT, "target %d listed twice", t);
        seen[t] = 1;
      }
    }
    const int T = ntarget, nvir = E.nvir, nov = E.nov, ldn = E.ldn, ldov = E.S.ldov;
    std::vector<double> lam(T);
    QX_CUDA(cudaMemcpy(E.om.data(), qp_energies, T * sizeof(double), cudaMemcpyDefault));
    QX_CUDA(cudaMemcpy(lam.data(), dl_dqp, T * sizeof(double), cudaMemcpyDefault));
    // Pass 1: slope of Sigma at the roots -> mu_t = lambda_t Z_t (Z unclipped).
    std::vector<int> all(T);
    for (int t = 0; t < T; ++t) all[t] = t;
    E.evaluate(all);
    std::vector<double> mu(T), zr(T);
    for (int t = 0; t < T; ++t) {
      zr[t] = 1.0 / (1.0 - E.dsig[t]);
      mu[t] = lam[t] * zr[t];
    }
    // Accumulators and small arrays.
    const int Tn = T * nmo, ldT = round_up(Tn, 8);
    const int npb = ceil_div(naux, 64);
    const int fcap = std::min(GRAD_FCMAX, nw);
    size_t off = 0;
    auto carve = [&](size_t doubles) {
      size_t o = off;
      off += (doubles + 31) / 32 * 32;
      return o;
    };
    const size_t o_bp = carve((size_t)Tn * ldn), o_gbp = carve((size_t)Tn * ldn), o_gbov = carve((size_t)naux * ldov),
                 o_geia = carve(ldov), o_ge = carve(Tn), o_mu = carve(T), o_qp = carve(T), o_c = carve((size_t)fcap * Tn),
                 o_gef = carve((size_t)fcap * Tn), o_part = carve((size_t)fcap * npb * ldov), o_tidx = carve(nmo),
                 o_nm = carve(Tn), o_rrow = carve(4096), o_rcoef = carve(4096);
    DevBuf& g0 = ctx->ws[WS_GRAD0];
    g0.reserve(off * sizeof(double));
    double* base = g0.as<double>();
    double* bp = base + o_bp;
    double* g_bp = base + o_gbp;
    double* g_bov = base + o_gbov;
    double* g_eia = base + o_geia;
    double* ge = base + o_ge;
    double* d_mu = base + o_mu;
    double* d_qp = base + o_qp;
    double* cbuf = base + o_c;
    double* gef = base + o_gef;
    double* part = base + o_part;
    int* d_tidx = reinterpret_cast<int*>(base + o_tidx);
    int2* d_nm = reinterpret_cast<int2*>(base + o_nm);
    int* d_rrow = reinterpret_cast<int*>(base + o_rrow);
    double* d_rcoef = base + o_rcoef;
    QX_CUDA(cudaMemsetAsync(g_bp, 0, (size_t)Tn * ldn * sizeof(double), ctx->stream));
    QX_CUDA(cudaMemsetAsync(g_bov, 0, (size_t)naux * ldov * sizeof(double), ctx->stream));
    QX_CUDA(cudaMemsetAsync(g_eia, 0, ldov * sizeof(double), ctx->stream));
    QX_CUDA(cudaMemsetAsync(ge, 0, Tn * sizeof(double), ctx->stream));
    QX_CUDA(cudaMemcpyAsync(d_mu, mu.data(), T * sizeof(double), cudaMemcpyHostToDevice, ctx->stream));
    QX_CUDA(cudaMemcpyAsync(d_qp, E.om.data(), T * sizeof(double), cudaMemcpyHostToDevice, ctx->stream));
    std::vector<int> tidx(nmo, -1);
    for (int t = 0; t < T; ++t) tidx[E.tg[t]] = t;
    QX_CUDA(cudaMemcpyAsync(d_tidx, tidx.data(), nmo * sizeof(int), cudaMemcpyHostToDevice, ctx->stream));
    std::vector<int2> nm(Tn);
    for (int t = 0; t < T; ++t)
      for (int m = 0; m < nmo; ++m) nm[(size_t)t * nmo + m] = make_int2(E.tg[t], m);
    QX_CUDA(cudaMemcpyAsync(d_nm, nm.data(), Tn * sizeof(int2), cudaMemcpyHostToDevice, ctx->stream));
    launch_cd_gather(ctx, E.d_lpq, naux, nmo, d_nm, Tn, bp, ldn);

    // Pass 2a: imaginary axis, frequencies in chunks (eps, W rebuilt).
    const size_t stride = (size_t)naux * ldn;
    const size_t per_f = stride + (size_t)Tn * ldn + 2 * (size_t)naux * ldT + stride + (size_t)naux * ldov + ldov;
    const int fc_max = (int)std::max<size_t>(1, std::min<size_t>(fcap, ((size_t)2 << 30) / (per_f * sizeof(double))));
    DevBuf& g1 = ctx->ws[WS_GRAD1];
    g1.reserve(per_f * fc_max * sizeof(double) + 4096);
    double* eps = g1.as<double>();
    double* Yb = eps + stride * fc_max;
    double* XT = Yb + (size_t)Tn * ldn * fc_max;
    double* XsT = XT + (size_t)naux * ldT * fc_max;
    double* G = XsT + (size_t)naux * ldT * fc_max;
    double* H = G + stride * fc_max;
    double* chi = H + (size_t)naux * ldov * fc_max;
    // Split forms: H_f^T = B_ov^T G_f on tcgen05 (G_f is symmetric), from
    // B_ov^T split once and G_f split per chunk, then transposed to H_f.
    TcOperand bovT_split{}, g_split{};
    double* Ht = nullptr;
    const int fp16 = precision == QX_PREC_FP16X3;
    if (E.tc) {
      const size_t ae = (size_t)nov * ldn, ge = (size_t)fc_max * naux * ldn;
      const size_t ab = ((ae * 2 + 255) / 256) * 256, gb = ((ge * 2 + 255) / 256) * 256;
      DevBuf& g2 = ctx->ws[WS_GRAD2];
      g2.reserve(2 * ab + 2 * gb + (size_t)fc_max * nov * ldn * sizeof(double) + 1024);
      uint8_t* p2 = g2.as<uint8_t>();
      bovT_split = TcOperand{p2, p2 + ab, nullptr};
      g_split = TcOperand{p2 + 2 * ab, p2 + 2 * ab + gb, nullptr};
      Ht = reinterpret_cast<double*>(p2 + 2 * ab + 2 * gb);
      launch_split(ctx, E.bovT, nov, naux, ldn, bovT_split.hi, bovT_split.lo, ldn, 0, 0, 1, fp16, 0,
                   &bovT_split.scale);
    }
    for (int f0 = 0; f0 < nw; f0 += fc_max) {
      const int fc = std::min(fc_max, nw - f0);
      launch_chi(ctx, E.S.d_en, nocc, nvir, E.S.d_freqs + f0, fc, 0, chi, ldov);
      if (E.tc)
        launch_eps_tc(ctx, E.S.bov, ldov, naux, nov, chi, fc, eps, ldn, stride, precision == QX_PREC_FP16X3);
      else
        launch_eps_fp64(ctx, E.S.bov, ldov, naux, nov, chi, fc, eps, ldn, stride);
      launch_invert_wc(ctx, eps, naux, ldn, stride, fc, !eps_at_least_identity(E.e.data(), nocc, nvir, 0.0), 0,
                       /*split_update=*/E.tc);
      // Y[f][p] = Wc_f b_p
      gemm(ctx, Tn, naux, naux, bp, ldn, 0, eps, ldn, stride, Yb, ldn, (size_t)Tn * ldn, fc, 1.0);
      k_grad_imag_pairs<<<dim3(Tn, fc), 256, 0, ctx->stream>>>(bp, ldn, Yb, Tn, naux, nmo, d_qp, d_mu, E.S.d_en,
                                                               E.S.d_freqs + f0, E.S.d_wts + f0, cbuf, gef, XT,
                                                               XsT, ldT);
      check_launch(ctx);
      k_grad_bp_accum<<<dim3(Tn, ceil_div(naux, 256)), 256, 0, ctx->stream>>>(Yb, ldn, Tn, naux, fc, cbuf, gef,
                                                                              g_bp, ge);
      check_launch(ctx);
      // G_f = -sum_p c X X^T;  H_f = G_f B_ov
      gemm(ctx, naux, naux, Tn, XsT, ldT, (size_t)naux * ldT, XT, ldT, (size_t)naux * ldT, G, ldn, stride, fc, -1.0);
      if (E.tc) {
        launch_split(ctx, G, naux, naux, ldn, g_split.hi, g_split.lo, ldn, stride, (size_t)naux * ldn, fc, fp16, 2,
                     &g_split.scale);
        launch_gemm_tc(ctx, bovT_split, nov, ldn, g_split, naux, ldn, naux, fc, Ht, ldn, (size_t)nov * ldn, fp16);
        transpose(ctx, Ht, nov, naux, ldn, (size_t)nov * ldn, H, ldov, (size_t)naux * ldov, fc);
      } else {
        gemm(ctx, naux, nov, naux, G, ldn, stride, E.bovT, ldn, 0, H, ldov, (size_t)naux * ldov, fc, 1.0);
      }
      k_grad_ov_imag<<<dim3(ceil_div(nov, 128), npb), 128, 0, ctx->stream>>>(E.S.bov, ldov, naux, nov, H, chi, fc,
                                                                             g_bov, part, npb);
      check_launch(ctx);
      k_grad_eia_imag<<<ceil_div(nov, 256), 256, 0, ctx->stream>>>(part, npb, ldov, nov, fc, E.S.d_en, nocc, nvir,
                                                                   E.S.d_freqs + f0, g_eia);
      check_launch(ctx);
    }

    // Pass 2b: residues at the roots.
    std::vector<double> g_e(nmo, 0.0);
    const std::vector<CdResidue> res = E.residues(all);
    const int R = (int)res.size();
    if (R > 0) {
      CdResidueChunk c = E.residue_buffers(R);
      const int cap = std::min(c.cap, 4096);
      for (int c0 = 0; c0 < R; c0 += cap) {
        const int rc = std::min(cap, R - c0);
        E.residue_compute(c, res.data() + c0, rc);
        std::vector<int> rrow(rc);
        std::vector<double> rcoef(rc), dv(rc);
        for (int r = 0; r < rc; ++r) {
          const CdResidue& q = res[c0 + r];
          rrow[r] = q.t * nmo + q.m;
          rcoef[r] = mu[q.t] * q.sgn;
        }
        QX_CUDA(cudaMemcpyAsync(d_rrow, rrow.data(), rc * sizeof(int), cudaMemcpyHostToDevice, ctx->stream));
        QX_CUDA(cudaMemcpyAsync(d_rcoef, rcoef.data(), rc * sizeof(double), cudaMemcpyHostToDevice, ctx->stream));
        k_grad_res_bp<<<rc, 256, 0, ctx->stream>>>(c.x, c.b, ldn, naux, d_rrow, d_rcoef, g_bp);
        check_launch(ctx);
        k_grad_res_ov<<<dim3(ceil_div(nov, 128), npb), 128, 0, ctx->stream>>>(
            c.x, ldn, c.tm, c.chi, ldov, naux, nov, rc, d_rcoef, c.wr, E.S.d_en, nocc, nvir, g_bov, g_eia);
        check_launch(ctx);
        QX_CUDA(cudaMemcpyAsync(dv.data(), c.dv, rc * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
        sync_and_check(ctx);
        // The shift w_r = sgn (E - e_m) moves with e_m: dWc_r/de_m = -dWc/dw.
        for (int r = 0; r < rc; ++r) g_e[res[c0 + r].m] -= mu[res[c0 + r].t] * dv[r];
      }
    }

    // Orbital-energy gradient.
    std::vector<double> h_ge(Tn), h_geia(nov);
    QX_CUDA(cudaMemcpyAsync(h_ge.data(), ge, Tn * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
    QX_CUDA(cudaMemcpyAsync(h_geia.data(), g_eia, nov * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
    if (grad_lpq) {
      const bool dev_out = is_device_ptr(grad_lpq);
      double* out = grad_lpq;
      if (!dev_out) {
        ctx->ws[WS_GRAD2].reserve((size_t)naux * nmo * nmo * sizeof(double));
        out = ctx->ws[WS_GRAD2].as<double>();
      }
      dim3 ag(std::min(ceil_div(nmo * nmo, 256), 1024), naux);
      k_grad_assemble_lpq<<<ag, 256, 0, ctx->stream>>>(nmo, nocc, ldn, ldov, g_bov, g_bp, d_tidx, d_mu, E.d_lpq, out);
      check_launch(ctx);
      if (!dev_out)
        QX_CUDA(cudaMemcpyAsync(grad_lpq, out, (size_t)naux * nmo * nmo * sizeof(double), cudaMemcpyDeviceToHost,
                                ctx->stream));
    }
    sync_and_check(ctx);
    for (int t = 0; t < T; ++t) {
      g_e[E.tg[t]] += mu[t];
      for (int m = 0; m < nmo; ++m) g_e[m] += h_ge[(size_t)t * nmo + m];
    }
    for (int i = 0; i < nocc; ++i)
      for (int a = 0; a < nvir; ++a) {
        g_e[i] += h_geia[(size_t)i * nvir + a];
        g_e[nocc + a] -= h_geia[(size_t)i * nvir + a];
      }
    if (grad_energy) QX_CUDA(cudaMemcpy(grad_energy, g_e.data(), nmo * sizeof(double), cudaMemcpyDefault));
    if (z_raw) QX_CUDA(cudaMemcpy(z_raw, zr.data(), T * sizeof(double), cudaMemcpyDefault));
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
