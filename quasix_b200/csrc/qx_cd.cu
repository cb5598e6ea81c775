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
#include <atomic>
#include <mutex>
#include <thread>

#include "qx_cd.cuh"

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

// x[r][P] = b[r][P] + sum_Q Wc[r][P][Q] b[r][Q] (= eps^-1 b): one warp per
// row P, many CTAs per residue.
__global__ void k_cd_solve_rows(const double* __restrict__ wc, int ldn, size_t stride, const double* __restrict__ b,
                                int n, int ld, double* __restrict__ x) {
  const int r = blockIdx.y;
  const int lane = threadIdx.x & 31;
  const int P = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
  if (P >= n) return;
  const double* W = wc + (size_t)r * stride + (size_t)P * ldn;
  const double* br = b + (size_t)r * ld;
  double s = 0.0;
  for (int Q = lane; Q < n; Q += 32) s += W[Q] * br[Q];
  for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
  if (lane == 0) x[(size_t)r * ld + P] = br[P] + s;
}

// val[r] = b^T Wc b = sum_P b[P] (x[P] - b[P])   (one CTA per residue, fixed order)
__global__ void k_cd_quad_reduce(const double* __restrict__ b, const double* __restrict__ x, int n, int ld,
                                 double* __restrict__ val) {
  const int r = blockIdx.x;
  double q = 0.0;
  for (int P = threadIdx.x; P < n; P += blockDim.x) {
    const double bv = b[(size_t)r * ld + P];
    q += bv * (x[(size_t)r * ld + P] - bv);
  }
  __shared__ double red[256];
  red[threadIdx.x] = q;
  __syncthreads();
  for (int o = 128; o > 0; o >>= 1) {
    if (threadIdx.x < o) red[threadIdx.x] += red[threadIdx.x + o];
    __syncthreads();
  }
  if (threadIdx.x == 0) val[r] = red[0];
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

void launch_cd_gather(qx_ctx* ctx, const double* lpq, int naux, int nmo, const int2* nm, int R, double* b, int ld) {
  dim3 gg(ceil_div(ld, 256), R);
  k_cd_gather<<<gg, 256, 0, ctx->stream>>>(lpq, naux, nmo, nm, R, b, ld);
  check_launch(ctx);
}

void CdEngine::setup(const double* mo_energy, const double* lpq, const int* targets, int ntarget_, int nmo_,
                     int nocc_, int naux_, int nw_, double x0, int precision_) {
  nmo = nmo_;
  nocc = nocc_;
  naux = naux_;
  ntarget = ntarget_;
  nw = nw_;
  precision = precision_;
  QX_REQUIRE(mo_energy && lpq && targets && ntarget > 0 && nw > 0, QX_ERR_INVALID_INPUT, "invalid CD arguments");
  validate_common(nmo, nocc, naux);
  nvir = nmo - nocc;
  nov = nocc * nvir;
  tc = is_tc_precision(precision);
  e.assign(nmo, 0.0);
  QX_CUDA(cudaMemcpy(e.data(), mo_energy, nmo * sizeof(double), cudaMemcpyDefault));
  tg.assign(ntarget, 0);
  QX_CUDA(cudaMemcpy(tg.data(), targets, ntarget * sizeof(int), cudaMemcpyDefault));
  for (int t : tg) QX_REQUIRE(t >= 0 && t < nmo, QX_ERR_INVALID_INPUT, "target orbital %d out of range", t);
  d_lpq = (const double*)device_view(ctx, WS_LPQ, lpq, (size_t)naux * nmo * nmo * sizeof(double));
  // Imaginary axis: Wc_nm(i f_k) for the target pairs (no cutoff: the sigma grid is unused).
  gw_setup(ctx, S, d_lpq, nmo, nocc, naux, tg, nw, 1e300, x0, precision);
  gw_wc_pairs(ctx, S, e.data());
  ldn = S.ldn;
  DevBuf& cb = ctx->ws[WS_CD0];
  cb.reserve((size_t)(nmo + 4 * ntarget + 64) * sizeof(double));
  double* d_sx = cb.as<double>();
  d_om = d_sx + nmo;
  d_imag = d_om + ntarget;
  launch_exchange_diag(ctx, d_lpq, naux, nmo, nocc, d_sx);
  sx.assign(nmo, 0.0);
  QX_CUDA(cudaMemcpyAsync(sx.data(), d_sx, nmo * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
  // B_ov^T [nov][ldn] for the residue derivatives.
  DevBuf& bt = ctx->ws[WS_CD1];
  bt.reserve((size_t)nov * ldn * sizeof(double));
  bovT = bt.as<double>();
  QX_CUDA(cudaMemsetAsync(bovT, 0, (size_t)nov * ldn * sizeof(double), ctx->stream));
  transpose(ctx, S.bov, naux, nov, S.ldov, 0, bovT, ldn, 0, 1);
  om.assign(ntarget, 0.0);
  sig.assign(ntarget, 0.0);
  dsig.assign(ntarget, 0.0);
  for (int t = 0; t < ntarget; ++t) om[t] = e[tg[t]];
}

std::vector<CdResidue> CdEngine::residues(const std::vector<int>& act) const {
  std::vector<CdResidue> out;
  for (int t : act) {
    for (int m = 0; m < nmo; ++m) {
      if (m < nocc && e[m] > om[t])
        out.push_back({t, m, -1.0, e[m] - om[t]});
      else if (m >= nocc && e[m] < om[t])
        out.push_back({t, m, 1.0, om[t] - e[m]});
    }
  }
  return out;
}

CdResidueChunk CdEngine::residue_buffers(int R) {
  // Chunks of RC frequencies keep the eps matrices (and, for the split forms,
  // the split operands) within ~2 GB.
  const size_t stride = (size_t)naux * ldn;
  const size_t per_res = (stride + S.ldov) * sizeof(double) + (tc ? (size_t)naux * S.ldov * 4 : 0);
  const int RC = (int)std::max<size_t>(1, std::min<size_t>((size_t)std::max(R, 1), ((size_t)2 << 30) / per_res));
  DevBuf& rb = ctx->ws[WS_CD2];
  rb.reserve((size_t)RC * (stride + 2 * ldn + S.ldov + 4) * sizeof(double) + RC * sizeof(int2) + 1024);
  CdResidueChunk c;
  c.cap = RC;
  c.eps = rb.as<double>();
  c.b = c.eps + (size_t)RC * stride;
  c.x = c.b + (size_t)RC * ldn;
  c.tm = c.x + (size_t)RC * ldn;
  c.wr = c.tm + (size_t)RC * S.ldov;
  c.val = c.wr + RC;
  c.dv = c.val + RC;
  c.nm = reinterpret_cast<int2*>(c.dv + RC + 1);
  ctx->ws[WS_CD3].reserve((size_t)RC * S.ldov * sizeof(double));
  c.chi = ctx->ws[WS_CD3].as<double>();
  return c;
}

void CdEngine::residue_compute(CdResidueChunk& c, const CdResidue* list, int rc) {
  const size_t stride = (size_t)naux * ldn;
  std::vector<double> wr(rc);
  std::vector<int2> nm(rc);
  for (int r = 0; r < rc; ++r) {
    wr[r] = list[r].w;
    nm[r] = make_int2(tg[list[r].t], list[r].m);
  }
  QX_CUDA(cudaMemcpyAsync(c.wr, wr.data(), rc * sizeof(double), cudaMemcpyHostToDevice, ctx->stream));
  QX_CUDA(cudaMemcpyAsync(c.nm, nm.data(), rc * sizeof(int2), cudaMemcpyHostToDevice, ctx->stream));
  // eps(w_r) = I + B_ov diag(chi'(w_r)) B_ov^T, real axis.
  launch_chi(ctx, S.d_en, nocc, nvir, c.wr, rc, 1, c.chi, S.ldov);
  if (tc)
    launch_eps_tc(ctx, S.bov, S.ldov, naux, nov, c.chi, rc, c.eps, ldn, stride, precision == QX_PREC_FP16X3);
  else
    launch_eps_fp64(ctx, S.bov, S.ldov, naux, nov, c.chi, rc, c.eps, ldn, stride);
  // Real axis: eps(w_r) is indefinite and can be ill-conditioned near an
  // excitation, so the sweep stays FP64 here.
  launch_invert_wc(ctx, c.eps, naux, ldn, stride, rc);
  launch_cd_gather(ctx, d_lpq, naux, nmo, c.nm, rc, c.b, ldn);
  k_cd_solve_rows<<<dim3(ceil_div(naux, 8), rc), 256, 0, ctx->stream>>>(c.eps, ldn, stride, c.b, naux, ldn, c.x);
  check_launch(ctx);
  k_cd_quad_reduce<<<rc, 256, 0, ctx->stream>>>(c.b, c.x, naux, ldn, c.val);
  check_launch(ctx);
  GemmNT g{};
  g.M = rc;
  g.N = nov;
  g.K = naux;
  g.A = c.x;
  g.lda = ldn;
  g.B = bovT;
  g.ldb = ldn;
  g.C = c.tm;
  g.ldc = S.ldov;
  g.batch = 1;
  g.alpha = 1.0;
  g.splitk = 0;
  gemm_nt_f64(ctx, g);
  k_cd_dres<<<rc, 256, 0, ctx->stream>>>(c.tm, S.ldov, S.d_en, nocc, nvir, c.wr, c.dv);
  check_launch(ctx);
}

void CdEngine::evaluate(const std::vector<int>& act) {
  // Imaginary-axis part for every target.
  QX_CUDA(cudaMemcpyAsync(d_om, om.data(), ntarget * sizeof(double), cudaMemcpyHostToDevice, ctx->stream));
  k_cd_imag<<<ntarget, 256, 0, ctx->stream>>>(S.v, S.npair, nw, S.d_pidx, nmo, S.d_en, S.d_freqs, S.d_wts, d_om,
                                               d_imag);
  check_launch(ctx);
  std::vector<double> hi(2 * ntarget);
  QX_CUDA(cudaMemcpyAsync(hi.data(), d_imag, 2 * ntarget * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
  const std::vector<CdResidue> res = residues(act);
  const int R = (int)res.size();
  std::vector<double> rv(R), rd(R);
  if (R > 0) {
    CdResidueChunk c = residue_buffers(R);
    for (int c0 = 0; c0 < R; c0 += c.cap) {
      const int rc = std::min(c.cap, R - c0);
      residue_compute(c, res.data() + c0, rc);
      QX_CUDA(cudaMemcpyAsync(rv.data() + c0, c.val, rc * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
      QX_CUDA(cudaMemcpyAsync(rd.data() + c0, c.dv, rc * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
    }
  }
  sync_and_check(ctx);
  for (int t : act) {
    sig[t] = hi[2 * t];
    dsig[t] = hi[2 * t + 1];
  }
  for (int r = 0; r < R; ++r) {
    sig[res[r].t] += res[r].sgn * rv[r];
    dsig[res[r].t] += rd[r];
  }
}

// One G0W0-CD problem (the arguments of qx_g0w0_cd).
struct CdProblem {
  const double* mo_energy;
  const double* lpq;
  const double* vxc;
  int nmo, nocc, naux;
  const int* targets;
  int ntarget, nw;
  double x0, tol;
  int max_iter, qp_solver, precision;
  double *qp, *z, *sc, *sx;
};

// Runs one system on ctx (throws qx::Error): imaginary-axis Wc for the target
// pairs once, then QP steps; each evaluation adds the residues of the poles
// between the target energy and the Fermi level.
void g0w0_cd_run(qx_ctx* ctx, const CdProblem& p) {
  QX_REQUIRE(p.qp && p.max_iter > 0, QX_ERR_INVALID_INPUT, "invalid arguments to g0w0_cd");
  QX_REQUIRE(p.qp_solver == QX_QP_NEWTON || p.qp_solver == QX_QP_LINEARIZED, QX_ERR_INVALID_INPUT,
             "qp_solver %d", p.qp_solver);
  CdEngine E;
  E.ctx = ctx;
  E.setup(p.mo_energy, p.lpq, p.targets, p.ntarget, p.nmo, p.nocc, p.naux, p.nw, p.x0, p.precision);
  const int ntarget = p.ntarget;
  std::vector<double> vx(p.nmo, 0.0);
  if (p.vxc) QX_CUDA(cudaMemcpy(vx.data(), p.vxc, p.nmo * sizeof(double), cudaMemcpyDefault));
  const std::vector<double>& e = E.e;
  const std::vector<double>& sx = E.sx;
  const std::vector<int>& tg = E.tg;
  std::vector<double>& om = E.om;
  const std::vector<double>& sig = E.sig;
  const std::vector<double>& dsig = E.dsig;
  constexpr double z_min = 0.1, z_max = 0.999;  // newton_solver.rs:93-95
  std::vector<double> zf(ntarget), sxo(ntarget);
  std::vector<int> all;
  for (int t = 0; t < ntarget; ++t) all.push_back(t);
  if (p.qp_solver == QX_QP_LINEARIZED) {
    // E = e_n + Z (Sx + Sigma(e_n) - Vxc), Z clipped (qp/evgw.rs:784-821).
    E.evaluate(all);
    for (int t = 0; t < ntarget; ++t) {
      const int n = tg[t];
      zf[t] = std::min(std::max(1.0 / (1.0 - dsig[t]), z_min), z_max);
      om[t] = e[n] + zf[t] * (sx[n] + sig[t] - vx[n]);
    }
  } else {
    // Newton with the step rule of NewtonQPSolver::solve (newton_solver.rs:174-280):
    // clipped step, adaptive damping in [0.1, 1].  fresh[t]: sig/dsig of
    // target t were evaluated at om[t].
    std::vector<int> act = all, fresh(ntarget, 0);
    std::vector<double> damping(ntarget, 1.0), prev(ntarget, HUGE_VAL);
    for (int it = 0; it < p.max_iter && !act.empty(); ++it) {
      E.evaluate(act);
      std::vector<int> next;
      for (int t : act) {
        const int n = tg[t];
        const double f = om[t] - e[n] - sx[n] - sig[t] + vx[n];
        const double af = std::fabs(f);
        fresh[t] = 1;
        if (af < p.tol) continue;  // converged at om[t]
        const double fp = 1.0 - dsig[t];
        double step = (std::fabs(fp) < 1e-10) ? -std::copysign(std::min(1.0, af), f) : -f / fp;
        step = std::min(std::max(step, -1.0), 1.0);
        if (af > prev[t])
          damping[t] = std::max(damping[t] * 0.5, 0.1);
        else if (af < 0.5 * prev[t] && damping[t] < 1.0)
          damping[t] = std::min(damping[t] * 1.2, 1.0);
        om[t] += damping[t] * step;
        prev[t] = af;
        fresh[t] = 0;
        next.push_back(t);
      }
      act.swap(next);
    }
    // Self-energy and slope at the returned energies (targets whose last
    // evaluation was before their final step).
    std::vector<int> stale;
    for (int t = 0; t < ntarget; ++t)
      if (!fresh[t]) stale.push_back(t);
    if (!stale.empty()) E.evaluate(stale);
    for (int t = 0; t < ntarget; ++t) zf[t] = std::min(std::max(1.0 / (1.0 - dsig[t]), z_min), z_max);
  }
  for (int t = 0; t < ntarget; ++t) {
    sxo[t] = sx[tg[t]];
    QX_REQUIRE(std::isfinite(om[t]) && std::isfinite(sig[t]), QX_ERR_NUMERICAL, "non-finite CD result for target %d",
               tg[t]);
  }
  QX_CUDA(cudaMemcpy(p.qp, om.data(), ntarget * sizeof(double), cudaMemcpyDefault));
  if (p.z) QX_CUDA(cudaMemcpy(p.z, zf.data(), ntarget * sizeof(double), cudaMemcpyDefault));
  if (p.sc) QX_CUDA(cudaMemcpy(p.sc, sig.data(), ntarget * sizeof(double), cudaMemcpyDefault));
  if (p.sx) QX_CUDA(cudaMemcpy(p.sx, sxo.data(), ntarget * sizeof(double), cudaMemcpyDefault));
}

// Worker context of a batch: its own non-blocking stream and workspace, so
// that systems on different workers overlap on the device.
qx_ctx* make_worker(int device) {
  qx_ctx* c = new qx_ctx();
  c->device = device;
  c->worker = true;
  try {
    cudaDeviceProp pr;
    QX_CUDA(cudaGetDeviceProperties(&pr, device));
    c->sm_count = pr.multiProcessorCount;
    QX_CUDA(cudaStreamCreateWithFlags(&c->own_stream, cudaStreamNonBlocking));
    c->stream = c->own_stream;
    for (auto& ev : c->ev) QX_CUDA(cudaEventCreate(&ev));
  } catch (...) {
    qx_ctx_destroy(c);
    throw;
  }
  return c;
}

}  // namespace qx

using namespace qx;

extern "C" qx_status qx_g0w0_cd(qx_ctx* ctx, const double* mo_energy, const double* lpq, const double* vxc, int nmo,
                                int nocc, int naux, const int* targets, int ntarget, int nw, double x0, double tol,
                                int max_iter, int qp_solver, int precision, double* qp_energies, double* z_factors,
                                double* sigma_c, double* sigma_x) {
  if (!ctx) return QX_ERR_INVALID_INPUT;
  try {
    reset_pending(ctx);
    ctx->launches = 0;
    for (double& v : ctx->stage_ms) v = 0.0;
    QX_CUDA(cudaSetDevice(ctx->device));
    CdProblem p{mo_energy, lpq, vxc, nmo, nocc, naux, targets, ntarget, nw, x0, tol, max_iter, qp_solver, precision,
                qp_energies, z_factors, sigma_c, sigma_x};
    g0w0_cd_run(ctx, p);
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

extern "C" qx_status qx_cd_sigma(qx_ctx* ctx, const double* mo_energy, const double* lpq, int nmo, int nocc,
                                 int naux, const int* targets, int ntarget, const double* omega, int nw, double x0,
                                 int precision, double* sigma_c, double* dsigma_c, double* sigma_x) {
  if (!ctx) return QX_ERR_INVALID_INPUT;
  try {
    reset_pending(ctx);
    ctx->launches = 0;
    for (double& v : ctx->stage_ms) v = 0.0;
    QX_CUDA(cudaSetDevice(ctx->device));
    QX_REQUIRE(omega && sigma_c, QX_ERR_INVALID_INPUT, "invalid arguments to cd_sigma");
    CdEngine E;
    E.ctx = ctx;
    E.setup(mo_energy, lpq, targets, ntarget, nmo, nocc, naux, nw, x0, precision);
    QX_CUDA(cudaMemcpy(E.om.data(), omega, ntarget * sizeof(double), cudaMemcpyDefault));
    std::vector<int> all(ntarget);
    for (int t = 0; t < ntarget; ++t) all[t] = t;
    E.evaluate(all);
    std::vector<double> sxo(ntarget);
    for (int t = 0; t < ntarget; ++t) sxo[t] = E.sx[E.tg[t]];
    QX_CUDA(cudaMemcpy(sigma_c, E.sig.data(), ntarget * sizeof(double), cudaMemcpyDefault));
    if (dsigma_c) QX_CUDA(cudaMemcpy(dsigma_c, E.dsig.data(), ntarget * sizeof(double), cudaMemcpyDefault));
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

extern "C" qx_status qx_g0w0_cd_batch(qx_ctx* ctx, qx_cd_system* systems, int nsys, int nw, double x0, double tol,
                                      int max_iter, int qp_solver, int precision, int nworkers) {
  if (!ctx) return QX_ERR_INVALID_INPUT;
  try {
    reset_pending(ctx);
    ctx->launches = 0;
    for (double& v : ctx->stage_ms) v = 0.0;
    QX_CUDA(cudaSetDevice(ctx->device));
    QX_REQUIRE(systems && nsys > 0 && nw > 0 && max_iter > 0, QX_ERR_INVALID_INPUT, "invalid arguments to g0w0_cd_batch");
    QX_REQUIRE(precision >= QX_PREC_FP64 && precision <= QX_PREC_FP16X3, QX_ERR_INVALID_INPUT, "precision %d",
               precision);
    if (nworkers <= 0) nworkers = 4;
    nworkers = std::min(std::min(nworkers, 16), nsys);
    // Inputs may have been produced on the caller's stream.
    QX_CUDA(cudaStreamSynchronize(ctx->stream));
    while ((int)ctx->workers.size() < nworkers) ctx->workers.push_back(make_worker(ctx->device));
    // Largest systems first (P0 cost nov * naux^2 dominates), so that the
    // small ones fill in behind them.
    std::vector<int> order(nsys);
    std::vector<double> cost(nsys);
    for (int i = 0; i < nsys; ++i) {
      const qx_cd_system& s = systems[i];
      order[i] = i;
      cost[i] = (double)s.nocc * (s.nmo - s.nocc) * s.naux * (double)s.naux + (double)s.naux * s.naux * s.naux;
      systems[i].status = QX_ERR_INVALID_INPUT;
    }
    std::stable_sort(order.begin(), order.end(), [&](int a, int b) { return cost[a] > cost[b]; });
    std::atomic<int> next{0};
    std::mutex mu;
    std::vector<std::string> msg(nsys);
    auto work = [&](qx_ctx* w) {
      if (cudaSetDevice(w->device) != cudaSuccess) return;
      for (;;) {
        const int k = next.fetch_add(1);
        if (k >= nsys) break;
        qx_cd_system& s = systems[order[k]];
        reset_pending(w);
        try {
          CdProblem p{s.mo_energy, s.lpq, s.vxc,    s.nmo,      s.nocc,       s.naux,      s.targets,
                      s.ntarget,   nw,    x0,      tol,      max_iter,   qp_solver,    precision,   s.qp_energies,
                      s.z_factors, s.sigma_c, s.sigma_x};
          g0w0_cd_run(w, p);
          s.status = QX_OK;
        } catch (const Error& ex) {
          s.status = ex.status;
          std::lock_guard<std::mutex> lock(mu);
          msg[order[k]] = ex.what();
        } catch (const std::exception& ex) {
          s.status = QX_ERR_INVALID_INPUT;
          std::lock_guard<std::mutex> lock(mu);
          msg[order[k]] = ex.what();
        }
      }
    };
    for (auto* w : ctx->workers) w->launches = 0;
    std::vector<std::thread> th;
    for (int i = 0; i < nworkers; ++i) th.emplace_back(work, ctx->workers[i]);
    for (auto& t : th) t.join();
    for (int i = 0; i < nworkers; ++i) ctx->launches += ctx->workers[i]->launches;
    for (int i = 0; i < nsys; ++i)
      if (systems[i].status != QX_OK)
        throw Error((qx_status)systems[i].status, fmt("system %d: %s", i, msg[i].c_str()));
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
