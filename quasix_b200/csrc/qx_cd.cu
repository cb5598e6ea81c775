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

// t[r][k] *= chi[r][k] over rc rows of n columns (row stride ld).
__global__ void k_cd_scale_rows(double* __restrict__ t, const double* __restrict__ chi, int rc, int n, int ld) {
  for (size_t e = (size_t)blockIdx.x * blockDim.x + threadIdx.x; e < (size_t)rc * n;
       e += (size_t)gridDim.x * blockDim.x) {
    const size_t r = e / n, k = e % n;
    t[r * ld + k] *= chi[r * ld + k];
  }
}

// y <- b - x - y (the residual b - eps x with y = B (chi' B^T x)), rc rows of n.
__global__ void k_cd_residual(const double* __restrict__ b, const double* __restrict__ x, double* __restrict__ y,
                              int rc, int n, int ld) {
  for (size_t e = (size_t)blockIdx.x * blockDim.x + threadIdx.x; e < (size_t)rc * n;
       e += (size_t)gridDim.x * blockDim.x) {
    const size_t i = (e / n) * ld + e % n;
    y[i] = b[i] - x[i] - y[i];
  }
}

// x += d, rc rows of n.
__global__ void k_cd_add_rows(double* __restrict__ x, const double* __restrict__ d, int rc, int n, int ld) {
  for (size_t e = (size_t)blockIdx.x * blockDim.x + threadIdx.x; e < (size_t)rc * n;
       e += (size_t)gridDim.x * blockDim.x) {
    const size_t i = (e / n) * ld + e % n;
    x[i] += d[i];
  }
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
  setup_begin(mo_energy, lpq, targets, ntarget_, nmo_, nocc_, naux_, nw_, x0, precision_);
  record_stage(ctx, QX_ST_INV, true);
  launch_invert_wc(ctx, S.eps, S.naux, S.ldn, S.eps_stride, S.nw, !eps_at_least_identity(e.data(), nocc, nvir, 0.0),
                   /*half_lower=*/1, /*split_update=*/tc);
  record_stage(ctx, QX_ST_INV, false);
  setup_end();
}

void CdEngine::setup_begin(const double* mo_energy, const double* lpq, const int* targets, int ntarget_, int nmo_,
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
  gw_wc_p0(ctx, S, e.data());
  ldn = S.ldn;
  // Pinned staging: diag(Sigma_x), the imaginary-axis values and the residue
  // values (at most ntarget * nmo residues).
  ctx->host_stage.reserve((size_t)(nmo + 2 * ntarget + 2 * (size_t)ntarget * nmo + 8) * sizeof(double));
  h_sx = ctx->host_stage.as<double>();
  h_hi = h_sx + nmo;
  h_rv = h_hi + 2 * ntarget;
  h_rd = h_rv + (size_t)ntarget * nmo;
}

void CdEngine::eps_matrices(std::vector<GMat>& out) const {
  const int guard = !eps_at_least_identity(e.data(), nocc, nvir, 0.0);
  for (int w = 0; w < nw; ++w) out.push_back(GMat{S.eps + (size_t)w * S.eps_stride, naux, S.ldn, 0, guard});
}

void CdEngine::setup_end() {
  // The imaginary-axis eps was inverted unguarded exactly when it is certified >= I.
  S.wc_unit_bound = eps_at_least_identity(e.data(), nocc, nvir, 0.0);
  gw_wc_contract(ctx, S);
  DevBuf& cb = ctx->ws[WS_CD0];
  cb.reserve((size_t)(nmo + 4 * ntarget + 64) * sizeof(double));
  double* d_sx = cb.as<double>();
  d_om = d_sx + nmo;
  d_imag = d_om + ntarget;
  // Sigma_x of the targets only (the other entries of sx stay zero).
  QX_CUDA(cudaMemsetAsync(d_sx, 0, nmo * sizeof(double), ctx->stream));
  launch_exchange_diag(ctx, d_lpq, naux, nmo, nocc, d_sx, S.d_orbs, ntarget);
  // Read into sx at the next evaluation's synchronisation.
  sx.assign(nmo, 0.0);
  QX_CUDA(cudaMemcpyAsync(h_sx, d_sx, nmo * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
  sx_pending = true;
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
  rb.reserve((size_t)RC * (stride + 4 * ldn + S.ldov + 4) * sizeof(double) + RC * sizeof(int2) + 1024);
  CdResidueChunk c;
  c.cap = RC;
  c.eps = rb.as<double>();
  c.b = c.eps + (size_t)RC * stride;
  c.x = c.b + (size_t)RC * ldn;
  c.y = c.x + (size_t)RC * ldn;
  c.dx = c.y + (size_t)RC * ldn;
  c.tm = c.dx + (size_t)RC * ldn;
  c.wr = c.tm + (size_t)RC * S.ldov;
  c.val = c.wr + RC;
  c.dv = c.val + RC;
  c.nm = reinterpret_cast<int2*>(c.dv + RC + 1);
  ctx->ws[WS_CD3].reserve((size_t)RC * S.ldov * sizeof(double));
  c.chi = ctx->ws[WS_CD3].as<double>();
  return c;
}

void CdEngine::residue_compute(CdResidueChunk& c, const CdResidue* list, int rc) {
  residue_p0(c, list, rc);
  // Real axis: eps(w_r) is indefinite once a shift passes the smallest
  // transition, and can be ill-conditioned near an excitation, so the sweep
  // stays FP64 here, guarded unless every shift lies below the gap.
  double wmax = 0.0;
  for (int r = 0; r < rc; ++r) wmax = std::max(wmax, std::fabs(list[r].w));
  const bool guard = !eps_at_least_identity(e.data(), nocc, nvir, wmax);
  launch_invert_wc(ctx, c.eps, naux, ldn, (size_t)naux * ldn, rc, guard);
  residue_post(c, rc, guard);
}

void CdEngine::residue_p0(CdResidueChunk& c, const CdResidue* list, int rc) {
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
    launch_eps_tc(ctx, S.bov, S.ldov, naux, nov, c.chi, rc, c.eps, ldn, stride, precision == QX_PREC_FP16X3,
                  /*reuse_a=*/1);
  else
    launch_eps_fp64(ctx, S.bov, S.ldov, naux, nov, c.chi, rc, c.eps, ldn, stride);
}

void CdEngine::residue_post(CdResidueChunk& c, int rc, bool refine) {
  const size_t stride = (size_t)naux * ldn;
  launch_cd_gather(ctx, d_lpq, naux, nmo, c.nm, rc, c.b, ldn);
  k_cd_solve_rows<<<dim3(ceil_div(naux, 8), rc), 256, 0, ctx->stream>>>(c.eps, ldn, stride, c.b, naux, ldn, c.x);
  check_launch(ctx);
  // One step of iterative refinement of x against the FP64 eps(w_r) = I + B_ov
  // diag(chi') B_ov^T, applied without forming it: near an excitation eps is
  // dominated by one huge rank-1 term, and the slope reads the small
  // component B_ov^T x along it, which the explicit (pivoted) inverse alone
  // gets only to ~kappa u (the reference's LU solve is componentwise accurate
  // there; one refinement step restores that).  A certified eps >= I (every
  // shift below the gap) is well conditioned and needs none.
  if (refine) {
    const int blk = std::min(ceil_div(rc * std::max(nov, naux), 256), 4 * ctx->sm_count);
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
    k_cd_scale_rows<<<blk, 256, 0, ctx->stream>>>(c.tm, c.chi, rc, nov, S.ldov);
    check_launch(ctx);
    GemmNT h{};
    h.M = rc;
    h.N = naux;
    h.K = nov;
    h.A = c.tm;
    h.lda = S.ldov;
    h.B = S.bov;
    h.ldb = S.ldov;
    h.C = c.y;
    h.ldc = ldn;
    h.batch = 1;
    h.alpha = 1.0;
    h.splitk = 0;
    gemm_nt_f64(ctx, h);
    k_cd_residual<<<blk, 256, 0, ctx->stream>>>(c.b, c.x, c.y, rc, naux, ldn);
    check_launch(ctx);
    k_cd_solve_rows<<<dim3(ceil_div(naux, 8), rc), 256, 0, ctx->stream>>>(c.eps, ldn, stride, c.y, naux, ldn,
                                                                          c.dx);
    check_launch(ctx);
    k_cd_add_rows<<<blk, 256, 0, ctx->stream>>>(c.x, c.dx, rc, naux, ldn);
    check_launch(ctx);
  }
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
  evaluate_begin(act, nullptr);
  evaluate_end();
}

void CdEngine::evaluate_begin(const std::vector<int>& act, std::vector<GMat>* group) {
  ev_act = act;
  // Imaginary-axis part for every target.
  QX_CUDA(cudaMemcpyAsync(d_om, om.data(), ntarget * sizeof(double), cudaMemcpyHostToDevice, ctx->stream));
  k_cd_imag<<<ntarget, 256, 0, ctx->stream>>>(S.v, S.npair, nw, S.d_pidx, nmo, S.d_en, S.d_freqs, S.d_wts, d_om,
                                               d_imag);
  check_launch(ctx);
  QX_CUDA(cudaMemcpyAsync(h_hi, d_imag, 2 * ntarget * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
  ev_res = residues(act);
  const int R = (int)ev_res.size();
  ev_grouped = false;
  // eps(w) = I + B diag(chi'(w)) B^T with chi'_ia(w) = -4 e_ia / (e_ia^2 - w^2)
  // is SPD when every shift is below the smallest transition |e_ia| (chi' >
  // 0); with a 0.9 margin its eigenvalues lie in [1, 1 + ||Pi(0)|| / 0.19].
  double wmax = 0.0;
  for (const CdResidue& r : ev_res) wmax = std::max(wmax, std::fabs(r.w));
  // The gap is min(virtual) - max(occupied): QP levels need not stay ordered.
  ev_spd = eps_at_least_identity(e.data(), nocc, nvir, wmax / 0.9);
  const int guard = !eps_at_least_identity(e.data(), nocc, nvir, wmax);
  ev_guard = guard != 0;
  if (R == 0) return;
  ev_chunk = residue_buffers(R);
  CdResidueChunk& c = ev_chunk;
  if (group && R <= c.cap) {
    // One chunk: its eps(w_r) join the caller's grouped inversion.
    residue_p0(c, ev_res.data(), R);
    for (int r = 0; r < R; ++r) group->push_back(GMat{c.eps + (size_t)r * naux * ldn, naux, ldn, 0, guard});
    ev_grouped = true;
    return;
  }
  for (int c0 = 0; c0 < R; c0 += c.cap) {
    const int rc = std::min(c.cap, R - c0);
    residue_compute(c, ev_res.data() + c0, rc);
    QX_CUDA(cudaMemcpyAsync(h_rv + c0, c.val, rc * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
    QX_CUDA(cudaMemcpyAsync(h_rd + c0, c.dv, rc * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
  }
}

void CdEngine::evaluate_end() {
  evaluate_post();
  evaluate_finish();
}

void CdEngine::evaluate_post() {
  const int R = (int)ev_res.size();
  if (ev_grouped) {
    residue_post(ev_chunk, R, ev_guard);
    QX_CUDA(cudaMemcpyAsync(h_rv, ev_chunk.val, R * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
    QX_CUDA(cudaMemcpyAsync(h_rd, ev_chunk.dv, R * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
  }
}

void CdEngine::evaluate_finish() {
  const int R = (int)ev_res.size();
  sync_and_check(ctx);
  if (sx_pending) {
    sx.assign(h_sx, h_sx + nmo);
    sx_pending = false;
  }
  ev_hi.assign(h_hi, h_hi + 2 * ntarget);
  ev_rv.assign(h_rv, h_rv + R);
  ev_rd.assign(h_rd, h_rd + R);
  for (int t : ev_act) {
    sig[t] = ev_hi[2 * t];
    dsig[t] = ev_hi[2 * t + 1];
  }
  for (int r = 0; r < R; ++r) {
    sig[ev_res[r].t] += ev_res[r].sgn * ev_rv[r];
    dsig[ev_res[r].t] += ev_rd[r];
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

// QP root search of one system as a sequence of evaluations: first() gives
// the targets to evaluate first, advance() consumes that evaluation (E.sig,
// E.dsig at E.om) and gives the next list (empty: done), finish() writes the
// outputs.  The single-system driver and the grouped batch step through it.
struct CdRun {
  CdEngine E;
  const CdProblem* p = nullptr;
  std::vector<double> vx, zf, damping, prev;
  std::vector<int> fresh;
  int it = 0;
  bool final_pass = false;
  static constexpr double z_min = 0.1, z_max = 0.999;  // newton_solver.rs:93-95

  void init(const CdProblem& prob) {
    p = &prob;
    QX_REQUIRE(p->qp && p->max_iter > 0, QX_ERR_INVALID_INPUT, "invalid arguments to g0w0_cd");
    QX_REQUIRE(p->qp_solver == QX_QP_NEWTON || p->qp_solver == QX_QP_LINEARIZED, QX_ERR_INVALID_INPUT,
               "qp_solver %d", p->qp_solver);
    vx.assign(p->nmo, 0.0);
    if (p->vxc) QX_CUDA(cudaMemcpy(vx.data(), p->vxc, p->nmo * sizeof(double), cudaMemcpyDefault));
    zf.assign(p->ntarget, 0.0);
    damping.assign(p->ntarget, 1.0);
    prev.assign(p->ntarget, HUGE_VAL);
    fresh.assign(p->ntarget, 0);
  }
  std::vector<int> first() const {
    std::vector<int> all(p->ntarget);
    for (int t = 0; t < p->ntarget; ++t) all[t] = t;
    return all;
  }
  std::vector<int> advance(const std::vector<int>& act) {
    const std::vector<double>& e = E.e;
    const std::vector<double>& sx = E.sx;
    const std::vector<int>& tg = E.tg;
    std::vector<double>& om = E.om;
    const int ntarget = p->ntarget;
    if (p->qp_solver == QX_QP_LINEARIZED) {
      // E = e_n + Z (Sx + Sigma(e_n) - Vxc), Z clipped (qp/evgw.rs:784-821).
      for (int t = 0; t < ntarget; ++t) {
        const int n = tg[t];
        zf[t] = std::min(std::max(1.0 / (1.0 - E.dsig[t]), z_min), z_max);
        om[t] = e[n] + zf[t] * (sx[n] + E.sig[t] - vx[n]);
      }
      return {};
    }
    if (!final_pass) {
      // Newton with the step rule of NewtonQPSolver::solve
      // (newton_solver.rs:174-280): clipped step, adaptive damping in
      // [0.1, 1].  fresh[t]: sig/dsig of target t were evaluated at om[t].
      std::vector<int> next;
      for (int t : act) {
        const int n = tg[t];
        const double f = om[t] - e[n] - sx[n] - E.sig[t] + vx[n];
        const double af = std::fabs(f);
        fresh[t] = 1;
        if (af < p->tol) continue;  // converged at om[t]
        const double fp = 1.0 - E.dsig[t];
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
      ++it;
      if (!next.empty() && it < p->max_iter) return next;
      // Self-energy and slope at the returned energies (targets whose last
      // evaluation was before their final step).
      final_pass = true;
      std::vector<int> stale;
      for (int t = 0; t < ntarget; ++t)
        if (!fresh[t]) stale.push_back(t);
      if (!stale.empty()) return stale;
    }
    for (int t = 0; t < ntarget; ++t) zf[t] = std::min(std::max(1.0 / (1.0 - E.dsig[t]), z_min), z_max);
    return {};
  }
  void finish() {
    const int ntarget = p->ntarget;
    std::vector<double> sxo(ntarget);
    for (int t = 0; t < ntarget; ++t) {
      sxo[t] = E.sx[E.tg[t]];
      QX_REQUIRE(std::isfinite(E.om[t]) && std::isfinite(E.sig[t]), QX_ERR_NUMERICAL,
                 "non-finite CD result for target %d", E.tg[t]);
    }
    QX_CUDA(cudaMemcpy(p->qp, E.om.data(), ntarget * sizeof(double), cudaMemcpyDefault));
    if (p->z) QX_CUDA(cudaMemcpy(p->z, zf.data(), ntarget * sizeof(double), cudaMemcpyDefault));
    if (p->sc) QX_CUDA(cudaMemcpy(p->sc, E.sig.data(), ntarget * sizeof(double), cudaMemcpyDefault));
    if (p->sx) QX_CUDA(cudaMemcpy(p->sx, sxo.data(), ntarget * sizeof(double), cudaMemcpyDefault));
  }
};

// Runs one system on ctx (throws qx::Error): imaginary-axis Wc for the target
// pairs once, then QP steps; each evaluation adds the residues of the poles
// between the target energy and the Fermi level.
void g0w0_cd_run(qx_ctx* ctx, const CdProblem& p) {
  CdRun R;
  R.init(p);
  R.E.ctx = ctx;
  R.E.setup(p.mo_energy, p.lpq, p.targets, p.ntarget, p.nmo, p.nocc, p.naux, p.nw, p.x0, p.precision);
  std::vector<int> act = R.first();
  while (!act.empty()) {
    R.E.evaluate(act);
    act = R.advance(act);
  }
  R.finish();
}

// Worker context of a batch: its own non-blocking stream and workspace, so
// that systems on different workers overlap on the device.
qx_ctx* make_worker(int device) {
  qx_ctx* c = new qx_ctx();
  c->device = device;
  c->worker = true;
  try {
    QX_CUDA(cudaDeviceGetAttribute(&c->sm_count, cudaDevAttrMultiProcessorCount, device));
    QX_CUDA(cudaStreamCreateWithFlags(&c->own_stream, cudaStreamNonBlocking));
    c->stream = c->own_stream;
    for (auto& ev : c->ev) QX_CUDA(cudaEventCreate(&ev));
  } catch (...) {
    qx_ctx_destroy(c);
    throw;
  }
  return c;
}

// Workspace estimate of one system in the grouped batch (bytes): eps of the
// grid and of the residues, the P0 operands (split forms: hi/lo of B_ov and of
// every chi-scaled copy), chi, B_ov^T and the pair tensors of the targets.
static double cd_system_bytes(const qx_cd_system& s, int nw, bool tc) {
  const double ldn = round_up(s.naux, 8), nov = (double)s.nocc * (s.nmo - s.nocc), ldov = round_up((int)nov, 8);
  const double eps = (nw + 2.0 * s.ntarget) * s.naux * ldn * 8.0;
  const double p0 = s.naux * ldov * 8.0 + nw * ldov * 8.0 + (tc ? (1.0 + nw) * s.naux * ldov * 4.0 : 0.0);
  const double pairs = (double)s.ntarget * s.nmo * ldn * (tc ? 16.0 : 8.0) + nw * (double)s.ntarget * s.nmo * 8.0;
  return eps + p0 + nov * ldn * 8.0 + pairs;
}

// Grouped batch.  The systems of a wave advance phase by phase, each on the
// stream of its own worker context (setup, P0, contraction, residue P0 and
// solves), and every inversion of the wave -- the imaginary-axis eps of all
// systems, then at each QP evaluation the real-axis residue eps of all
// systems -- runs as one grouped block sweep on the context stream, so that
// each sweep step is one launch over hundreds of matrices instead of a
// latency-bound launch per system.  Waves hold at most 64 systems and about
// 48 GB of estimated workspace.  Per-system failures are recorded in
// status / msg; a failure of a grouped step throws.
static void cd_batch_grouped(qx_ctx* ctx, qx_cd_system* systems, int nsys, int nw, double x0, double tol,
                             int max_iter, int qp_solver, int precision, std::vector<std::string>& msg) {
  const bool tc = is_tc_precision(precision);
  std::vector<int> order(nsys);
  for (int i = 0; i < nsys; ++i) order[i] = i;
  std::stable_sort(order.begin(), order.end(), [&](int a, int b) {
    return cd_system_bytes(systems[a], nw, tc) > cd_system_bytes(systems[b], nw, tc);
  });
  constexpr double kWaveBytes = 48e9;
  constexpr int kWaveSystems = 64;
  for (int k = 0; k < nsys;) {
    std::vector<int> wave;
    double used = 0.0;
    while (k < nsys && (int)wave.size() < kWaveSystems) {
      const double b = cd_system_bytes(systems[order[k]], nw, tc);
      if (!wave.empty() && used + b > kWaveBytes) break;
      wave.push_back(order[k++]);
      used += b;
    }
    const int W = (int)wave.size();
    while ((int)ctx->workers.size() < W) ctx->workers.push_back(make_worker(ctx->device));
    for (qx_ctx* wk : ctx->workers) {
      wk->p0_form = ctx->p0_form;
      wk->contraction_form = ctx->contraction_form;
    }
    std::vector<CdProblem> probs(W);
    std::vector<CdRun> runs(W);
    std::vector<char> ok(W, 1);
    std::vector<std::vector<int>> act(W);
    auto fail = [&](int j, qx_status st, const char* what) {
      ok[j] = 0;
      systems[wave[j]].status = st;
      msg[wave[j]] = what;
    };
    auto guarded = [&](int j, auto&& f) {
      try {
        f();
      } catch (const Error& ex) {
        fail(j, ex.status, ex.what());
      } catch (const std::exception& ex) {
        fail(j, QX_ERR_INVALID_INPUT, ex.what());
      }
    };
    std::vector<cudaEvent_t> evs(W + 1, nullptr);
    for (auto& e : evs) QX_CUDA(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
    // One grouped inversion on the context stream between the work of the
    // systems in `live` before and after it.
    auto grouped_inversion = [&](const std::vector<int>& live, std::vector<GMat>& mats, int half_lower,
                                 int split_update) {
      for (int j : live) {
        QX_CUDA(cudaEventRecord(evs[j], ctx->workers[j]->stream));
        QX_CUDA(cudaStreamWaitEvent(ctx->stream, evs[j], 0));
      }
      if (!mats.empty()) launch_invert_wc_group(ctx, mats.data(), (int)mats.size(), half_lower, split_update);
      QX_CUDA(cudaEventRecord(evs[W], ctx->stream));
      for (int j : live) QX_CUDA(cudaStreamWaitEvent(ctx->workers[j]->stream, evs[W], 0));
    };
    try {
      // Setup and P0 of every system, then one inversion of all their eps.
      std::vector<GMat> mats;
      std::vector<int> live;
      for (int j = 0; j < W; ++j) {
        qx_cd_system& s = systems[wave[j]];
        qx_ctx* w = ctx->workers[j];
        reset_pending(w);
        w->launches = 0;
        probs[j] = CdProblem{s.mo_energy, s.lpq, s.vxc, s.nmo, s.nocc, s.naux, s.targets, s.ntarget, nw, x0, tol,
                             max_iter, qp_solver, precision, s.qp_energies, s.z_factors, s.sigma_c, s.sigma_x};
        guarded(j, [&] {
          runs[j].init(probs[j]);
          runs[j].E.ctx = w;
          runs[j].E.setup_begin(s.mo_energy, s.lpq, s.targets, s.ntarget, s.nmo, s.nocc, s.naux, nw, x0, precision);
          runs[j].E.eps_matrices(mats);
          live.push_back(j);
        });
      }
      grouped_inversion(live, mats, /*half_lower=*/1, /*split_update=*/tc);
      for (int j : live)
        if (ok[j])
          guarded(j, [&] {
            runs[j].E.setup_end();
            act[j] = runs[j].first();
          });
      // QP evaluations in lockstep; the residue eps of all systems of an
      // evaluation are inverted together (FP64: real axis).
      for (;;) {
        mats.clear();
        live.clear();
        for (int j = 0; j < W; ++j)
          if (ok[j] && !act[j].empty())
            guarded(j, [&] {
              runs[j].E.evaluate_begin(act[j], &mats);
              live.push_back(j);
            });
        if (live.empty()) break;
        // The split trailing update needs SPD matrices: all residue eps of
        // the wave below the smallest transition of their system.
        bool spd = tc;
        for (int j : live) spd = spd && runs[j].E.ev_spd;
        grouped_inversion(live, mats, /*half_lower=*/0, /*split_update=*/spd);
        for (int j : live)
          if (ok[j]) guarded(j, [&] { runs[j].E.evaluate_post(); });
        for (int j : live)
          if (ok[j])
            guarded(j, [&] {
              runs[j].E.evaluate_finish();
              act[j] = runs[j].advance(act[j]);
            });
        sync_and_check(ctx);
      }
      for (int j = 0; j < W; ++j)
        if (ok[j])
          guarded(j, [&] {
            runs[j].finish();
            systems[wave[j]].status = QX_OK;
          });
    } catch (...) {
      for (auto& e : evs) cudaEventDestroy(e);
      throw;
    }
    for (int j = 0; j < W; ++j) ctx->launches += ctx->workers[j]->launches;
    for (auto& e : evs) cudaEventDestroy(e);
  }
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
    // Inputs may have been produced on the caller's stream.
    QX_CUDA(cudaStreamSynchronize(ctx->stream));
    if (nworkers == 0) {
      std::vector<std::string> msg(nsys);
      for (int i = 0; i < nsys; ++i) systems[i].status = QX_ERR_INVALID_INPUT;
      cd_batch_grouped(ctx, systems, nsys, nw, x0, tol, max_iter, qp_solver, precision, msg);
      for (int i = 0; i < nsys; ++i)
        if (systems[i].status != QX_OK)
          throw Error((qx_status)systems[i].status, fmt("system %d: %s", i, msg[i].c_str()));
      ctx->err.clear();
      return QX_OK;
    }
    if (nworkers < 0) nworkers = 4;
    nworkers = std::min(std::min(nworkers, 16), nsys);
    while ((int)ctx->workers.size() < nworkers) ctx->workers.push_back(make_worker(ctx->device));
    for (qx_ctx* wk : ctx->workers) {
      wk->p0_form = ctx->p0_form;
      wk->contraction_form = ctx->contraction_form;
    }
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
