// C ABI of libqxgpu: contexts, argument checking, host/device staging and the
// host-side drivers (get_sigma_diag, evGW loop, Pade, exchange).
#include <algorithm>
#include <map>

#include "qx_gw_sys.cuh"
#include "qx_internal.cuh"

#define QX_VERSION "qx-b200 0.1.0 (sm_100a)"

namespace qx {

bool is_device_ptr(const void* p) {
  if (p == nullptr) return false;
  cudaPointerAttributes at;
  cudaError_t e = cudaPointerGetAttributes(&at, p);
  if (e != cudaSuccess) {
    cudaGetLastError();
    return false;
  }
  return at.type == cudaMemoryTypeDevice || at.type == cudaMemoryTypeManaged;
}

const void* device_view(qx_ctx* ctx, int slot, const void* p, size_t bytes) {
  if (is_device_ptr(p)) return p;
  DevBuf& b = ctx->ws[slot];
  b.reserve(bytes);
  QX_CUDA(cudaMemcpyAsync(b.ptr, p, bytes, cudaMemcpyHostToDevice, ctx->stream));
  return b.ptr;
}

const void* mapped_view(qx_ctx* ctx, int slot, const void* p, size_t bytes, bool* in_place) {
  if (in_place) *in_place = false;
  if (p != nullptr) {
    cudaPointerAttributes at;
    if (cudaPointerGetAttributes(&at, p) == cudaSuccess) {
      if (at.type == cudaMemoryTypeDevice || at.type == cudaMemoryTypeManaged) return p;
      if (at.type == cudaMemoryTypeHost && at.devicePointer != nullptr) {
        if (in_place) *in_place = true;
        return at.devicePointer;
      }
    } else {
      cudaGetLastError();
    }
  }
  return device_view(ctx, slot, p, bytes);
}

// Gauss-Legendre rule by Newton iteration on P_n (the nodes and weights of the
// Golub-Welsch eigen-solve, correlation_ac.rs:122-160, to rounding).
void scaled_legendre_roots(int nw, double x0, double* freqs, double* wts) {
  std::vector<double> t(nw), w(nw);
  if (nw == 1) {
    t[0] = 0.0;
    w[0] = 2.0;
  }
  for (int i = 0; i < nw && nw > 1; ++i) {
    double x = std::cos(M_PI * (i + 0.75) / (nw + 0.5));
    double dp = 0.0;
    for (int it = 0; it < 100; ++it) {
      double p0 = 1.0, p1 = x;
      for (int k = 2; k <= nw; ++k) {
        double pk = ((2.0 * k - 1.0) * x * p1 - (k - 1.0) * p0) / k;
        p0 = p1;
        p1 = pk;
      }
      dp = nw * (x * p1 - p0) / (x * x - 1.0);
      double dx = p1 / dp;
      x -= dx;
      if (std::fabs(dx) < 1e-16) break;
    }
    {
      double p0 = 1.0, p1 = x;
      for (int k = 2; k <= nw; ++k) {
        double pk = ((2.0 * k - 1.0) * x * p1 - (k - 1.0) * p0) / k;
        p0 = p1;
        p1 = pk;
      }
      dp = nw * (x * p1 - p0) / (x * x - 1.0);
    }
    t[nw - 1 - i] = x;
    w[nw - 1 - i] = 2.0 / ((1.0 - x * x) * dp * dp);
  }
  for (int i = 0; i < nw; ++i) {
    freqs[i] = x0 * (1.0 + t[i]) / (1.0 - t[i]);
    wts[i] = w[i] * 2.0 * x0 / ((1.0 - t[i]) * (1.0 - t[i]));
  }
}

// Pade sample indices: reference rule (correlation_ac.rs:599-622) or 2k points.
std::vector<int> pade_indices(int nws, int npade) {
  std::vector<int> idx;
  if (npade < 0) {
    std::vector<int> i1, i2;
    for (int i = 1; i < std::min(40, nws); i += 6) i1.push_back(i);
    if (!i1.empty())
      for (int j = i1.back() + 4; j < nws; j += 4) i2.push_back(j);
    idx = i1;
    idx.insert(idx.end(), i2.begin(), i2.end());
    idx.resize((idx.size() / 2) * 2);
  } else {
    QX_REQUIRE(2 * npade + 1 <= nws, QX_ERR_INVALID_INPUT, "[%d/%d] Pade needs %d sigma points, have %d", npade,
               npade, 2 * npade + 1, nws);
    // 2k points spread evenly over indices 1 .. nws-1 (clustered points make
    // the reciprocal differences ill-conditioned).
    const int m = 2 * npade;
    for (int j = 0; j < m; ++j)
      idx.push_back(m == 1 ? 1 : (int)std::floor(1.0 + (double)j * (nws - 2) / (m - 1) + 0.5));
  }
  return idx;
}

SigmaGrid sigma_grid(int nw, double cutoff, double x0) {
  SigmaGrid g;
  g.freqs.resize(nw);
  g.wts.resize(nw);
  scaled_legendre_roots(nw, x0, g.freqs.data(), g.wts.data());
  std::vector<int> idx;
  for (int i = 0; i < nw; ++i)
    if (g.freqs[i] < cutoff) idx.push_back(i);
  int nws = std::min((int)idx.size() + 1, nw + 1);
  g.iw.assign(nws, 0.0);
  for (size_t k = 0; k < idx.size(); ++k)
    if ((int)k + 1 < nws) g.iw[k + 1] = g.freqs[idx[k]];
  return g;
}

PairSet build_pairs(const std::vector<int>& orbs, int nmo) {
  PairSet ps;
  std::vector<int> pid((size_t)nmo * nmo, -1);
  ps.index.resize(orbs.size() * (size_t)nmo);
  for (size_t t = 0; t < orbs.size(); ++t) {
    int n = orbs[t];
    for (int m = 0; m < nmo; ++m) {
      int a = std::min(n, m), b = std::max(n, m);
      int& id = pid[(size_t)a * nmo + b];
      if (id < 0) {
        id = (int)ps.pairs.size();
        ps.pairs.push_back(make_int2(a, b));
      }
      ps.index[t * nmo + m] = id;
    }
  }
  return ps;
}

__global__ void k_to_f32(const double* __restrict__ s, float* __restrict__ d, size_t n) {
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
    d[i] = (float)s[i];
}

void gw_setup(qx_ctx* ctx, GWSystem& S, const double* d_lpq, int nmo, int nocc, int naux, const std::vector<int>& orbs,
              int nw, double cutoff, double x0, int precision, bool host_lpq) {
  S.nmo = nmo;
  S.nocc = nocc;
  S.nvir = nmo - nocc;
  S.naux = naux;
  S.nov = nocc * S.nvir;
  S.ldk = round_up(naux, 8);
  S.ldov = round_up(S.nov, 8);
  S.ldn = round_up(naux, 8);
  S.nw = nw;
  S.precision = precision;
  S.orbs = orbs;
  S.norbs = (int)orbs.size();
  S.grid = sigma_grid(nw, cutoff, x0);
  S.nws = (int)S.grid.iw.size();
  PairSet ps = build_pairs(orbs, nmo);
  S.npair = (int)ps.pairs.size();
  S.eps_stride = (size_t)naux * S.ldn;

  ctx->ws[WS_BPT].reserve((size_t)S.npair * S.ldk * sizeof(double));
  ctx->ws[WS_BOV].reserve((size_t)naux * S.ldov * sizeof(double));
  ctx->ws[WS_CHI].reserve((size_t)nw * S.ldov * sizeof(double));
  ctx->ws[WS_EPS].reserve((size_t)nw * S.eps_stride * sizeof(double));
  const int ldv = S.npair;
  ctx->ws[WS_VPAIR].reserve((size_t)nw * ldv * sizeof(double));
  ctx->ws[WS_SIGMA].reserve(sigma_workspace_doubles(S.norbs, S.nws, nw, nmo) * sizeof(double));
  size_t small = (3 * (size_t)nw + S.nws + nmo + 8) * sizeof(double) + (ps.index.size() + orbs.size()) * sizeof(int) +
                 ps.pairs.size() * sizeof(int2) + 1024;
  ctx->ws[WS_SMALL].reserve(small);
  S.bpt = ctx->ws[WS_BPT].as<double>();
  S.bov = ctx->ws[WS_BOV].as<double>();
  S.chi = ctx->ws[WS_CHI].as<double>();
  S.eps = ctx->ws[WS_EPS].as<double>();
  S.v = ctx->ws[WS_VPAIR].as<double>();
  S.sigma = ctx->ws[WS_SIGMA].as<double>();
  char* sp = ctx->ws[WS_SMALL].as<char>();
  S.d_freqs = reinterpret_cast<double*>(sp);
  S.d_wts = S.d_freqs + nw;
  S.d_iw = S.d_wts + nw;
  S.d_en = S.d_iw + S.nws;
  int2* d_pairs = reinterpret_cast<int2*>(S.d_en + nmo + 8);
  S.d_pidx = reinterpret_cast<int*>(d_pairs + ps.pairs.size());
  S.d_orbs = S.d_pidx + ps.index.size();
  QX_CUDA(cudaMemcpyAsync(S.d_freqs, S.grid.freqs.data(), nw * sizeof(double), cudaMemcpyHostToDevice, ctx->stream));
  QX_CUDA(cudaMemcpyAsync(S.d_wts, S.grid.wts.data(), nw * sizeof(double), cudaMemcpyHostToDevice, ctx->stream));
  QX_CUDA(cudaMemcpyAsync(S.d_iw, S.grid.iw.data(), S.nws * sizeof(double), cudaMemcpyHostToDevice, ctx->stream));
  QX_CUDA(cudaMemcpyAsync(d_pairs, ps.pairs.data(), ps.pairs.size() * sizeof(int2), cudaMemcpyHostToDevice,
                          ctx->stream));
  QX_CUDA(cudaMemcpyAsync(S.d_pidx, ps.index.data(), ps.index.size() * sizeof(int), cudaMemcpyHostToDevice,
                          ctx->stream));
  QX_CUDA(cudaMemcpyAsync(S.d_orbs, orbs.data(), orbs.size() * sizeof(int), cudaMemcpyHostToDevice, ctx->stream));
  // With every orbital a target the pair tensor holds the occupied-virtual
  // block: B_ov comes from it, and the setup reads only lpq's upper triangle.
  bool all_orbitals = S.norbs == nmo;
  for (int t = 0; all_orbitals && t < S.norbs; ++t) all_orbitals = orbs[t] == t;
  // Host lpq read in place with every orbital a target: the pairs of the
  // occupied rows (a < nocc, the first pairs in row-major order) hold B_ov and
  // everything the exchange diagonal reads, so they are gathered first; the
  // rest crosses the host link on the side stream, one block per SM, while the
  // first P0 and inversion run, and the first contraction waits for it.
  const bool overlap = host_lpq && all_orbitals;
  const int npre = overlap ? std::min(S.npair, nocc * nmo - nocc * (nocc - 1) / 2) : S.npair;
  launch_gather_pairs(ctx, ctx->stream, d_lpq, naux, nmo, d_pairs, npre, S.bpt, S.ldk);
  if (all_orbitals)
    launch_ov_from_pairs(ctx, S.bpt, S.ldk, S.d_pidx, naux, nmo, nocc, S.bov, S.ldov);
  else
    launch_gather_ov(ctx, d_lpq, naux, nmo, nocc, S.bov, S.ldov);
  S.pairs_wait = nullptr;
  if (npre < S.npair) {
    if (!ctx->side) {
      QX_CUDA(cudaStreamCreateWithFlags(&ctx->side, cudaStreamNonBlocking));
      for (auto& e : ctx->side_ev) QX_CUDA(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
    }
    QX_CUDA(cudaEventRecord(ctx->side_ev[0], ctx->stream));
    QX_CUDA(cudaStreamWaitEvent(ctx->side, ctx->side_ev[0], 0));
    launch_gather_pairs(ctx, ctx->side, d_lpq, naux, nmo, d_pairs + npre, S.npair - npre,
                        S.bpt + (size_t)npre * S.ldk, S.ldk, ctx->sm_count);
    QX_CUDA(cudaEventRecord(ctx->side_ev[1], ctx->side));
    S.pairs_wait = ctx->side_ev[1];
  }
  S.pairs_split_due = false;
  if (is_tc_precision(precision)) {
    QX_REQUIRE(tc_supported(ctx), QX_ERR_NO_DEVICE, "tensor-core precision needs an sm_100 device");
    const size_t nb = (size_t)S.npair * S.ldk;
    ctx->ws[WS_BPT_HI].reserve(nb * 2);
    ctx->ws[WS_BPT_LO].reserve(nb * 2);
    ctx->ws[WS_BPT_F32].reserve(nb * 4);
    S.bpt_split.hi = ctx->ws[WS_BPT_HI].ptr;
    S.bpt_split.lo = ctx->ws[WS_BPT_LO].ptr;
    S.bpt_f32 = ctx->ws[WS_BPT_F32].as<float>();
    S.pairs_split_due = true;
    const size_t nwc = (size_t)nw * S.eps_stride;
    ctx->ws[WS_WC_HI].reserve(nwc * 2);
    ctx->ws[WS_WC_LO].reserve(nwc * 2);
    S.wc_split.hi = ctx->ws[WS_WC_HI].ptr;
    S.wc_split.lo = ctx->ws[WS_WC_LO].ptr;
  }
  if (!S.pairs_wait) gw_pairs_ready(ctx, S);
}

void gw_pairs_ready(qx_ctx* ctx, GWSystem& S) {
  if (S.pairs_wait) {
    QX_CUDA(cudaStreamWaitEvent(ctx->stream, S.pairs_wait, 0));
    S.pairs_wait = nullptr;
  }
  if (S.pairs_split_due) {
    const int fp16 = S.precision == QX_PREC_FP16X3;
    const size_t nb = (size_t)S.npair * S.ldk;
    launch_split(ctx, S.bpt, S.npair, S.ldk, S.ldk, S.bpt_split.hi, S.bpt_split.lo, S.ldk, 0, 0, 1, fp16, 2,
                 &S.bpt_split.scale);
    k_to_f32<<<1184, 256, 0, ctx->stream>>>(S.bpt, S.bpt_f32, nb);
    check_launch(ctx);
    S.pairs_split_due = false;
  }
}

int* status_words(qx_ctx* ctx, int n) {
  constexpr int kCap = 1 << 16;
  QX_REQUIRE(n > 0 && n <= kCap, QX_ERR_INVALID_INPUT, "%d status words requested", n);
  if (!ctx->status_arena.ptr) ctx->status_arena.reserve(kCap * sizeof(int));
  if (ctx->status_used + n > kCap) sync_and_check(ctx);
  int* p = ctx->status_arena.as<int>() + ctx->status_used;
  ctx->status_used += n;
  return p;
}

void sync_and_check(qx_ctx* ctx) {
  QX_CUDA(cudaStreamSynchronize(ctx->stream));
  ctx->status_used = 0;
  std::vector<qx_ctx::Pending> pend;
  pend.swap(ctx->pending);
  for (const auto& pd : pend) {
    std::vector<int> h(pd.count);
    QX_CUDA(cudaMemcpy(h.data(), pd.dev, pd.count * sizeof(int), cudaMemcpyDeviceToHost));
    for (int i = 0; i < pd.count; ++i) {
      if (!h[i]) continue;
      if (pd.kind == 0)
        throw Error(QX_ERR_CUDA, fmt("tcgen05 GEMM pipeline wait timed out (code %d)", h[i]));
      // Singular eps: the reference substitutes the identity for eps^-1
      // (correlation_ac.rs:390-397); the device already set Wc = 0 there.
      fprintf(stderr, "WARNING: Matrix inversion failed at freq %d: singular eps, using Wc = 0\n", i);
    }
  }
}

void record_stage(qx_ctx* ctx, int st, bool begin) { cudaEventRecord(ctx->ev[2 * st + (begin ? 0 : 1)], ctx->stream); }

void accumulate_stage_times(qx_ctx* ctx) {
  sync_and_check(ctx);
  for (int s = 0; s < QX_ST_COUNT; ++s) {
    float ms = 0.f;
    if (cudaEventElapsedTime(&ms, ctx->ev[2 * s], ctx->ev[2 * s + 1]) == cudaSuccess) ctx->stage_ms[s] += ms;
    cudaGetLastError();
  }
}

// eps(iw) = I - Pi(iw) for the grid of the system (energies e on the host).
void gw_wc_p0(qx_ctx* ctx, GWSystem& S, const double* e_host) {
  QX_CUDA(cudaMemcpyAsync(S.d_en, e_host, S.nmo * sizeof(double), cudaMemcpyHostToDevice, ctx->stream));
  record_stage(ctx, QX_ST_P0, true);
  launch_chi(ctx, S.d_en, S.nocc, S.nvir, S.d_freqs, S.nw, 0, S.chi, S.ldov);
  if (is_tc_precision(S.precision))
    launch_eps_tc(ctx, S.bov, S.ldov, S.naux, S.nov, S.chi, S.nw, S.eps, S.ldn, S.eps_stride,
                  S.precision == QX_PREC_FP16X3);
  else
    launch_eps_fp64(ctx, S.bov, S.ldov, S.naux, S.nov, S.chi, S.nw, S.eps, S.ldn, S.eps_stride);
  record_stage(ctx, QX_ST_P0, false);
}

// v[w][pair] = Wc_nm(iw) of every pair, from S.eps holding W' (half-lower Wc).
void gw_wc_contract(qx_ctx* ctx, GWSystem& S) {
  gw_pairs_ready(ctx, S);
  record_stage(ctx, QX_ST_CONTRACT, true);
  if (is_tc_precision(S.precision)) {
    const int fp16 = S.precision == QX_PREC_FP16X3;
    const unsigned long long* bound = S.wc_unit_bound && fp16 ? split_bound_words(ctx, 0, S.nw, 1.0) : nullptr;
    launch_split(ctx, S.eps, S.naux, S.naux, S.ldn, S.wc_split.hi, S.wc_split.lo, S.ldn, S.eps_stride, S.eps_stride,
                 S.nw, fp16, 0, &S.wc_split.scale, bound);
    launch_pair_contract_tc(ctx, S.bpt_split, S.bpt_f32, S.ldk, S.npair, S.naux, S.wc_split, S.ldn, S.eps_stride, S.nw,
                            S.v, S.npair, fp16);
  } else {
    launch_pair_contract_fp64(ctx, S.bpt, S.ldk, S.npair, S.naux, S.eps, S.ldn, S.eps_stride, S.nw, S.v, S.npair);
  }
  record_stage(ctx, QX_ST_CONTRACT, false);
}

// Wc_nm(iw) for every pair of the system: v[w][pair] (energies e on the host).
void gw_wc_pairs(qx_ctx* ctx, GWSystem& S, const double* e_host) {
  gw_wc_p0(ctx, S, e_host);
  record_stage(ctx, QX_ST_INV, true);
  // Imaginary axis with ordered levels: eps is SPD with eigenvalues in
  // [1, 1 + ||Pi||], so the split trailing update of the sweep keeps Wc within
  // the split forms' error.  Once levels cross, eps may be indefinite and the
  // sweep runs guarded (with the pivoted fallback).
  S.wc_unit_bound = eps_at_least_identity(e_host, S.nocc, S.nvir, 0.0);
  launch_invert_wc(ctx, S.eps, S.naux, S.ldn, S.eps_stride, S.nw, !S.wc_unit_bound, /*half_lower=*/1,
                   /*split_update=*/is_tc_precision(S.precision));
  record_stage(ctx, QX_ST_INV, false);
  gw_wc_contract(ctx, S);
}

// One imaginary-axis Sigma_c evaluation with energies e (host array [nmo]).
void gw_sigma(qx_ctx* ctx, GWSystem& S, const double* e_host) {
  gw_wc_pairs(ctx, S, e_host);
  const double ef = 0.5 * (e_host[S.nocc - 1] + e_host[S.nocc]);
  record_stage(ctx, QX_ST_SIGMA, true);
  launch_sigma_assemble(ctx, S.v, S.npair, S.nw, S.d_pidx, S.norbs, S.nmo, S.d_orbs, S.nocc, S.d_en, ef, S.d_freqs,
                        S.d_wts, S.d_iw, S.nws, S.sigma);
  record_stage(ctx, QX_ST_SIGMA, false);
}

// Host copy of the reference's ConvergenceMonitor DIIS (qp/convergence.rs:146-330).
struct Diis {
  int max_vectors;  // <= 0: disabled
  std::vector<std::vector<double>> ehist, zhist, vecs, errs;
  void check(const std::vector<double>& e, const std::vector<double>& z) {
    ehist.push_back(e);
    zhist.push_back(z);
    if (ehist.size() > 1 && max_vectors > 0)
      while ((int)ehist.size() > max_vectors) {
        ehist.erase(ehist.begin());
        zhist.erase(zhist.begin());
      }
  }
  // Returns false when the reference would return an error.
  bool accelerate(const std::vector<double>& e, const std::vector<double>& z, std::vector<double>& eo,
                  std::vector<double>& zo) {
    const size_t n = e.size();
    if (max_vectors <= 0 || ehist.empty()) {
      eo = e;
      zo = z;
      return true;
    }
    std::vector<double> err(n), comb(2 * n);
    for (size_t i = 0; i < n; ++i) err[i] = e[i] - ehist.back()[i];
    for (size_t i = 0; i < n; ++i) {
      comb[i] = e[i];
      comb[n + i] = z[i];
    }
    vecs.push_back(comb);
    errs.push_back(err);
    while ((int)vecs.size() > max_vectors) {
      vecs.erase(vecs.begin());
      errs.erase(errs.begin());
    }
    const int nv = (int)vecs.size();
    if (nv < 2) {
      eo = e;
      zo = z;
      return true;
    }
    const int N = nv + 1;
    std::vector<double> aug((size_t)N * (N + 1), 0.0);
    auto A = [&](int i, int j) -> double& { return aug[(size_t)i * (N + 1) + j]; };
    for (int i = 0; i < nv; ++i) {
      for (int j = 0; j <= i; ++j) {
        double d = 0;
        for (size_t k = 0; k < n; ++k) d += errs[i][k] * errs[j][k];
        A(i, j) = d;
        A(j, i) = d;
      }
      A(i, nv) = -1.0;
      A(nv, i) = -1.0;
    }
    A(nv, N) = -1.0;
    double maxe = 0;
    for (int i = 0; i < N; ++i)
      for (int j = 0; j < N; ++j) maxe = std::max(maxe, std::fabs(A(i, j)));
    const double tol = 1e-12 * std::max(maxe, 1.0);
    for (int i = 0; i < N - 1; ++i) {
      int mr = i;
      double mv = std::fabs(A(i, i));
      for (int k = i + 1; k < N; ++k)
        if (std::fabs(A(k, i)) > mv) {
          mv = std::fabs(A(k, i));
          mr = k;
        }
      if (mv < tol) return false;
      if (mr != i)
        for (int j = 0; j <= N; ++j) std::swap(A(i, j), A(mr, j));
      double piv = A(i, i);
      for (int k = i + 1; k < N; ++k)
        if (std::fabs(A(k, i)) > 1e-10 * std::fabs(piv)) {
          double f = A(k, i) / piv;
          for (int j = i; j <= N; ++j) A(k, j) -= f * A(i, j);
        }
    }
    if (std::fabs(A(N - 1, N - 1)) < tol) return false;
    std::vector<double> x(N);
    for (int i = N - 1; i >= 0; --i) {
      double s = A(i, N);
      for (int j = i + 1; j < N; ++j) s -= A(i, j) * x[j];
      if (std::fabs(A(i, i)) < tol) return false;
      x[i] = s / A(i, i);
    }
    double cs = 0;
    for (int i = 0; i < N - 1; ++i) cs += x[i];
    if (std::fabs(cs - 1.0) > 0.5) return false;
    for (double v : x)
      if (!std::isfinite(v)) return false;
    std::vector<double> r(2 * n, 0.0);
    for (int i = 0; i < nv; ++i)
      for (size_t k = 0; k < 2 * n; ++k) r[k] += x[i] * vecs[i][k];
    eo.assign(r.begin(), r.begin() + n);
    zo.assign(r.begin() + n, r.end());
    return true;
  }
};

void convergence_window(const double* e, int nmo, int nocc, const qx_evgw_config& c, int& s, int& en) {
  if (!c.frontier_convergence) {
    s = 0;
    en = nmo;
    return;
  }
  const double w = c.frontier_window;
  const double homo = e[nocc - 1];
  s = std::max(nocc - 1, 0);
  for (int i = nocc - 1; i >= 0; --i) {
    if (e[i] >= homo - w) s = i;
    else break;
  }
  const double lumo = e[nocc];
  en = nocc + 1;
  for (int i = nocc; i < nmo; ++i) {
    if (e[i] <= lumo + w) en = i + 1;
    else break;
  }
}

bool eps_at_least_identity(const double* energies, int nocc, int nvir, double wmax) {
  double homo = -INFINITY, lumo = INFINITY;
  for (int i = 0; i < nocc + nvir; ++i)
    if (!std::isfinite(energies[i])) return false;
  for (int i = 0; i < nocc; ++i) homo = std::max(homo, energies[i]);
  for (int a = 0; a < nvir; ++a) lumo = std::min(lumo, energies[nocc + a]);
  const double gap = lumo - homo;
  return std::isfinite(gap) && gap > 0.0 && gap > std::fabs(wmax);
}

void validate_common(int nmo, int nocc, int naux) {
  QX_REQUIRE(nmo > 0 && naux > 0, QX_ERR_INVALID_INPUT, "nmo=%d naux=%d must be positive", nmo, naux);
  QX_REQUIRE(nocc >= 1 && nocc < nmo, QX_ERR_INVALID_INPUT, "Invalid nocc=%d: must be in range [1, %d)", nocc, nmo);
}

}  // namespace qx

using namespace qx;

// A call that fails may leave setup work on the side stream reading the
// caller's host arrays: it ends before the call returns.
static void settle_side(qx_ctx* ctx) {
  if (ctx && ctx->side) cudaStreamSynchronize(ctx->side);
}

template <class F>
static qx_status guarded(qx_ctx* ctx, F&& f) {
  try {
    if (ctx) {
      reset_pending(ctx);
      ctx->launches = 0;
      for (double& v : ctx->stage_ms) v = 0.0;
      QX_CUDA(cudaSetDevice(ctx->device));
    }
    f();
    if (ctx) ctx->err.clear();
    return QX_OK;
  } catch (const Error& e) {
    settle_side(ctx);
    if (ctx) ctx->err = e.what();
    return e.status;
  } catch (const std::bad_alloc&) {
    settle_side(ctx);
    if (ctx) ctx->err = "host allocation failed";
    return QX_ERR_CUDA;
  } catch (const std::exception& e) {
    settle_side(ctx);
    if (ctx) ctx->err = e.what();
    return QX_ERR_INVALID_INPUT;
  }
}

extern "C" {

const char* qx_version(void) { return QX_VERSION; }

qx_status qx_ctx_create(qx_ctx** out, int device) {
  if (!out) return QX_ERR_INVALID_INPUT;
  *out = nullptr;
  int n = 0;
  if (cudaGetDeviceCount(&n) != cudaSuccess || n == 0) {
    cudaGetLastError();
    return QX_ERR_NO_DEVICE;
  }
  if (device < 0 || device >= n) return QX_ERR_NO_DEVICE;
  qx_ctx* c = new qx_ctx();
  c->device = device;
  qx_status st = guarded(c, [&] {
    cudaDeviceProp p;
    QX_CUDA(cudaGetDeviceProperties(&p, device));
    QX_REQUIRE(p.major >= 10, QX_ERR_NO_DEVICE, "device %d is sm_%d%d; this library is built for sm_100a", device,
               p.major, p.minor);
    c->sm_count = p.multiProcessorCount;
    // A blocking stream: it orders after work the caller queued on the legacy
    // default stream (e.g. a framework's host-to-device copy of an input).
    QX_CUDA(cudaStreamCreateWithFlags(&c->own_stream, cudaStreamDefault));
    c->stream = c->own_stream;
    for (auto& e : c->ev) QX_CUDA(cudaEventCreate(&e));
  });
  if (st != QX_OK) {
    fprintf(stderr, "qx_ctx_create: %s\n", c->err.c_str());
    delete c;
    return st;
  }
  *out = c;
  return QX_OK;
}

qx_status qx_ctx_destroy(qx_ctx* c) {
  if (!c) return QX_OK;
  for (qx_ctx* w : c->workers) qx_ctx_destroy(w);
  c->workers.clear();
  cudaSetDevice(c->device);
  if (c->stream) cudaStreamSynchronize(c->stream);
  for (auto& e : c->sweep_ev)
    if (e) cudaEventDestroy(e);
  if (c->sweep_hi) cudaStreamDestroy(c->sweep_hi);
  if (c->sweep_lo) cudaStreamDestroy(c->sweep_lo);
  if (c->side) cudaStreamSynchronize(c->side);
  for (auto& e : c->side_ev)
    if (e) cudaEventDestroy(e);
  if (c->side) cudaStreamDestroy(c->side);
  for (auto& e : c->ev)
    if (e) cudaEventDestroy(e);
  if (c->own_stream) cudaStreamDestroy(c->own_stream);
  delete c;
  return QX_OK;
}

const char* qx_last_error(const qx_ctx* c) { return c ? c->err.c_str() : "null context"; }

qx_status qx_ctx_set_stream(qx_ctx* c, void* stream) {
  if (!c) return QX_ERR_INVALID_INPUT;
  c->stream = stream ? reinterpret_cast<cudaStream_t>(stream) : c->own_stream;
  return QX_OK;
}

qx_status qx_ctx_set_contraction_form(qx_ctx* c, int form) {
  if (!c || form < QX_CONTRACT_AUTO || form > QX_CONTRACT_PAIR) return QX_ERR_INVALID_INPUT;
  c->contraction_form = form;
  for (qx_ctx* w : c->workers) w->contraction_form = form;
  return QX_OK;
}

qx_status qx_ctx_set_p0_form(qx_ctx* c, int form) {
  if (!c || form < QX_P0_AUTO || form > QX_P0_PAIR) return QX_ERR_INVALID_INPUT;
  c->p0_form = form;
  for (qx_ctx* w : c->workers) w->p0_form = form;
  return QX_OK;
}

qx_status qx_ctx_last_timings(const qx_ctx* c, double* a, double* b, double* d, double* e, double* f) {
  if (!c) return QX_ERR_INVALID_INPUT;
  if (a) *a = c->stage_ms[QX_ST_P0];
  if (b) *b = c->stage_ms[QX_ST_INV];
  if (d) *d = c->stage_ms[QX_ST_CONTRACT];
  if (e) *e = c->stage_ms[QX_ST_SIGMA];
  if (f) *f = c->stage_ms[QX_ST_QP];
  return QX_OK;
}

int64_t qx_ctx_last_launches(const qx_ctx* c) { return c ? c->launches : 0; }

qx_status qx_ctx_last_guard_stats(const qx_ctx* c, int64_t* guarded, int64_t* reinverted) {
  if (!c) return QX_ERR_INVALID_INPUT;
  int64_t g = c->guard_matrices, r = c->guard_reinverted;
  for (const qx_ctx* w : c->workers) {
    g += w->guard_matrices;
    r += w->guard_reinverted;
  }
  if (guarded) *guarded = g;
  if (reinverted) *reinverted = r;
  return QX_OK;
}

qx_status qx_get_scaled_legendre_roots(int nw, double x0, double* freqs, double* wts) {
  if (nw < 0 || (nw > 0 && (!freqs || !wts))) return QX_ERR_INVALID_INPUT;
  if (nw == 0) return QX_OK;
  scaled_legendre_roots(nw, x0, freqs, wts);
  return QX_OK;
}

void qx_evgw_config_default(qx_evgw_config* c) {
  c->max_iterations = 12;
  c->energy_tolerance = 1e-4;
  c->damping_factor = 0.5;
  c->z_min = 0.1;
  c->z_max = 0.999;
  c->use_diis = 1;
  c->diis_space_dim = 6;
  c->frontier_convergence = 1;
  c->frontier_window = 1.0;
  c->nfreq = 100;
  c->iw_cutoff = 5.0;
  c->x0 = 0.5;
  c->use_solved_qp = 0;
  c->newton_energy_tolerance = 1e-8;
  c->newton_max_iterations = 50;
  c->npade = -1;
  c->precision = QX_PREC_FP64;
  c->fixed_iterations = 0;
}

qx_status qx_get_rho_response(qx_ctx* ctx, int nfreq, const double* freqs, const double* mo_energy,
                              const double* lpq_ov, int naux, int nocc, int nvir, int precision, double* pi) {
  return guarded(ctx, [&] {
    QX_REQUIRE(ctx && nfreq > 0 && naux > 0 && nocc > 0 && nvir > 0 && freqs && mo_energy && lpq_ov && pi,
               QX_ERR_INVALID_INPUT, "invalid arguments to get_rho_response");
    const int nov = nocc * nvir, ldov = round_up(nov, 8), ldn = round_up(naux, 8);
    const double* d_lov = (const double*)device_view(ctx, WS_LPQ, lpq_ov, (size_t)naux * nov * sizeof(double));
    ctx->ws[WS_SMALL].reserve((nfreq + nocc + nvir) * sizeof(double));
    double* d_f = ctx->ws[WS_SMALL].as<double>();
    double* d_e = d_f + nfreq;
    QX_CUDA(cudaMemcpyAsync(d_f, freqs, nfreq * sizeof(double), cudaMemcpyDefault, ctx->stream));
    QX_CUDA(cudaMemcpyAsync(d_e, mo_energy, (nocc + nvir) * sizeof(double), cudaMemcpyDefault, ctx->stream));
    ctx->ws[WS_BOV].reserve((size_t)naux * ldov * sizeof(double));
    double* bov = ctx->ws[WS_BOV].as<double>();
    // lpq_ov [naux][nocc][nvir] is already B_ov rows; re-pitch to ldov.
    QX_CUDA(cudaMemcpy2DAsync(bov, ldov * sizeof(double), d_lov, nov * sizeof(double), nov * sizeof(double), naux,
                              cudaMemcpyDeviceToDevice, ctx->stream));
    if (ldov > nov)
      QX_CUDA(cudaMemset2DAsync(bov + nov, ldov * sizeof(double), 0, (ldov - nov) * sizeof(double), naux, ctx->stream));
    ctx->ws[WS_CHI].reserve((size_t)nfreq * ldov * sizeof(double));
    double* chi = ctx->ws[WS_CHI].as<double>();
    const size_t stride = (size_t)naux * ldn;
    ctx->ws[WS_EPS].reserve((size_t)nfreq * stride * sizeof(double));
    double* eps = ctx->ws[WS_EPS].as<double>();
    launch_chi(ctx, d_e, nocc, nvir, d_f, nfreq, 0, chi, ldov);
    if (is_tc_precision(precision))
      launch_eps_tc(ctx, bov, ldov, naux, nov, chi, nfreq, eps, ldn, stride, precision == QX_PREC_FP16X3);
    else launch_eps_fp64(ctx, bov, ldov, naux, nov, chi, nfreq, eps, ldn, stride);
    // Pi = I - eps.
    std::vector<double> h((size_t)nfreq * stride);
    QX_CUDA(cudaMemcpyAsync(h.data(), eps, h.size() * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
    sync_and_check(ctx);
    std::vector<double> out((size_t)nfreq * naux * naux);
    for (int w = 0; w < nfreq; ++w)
      for (int r = 0; r < naux; ++r)
        for (int c = 0; c < naux; ++c)
          out[((size_t)w * naux + r) * naux + c] = (r == c ? 1.0 : 0.0) - h[w * stride + (size_t)r * ldn + c];
    QX_CUDA(cudaMemcpy(pi, out.data(), out.size() * sizeof(double), cudaMemcpyDefault));
  });
}

int qx_eps_at_least_identity(const double* mo_energy, int nocc, int nvir, double wmax) {
  if (!mo_energy || nocc <= 0 || nvir <= 0) return 0;
  return eps_at_least_identity(mo_energy, nocc, nvir, wmax) ? 1 : 0;
}

qx_status qx_screened_interaction(qx_ctx* ctx, int nfreq, int naux, const double* pi, double* wc) {
  return guarded(ctx, [&] {
    QX_REQUIRE(ctx && nfreq > 0 && naux > 0 && pi && wc, QX_ERR_INVALID_INPUT, "invalid arguments");
    const int ldn = round_up(naux, 8);
    const size_t stride = (size_t)naux * ldn;
    std::vector<double> hp((size_t)nfreq * naux * naux);
    QX_CUDA(cudaMemcpy(hp.data(), pi, hp.size() * sizeof(double), cudaMemcpyDefault));
    std::vector<double> he((size_t)nfreq * stride, 0.0);
    for (int w = 0; w < nfreq; ++w)
      for (int r = 0; r < naux; ++r)
        for (int c = 0; c < naux; ++c)
          he[w * stride + (size_t)r * ldn + c] = (r == c ? 1.0 : 0.0) - hp[((size_t)w * naux + r) * naux + c];
    ctx->ws[WS_EPS].reserve(he.size() * sizeof(double));
    double* eps = ctx->ws[WS_EPS].as<double>();
    QX_CUDA(cudaMemcpyAsync(eps, he.data(), he.size() * sizeof(double), cudaMemcpyHostToDevice, ctx->stream));
    // Pi comes from the caller: eps >= I cannot be assumed.
    launch_invert_wc(ctx, eps, naux, ldn, stride, nfreq, /*guard=*/1);
    QX_CUDA(cudaMemcpyAsync(he.data(), eps, he.size() * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
    sync_and_check(ctx);
    for (int w = 0; w < nfreq; ++w)
      for (int r = 0; r < naux; ++r)
        for (int c = 0; c < naux; ++c) hp[((size_t)w * naux + r) * naux + c] = he[w * stride + (size_t)r * ldn + c];
    QX_CUDA(cudaMemcpy(wc, hp.data(), hp.size() * sizeof(double), cudaMemcpyDefault));
  });
}

qx_status qx_get_sigma_diag(qx_ctx* ctx, const double* mo_energy, const double* lpq, const int* orbs, int norbs, int nmo,
                            int nocc, int naux, int nw, double iw_cutoff, double x0, int precision, double* sigma,
                            double* omega, int nw_sigma_max, int* nw_sigma) {
  return guarded(ctx, [&] {
    QX_REQUIRE(ctx && mo_energy && lpq && orbs && sigma && omega && nw_sigma, QX_ERR_INVALID_INPUT, "null argument");
    validate_common(nmo, nocc, naux);
    QX_REQUIRE(nw > 0 && norbs > 0, QX_ERR_INVALID_INPUT, "nw=%d norbs=%d must be positive", nw, norbs);
    std::vector<int> o(norbs);
    QX_CUDA(cudaMemcpy(o.data(), orbs, norbs * sizeof(int), cudaMemcpyDefault));
    for (int v : o) QX_REQUIRE(v >= 0 && v < nmo, QX_ERR_INVALID_INPUT, "orbital index %d out of range", v);
    std::vector<double> e(nmo);
    QX_CUDA(cudaMemcpy(e.data(), mo_energy, nmo * sizeof(double), cudaMemcpyDefault));
    // Page-locked host lpq is read in place by the setup gathers (only the
    // pairs they need cross the host link).
    const double* d_lpq = (const double*)mapped_view(ctx, WS_LPQ, lpq, (size_t)naux * nmo * nmo * sizeof(double));
    GWSystem S;
    gw_setup(ctx, S, d_lpq, nmo, nocc, naux, o, nw, iw_cutoff, x0, precision);
    QX_REQUIRE(nw_sigma_max >= S.nws, QX_ERR_INVALID_INPUT, "nw_sigma_max %d < %d", nw_sigma_max, S.nws);
    gw_sigma(ctx, S, e.data());
    std::vector<double> hs((size_t)norbs * S.nws * 2);
    QX_CUDA(cudaMemcpyAsync(hs.data(), S.sigma, hs.size() * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
    accumulate_stage_times(ctx);
    std::vector<double> out((size_t)norbs * nw_sigma_max * 2, 0.0), om((size_t)norbs * nw_sigma_max * 2, 0.0);
    for (int t = 0; t < norbs; ++t) {
      const double s = o[t] < nocc ? -1.0 : 1.0;
      for (int k = 0; k < S.nws; ++k) {
        out[((size_t)t * nw_sigma_max + k) * 2] = hs[((size_t)t * S.nws + k) * 2];
        out[((size_t)t * nw_sigma_max + k) * 2 + 1] = hs[((size_t)t * S.nws + k) * 2 + 1];
        om[((size_t)t * nw_sigma_max + k) * 2 + 1] = s * S.grid.iw[k];
      }
    }
    for (double v : out) QX_REQUIRE(std::isfinite(v), QX_ERR_NUMERICAL, "Sigma_c contains NaN or Inf");
    QX_CUDA(cudaMemcpy(sigma, out.data(), out.size() * sizeof(double), cudaMemcpyDefault));
    QX_CUDA(cudaMemcpy(omega, om.data(), om.size() * sizeof(double), cudaMemcpyDefault));
    *nw_sigma = S.nws;
  });
}

qx_status qx_compute_exchange_diag(qx_ctx* ctx, const double* lpq, int naux, int nmo, int nocc, double* sigma_x) {
  return guarded(ctx, [&] {
    QX_REQUIRE(ctx && lpq && sigma_x, QX_ERR_INVALID_INPUT, "null argument");
    validate_common(nmo, nocc, naux);
    const double* d_lpq = (const double*)device_view(ctx, WS_LPQ, lpq, (size_t)naux * nmo * nmo * sizeof(double));
    ctx->ws[WS_QPOUT].reserve(nmo * sizeof(double));
    double* d = ctx->ws[WS_QPOUT].as<double>();
    launch_exchange_diag(ctx, d_lpq, naux, nmo, nocc, d);
    QX_CUDA(cudaMemcpyAsync(sigma_x, d, nmo * sizeof(double), cudaMemcpyDefault, ctx->stream));
    sync_and_check(ctx);
  });
}

qx_status qx_evgw(qx_ctx* ctx, const double* mo_energy, const double* lpq, const double* vxc, int nmo, int nocc,
                  int naux, const qx_evgw_config* cfgp, qx_evgw_result* res) {
  return guarded(ctx, [&] {
    QX_REQUIRE(ctx && mo_energy && lpq && vxc && cfgp && res && res->qp_energies && res->z_factors,
               QX_ERR_INVALID_INPUT, "null argument");
    validate_common(nmo, nocc, naux);
    const qx_evgw_config cfg = *cfgp;
    QX_REQUIRE(cfg.nfreq > 0 && cfg.max_iterations > 0, QX_ERR_INVALID_INPUT, "nfreq and max_iterations must be > 0");
    std::vector<double> e0(nmo), vx(nmo);
    QX_CUDA(cudaMemcpy(e0.data(), mo_energy, nmo * sizeof(double), cudaMemcpyDefault));
    QX_CUDA(cudaMemcpy(vx.data(), vxc, nmo * sizeof(double), cudaMemcpyDefault));
    // Page-locked host lpq is read in place: the setup gathers its upper
    // triangle (the pairs p <= q) straight into the pair tensor, and nothing
    // reads it afterwards, so half of it crosses the host link.
    bool in_place = false;
    const double* d_lpq =
        (const double*)mapped_view(ctx, WS_LPQ, lpq, (size_t)naux * nmo * nmo * sizeof(double), &in_place);
    std::vector<int> orbs(nmo);
    for (int i = 0; i < nmo; ++i) orbs[i] = i;
    GWSystem S;
    gw_setup(ctx, S, d_lpq, nmo, nocc, naux, orbs, cfg.nfreq, cfg.iw_cutoff, cfg.x0, cfg.precision,
             /*host_lpq=*/in_place);
    std::vector<int> fit = pade_indices(S.nws, cfg.npade);
    const int nfit = (int)fit.size();
    QX_REQUIRE(nfit > 0, QX_ERR_INVALID_INPUT, "not enough sigma points for a Pade fit (nw_sigma=%d)", S.nws);
    // QP buffers: fit idx, mo_energy, eval energies, sigma_x, vxc, coeff, outputs.
    DevBuf& qb = ctx->ws[WS_QPOUT];
    qb.reserve((size_t)(6 * nmo + 2 * nfit * nmo + 2 * nmo + 64) * sizeof(double) + nfit * sizeof(int));
    double* d_mo = qb.as<double>();
    double* d_ev = d_mo + nmo;
    double* d_sx = d_ev + nmo;
    double* d_vx = d_sx + nmo;
    double* d_qp = d_vx + nmo;
    double* d_z = d_qp + nmo;
    double* d_sc = d_z + nmo;
    double* d_coeff = d_sc + 2 * nmo;
    int* d_fit = reinterpret_cast<int*>(d_coeff + 2 * (size_t)nfit * nmo);
    QX_CUDA(cudaMemcpyAsync(d_mo, e0.data(), nmo * sizeof(double), cudaMemcpyHostToDevice, ctx->stream));
    QX_CUDA(cudaMemcpyAsync(d_vx, vx.data(), nmo * sizeof(double), cudaMemcpyHostToDevice, ctx->stream));
    QX_CUDA(cudaMemcpyAsync(d_fit, fit.data(), nfit * sizeof(int), cudaMemcpyHostToDevice, ctx->stream));
    launch_exchange_pairs(ctx, S.bpt, S.ldk, S.d_pidx, naux, nmo, nocc, nmo, d_sx);
    std::vector<double> sx(nmo);
    QX_CUDA(cudaMemcpyAsync(sx.data(), d_sx, nmo * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));

    const double ef = 0.5 * (e0[nocc - 1] + e0[nocc]);
    std::vector<double> qp = e0, z(nmo, 1.0), nqp(nmo), nz(nmo), sc(2 * nmo, 0.0);
    Diis diis;
    diis.max_vectors = cfg.use_diis ? cfg.diis_space_dim : 0;
    const int iters = cfg.fixed_iterations > 0 ? cfg.fixed_iterations : cfg.max_iterations;
    int done = 0;
    bool converged = false;
    for (int it = 0; it < iters; ++it) {
      std::vector<double> qold = qp;
      const std::vector<double>& ep0 = (it == 0) ? e0 : qold;
      gw_sigma(ctx, S, ep0.data());
      QX_CUDA(cudaMemcpyAsync(d_ev, ep0.data(), nmo * sizeof(double), cudaMemcpyHostToDevice, ctx->stream));
      QPParams p{};
      p.norbs = nmo;
      p.nws = S.nws;
      p.nfit = nfit;
      p.fit_idx = d_fit;
      p.sigma = S.sigma;
      p.iw = S.d_iw;
      p.orbs = S.d_orbs;
      p.nocc = nocc;
      p.mo_energy = d_mo;
      p.eval_energy = d_ev;
      p.sigma_x = d_sx;
      p.vxc = d_vx;
      p.ef = ef;
      p.z_min = cfg.z_min;
      p.z_max = cfg.z_max;
      p.solved = cfg.use_solved_qp;
      p.first_iteration = (it == 0);
      p.newton_tol = cfg.newton_energy_tolerance;
      p.newton_max_iter = cfg.newton_max_iterations;
      p.coeff = d_coeff;
      p.qp_out = d_qp;
      p.z_out = d_z;
      p.sc_out = d_sc;
      record_stage(ctx, QX_ST_QP, true);
      launch_pade_qp(ctx, p);
      record_stage(ctx, QX_ST_QP, false);
      QX_CUDA(cudaMemcpyAsync(nqp.data(), d_qp, nmo * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
      QX_CUDA(cudaMemcpyAsync(nz.data(), d_z, nmo * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
      QX_CUDA(cudaMemcpyAsync(sc.data(), d_sc, 2 * nmo * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
      accumulate_stage_times(ctx);
      for (int i = 0; i < nmo; ++i)
        QX_REQUIRE(std::isfinite(nqp[i]) && std::isfinite(nz[i]), QX_ERR_NUMERICAL,
                   "non-finite QP energy for orbital %d at iteration %d", i, it);
      // Mixing (qp/evgw.rs:832-927).
      const double d = cfg.damping_factor;
      auto damp = [&] {
        for (int i = 0; i < nmo; ++i) {
          qp[i] = (1.0 - d) * qold[i] + d * nqp[i];
          z[i] = (1.0 - d) * z[i] + d * nz[i];
        }
      };
      if (it == 0) {
        qp = nqp;
        z = nz;
        diis.check(qp, z);
      } else if (it == 1) {
        damp();
        diis.check(qp, z);
      } else if (cfg.use_diis) {
        diis.check(nqp, nz);
        std::vector<double> de, dz;
        bool ok = diis.accelerate(nqp, nz, de, dz);
        if (ok) {
          double me = 0, mz = 0;
          for (int i = 0; i < nmo; ++i) {
            me = std::max(me, std::fabs(de[i] - nqp[i]));
            mz = std::max(mz, std::fabs(dz[i] - nz[i]));
          }
          if (me < 0.5 && mz < 0.2) {
            qp = de;
            z = dz;
          } else {
            damp();
          }
        } else {
          damp();
        }
        for (int i = 0; i < nmo; ++i) z[i] = std::min(std::max(z[i], cfg.z_min), cfg.z_max);
      } else {
        damp();
      }
      int cs, ce;
      convergence_window(e0.data(), nmo, nocc, cfg, cs, ce);
      double mx = 0, ss = 0;
      for (int i = cs; i < ce; ++i) {
        double dd = std::fabs(qp[i] - qold[i]);
        mx = std::max(mx, dd);
        ss += dd * dd;
      }
      if (res->history_energies)
        std::copy(qp.begin(), qp.end(), res->history_energies + (size_t)it * nmo);
      if (res->history_max_change) res->history_max_change[it] = mx;
      if (res->history_rms_change) res->history_rms_change[it] = std::sqrt(ss / (ce - cs));
      done = it + 1;
      if (cfg.fixed_iterations <= 0 && mx < cfg.energy_tolerance) {
        converged = true;
        break;
      }
    }
    std::copy(qp.begin(), qp.end(), res->qp_energies);
    std::copy(z.begin(), z.end(), res->z_factors);
    if (res->sigma_x) std::copy(sx.begin(), sx.end(), res->sigma_x);
    if (res->sigma_c) std::copy(sc.begin(), sc.end(), res->sigma_c);
    res->n_iterations = done;
    res->converged = converged ? 1 : 0;
  });
}

}  // extern "C"
