// Device-resident GW system state shared by the AC driver (qx_api.cu) and
// the contour-deformation driver (qx_cd.cu).
#pragma once
#include "qx_internal.cuh"

namespace qx {

// Self-energy grid (correlation_ac.rs:268-302).
struct SigmaGrid {
  std::vector<double> freqs, wts, iw;
};
// Unique unordered MO pairs touched by the target orbitals.
struct PairSet {
  std::vector<int2> pairs;
  std::vector<int> index;  // [norbs][nmo]
};
// Device-resident state of one GW system: pair tensor, B_ov and grids.
struct GWSystem {
  int nmo, nocc, nvir, naux, nov, ldk, ldov, ldn, npair, nw, nws, norbs;
  int precision;
  double *bpt, *bov, *chi, *eps, *v, *sigma;
  double *d_freqs, *d_wts, *d_iw, *d_en;
  int *d_pidx, *d_orbs;
  size_t eps_stride;
  // The rest of the pair gather may still run on the context's side stream
  // (pairs_wait: the event to wait on), and the pair tensor's split forms may
  // still be due; gw_pairs_ready settles both before the first contraction.
  cudaEvent_t pairs_wait = nullptr;
  bool pairs_split_due = false;
  std::vector<int> orbs;
  SigmaGrid grid;
  TcOperand bpt_split{}, wc_split{};
  float* bpt_f32 = nullptr;
  // eps(iw) >= I was certified for the last inversion: eps^-1 has its
  // eigenvalues in (0, 1], so every entry of Wc = eps^-1 - I (and of W') is at
  // most 1 in magnitude, and the split of W' takes 1 as its bound instead of a
  // pass over the matrices.
  bool wc_unit_bound = false;
};

SigmaGrid sigma_grid(int nw, double cutoff, double x0);
PairSet build_pairs(const std::vector<int>& orbs, int nmo);
// host_lpq: d_lpq is host memory read in place over the host link (the
// setup then overlaps part of its gather with the first P0 and inversion).
void gw_setup(qx_ctx* ctx, GWSystem& S, const double* d_lpq, int nmo, int nocc, int naux, const std::vector<int>& orbs,
              int nw, double cutoff, double x0, int precision, bool host_lpq = false);
// Before the first contraction: wait for the rest of the pair gather and
// make the pair tensor's split forms.
void gw_pairs_ready(qx_ctx* ctx, GWSystem& S);
void gw_wc_pairs(qx_ctx* ctx, GWSystem& S, const double* e_host);
// The two halves of gw_wc_pairs around the inversion of S.eps (to W', the
// half-lower Wc): P0 into S.eps, then the pair contraction.
void gw_wc_p0(qx_ctx* ctx, GWSystem& S, const double* e_host);
void gw_wc_contract(qx_ctx* ctx, GWSystem& S);
void gw_sigma(qx_ctx* ctx, GWSystem& S, const double* e_host);
void record_stage(qx_ctx* ctx, int st, bool begin);
void accumulate_stage_times(qx_ctx* ctx);
void validate_common(int nmo, int nocc, int naux);

}  // namespace qx
