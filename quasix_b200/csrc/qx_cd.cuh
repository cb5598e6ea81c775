// Contour-deformation G0W0 engine shared by the forward driver (qx_cd.cu)
// and the adjoint (qx_grad.cu).
#pragma once
#include "qx_blas.cuh"
#include "qx_gw_sys.cuh"
#include "qx_internal.cuh"

namespace qx {

// One residue of target t: Wc_{n_t m}(w) enters Sigma_n with sign sgn, at the
// real shift w = sgn (E_t - e_m) (occupied m above E_t: sgn = -1; virtual m
// below E_t: sgn = +1).
struct CdResidue {
  int t, m;
  double sgn, w;
};

// Device buffers of one chunk of residues (rc <= the chunk capacity).
struct CdResidueChunk {
  double* eps;  // [rc][naux][ldn]: eps(w_r), then Wc(w_r) = eps^-1 - I
  double* b;    // [rc][ldn]: b_r = lpq[:, n_t, m]
  double* x;    // [rc][ldn]: eps(w_r)^-1 b_r
  double* y;    // [rc][ldn]: refinement: the residual b - eps x
  double* dx;   // [rc][ldn]: refinement: its correction eps^-1 (b - eps x)
  double* tm;   // [rc][ldov]: B_ov^T x_r
  double* chi;  // [rc][ldov]: real-axis chi'(w_r)
  double* wr;   // [rc]
  double* val;  // [rc]: Wc_r = b^T Wc(w_r) b
  double* dv;   // [rc]: dWc_r/dw
  int2* nm;     // [rc]
  int cap;
};

struct CdEngine {
  qx_ctx* ctx = nullptr;
  int nmo = 0, nocc = 0, nvir = 0, naux = 0, nov = 0, ldn = 0, ntarget = 0, nw = 0, precision = 0;
  bool tc = false;
  std::vector<double> e, sx, om, sig, dsig;
  std::vector<int> tg;
  const double* d_lpq = nullptr;
  GWSystem S;
  double* bovT = nullptr;   // [nov][ldn]
  double* d_om = nullptr;   // [ntarget]
  double* d_imag = nullptr; // [ntarget][2]

  // Copies the inputs, builds the imaginary-axis Wc_nm(i f_k) of the target
  // pairs, Sigma_x and B_ov^T.  om starts at the mean-field energies.
  void setup(const double* mo_energy, const double* lpq, const int* targets, int ntarget, int nmo, int nocc,
             int naux, int nw, double x0, int precision);
  // setup in two halves around the inversion of the nw eps(i f_k) (to W',
  // half-lower), for a caller that inverts the matrices of many systems at
  // once: setup_begin ends with eps on the device (eps_matrices lists them),
  // setup_end runs on the inverted matrices.
  void setup_begin(const double* mo_energy, const double* lpq, const int* targets, int ntarget, int nmo, int nocc,
                   int naux, int nw, double x0, int precision);
  void eps_matrices(std::vector<GMat>& out) const;
  void setup_end();
  // Residues of the targets in act at their current om.
  std::vector<CdResidue> residues(const std::vector<int>& act) const;
  // Buffers for chunks of up to the returned capacity (~2 GB of eps).
  CdResidueChunk residue_buffers(int R);
  // Wc, x, B_ov^T x and dWc/dw for residues list[0..rc) (device, async):
  // residue_p0 (eps(w_r)), the FP64 inversion, residue_post (the rest).
  void residue_compute(CdResidueChunk& c, const CdResidue* list, int rc);
  void residue_p0(CdResidueChunk& c, const CdResidue* list, int rc);
  // refine: one step of iterative refinement of the solves (eps not
  // certified >= I: guarded, possibly pivoted, possibly ill-conditioned).
  void residue_post(CdResidueChunk& c, int rc, bool refine);
  // sig/dsig of the targets in act at om (synchronises).
  void evaluate(const std::vector<int>& act);
  // evaluate in two halves.  With group given and the residues in one chunk,
  // evaluate_begin stops after their eps(w_r) and appends them to group
  // (FP64 inversion to Wc by the caller, half_lower = 0) before
  // evaluate_end; otherwise it does the whole residue work itself.
  void evaluate_begin(const std::vector<int>& act, std::vector<GMat>* group);
  void evaluate_end();
  // evaluate_end in two halves: enqueue the rest of the residue work and the
  // copies, then synchronise and combine (so that a caller can enqueue the
  // work of many systems before waiting on any).
  void evaluate_post();
  void evaluate_finish();

  // State of an evaluation between its halves.
  std::vector<int> ev_act;
  std::vector<CdResidue> ev_res;
  std::vector<double> ev_hi, ev_rv, ev_rd;
  CdResidueChunk ev_chunk{};
  bool ev_grouped = false;
  bool ev_spd = false;  // every residue eps of this evaluation is SPD (see evaluate_begin)
  bool ev_guard = false;  // the residue eps of this evaluation are not certified >= I
  // Pinned staging in ctx->host_stage (reserved by setup_begin); sx is
  // filled from h_sx at the first evaluation's synchronisation.
  double *h_sx = nullptr, *h_hi = nullptr, *h_rv = nullptr, *h_rd = nullptr;
  bool sx_pending = false;
};

void launch_cd_gather(qx_ctx* ctx, const double* lpq, int naux, int nmo, const int2* nm, int R, double* b, int ld);

}  // namespace qx
