/*
 * qx_gw.h -- C ABI of the B200-native RI GW/BSE hot path (libqxgpu.so).
 *
 * The entry points mirror the QuasiX Rust API (quasix_core) and its PyO3
 * bindings; each declaration names the reference interface it replaces, by
 * file:line within the QuasiX project.  Conventions:
 *
 *  - Row-major (C order) arrays, FP64 unless stated.  Complex arrays are
 *    interleaved (re, im) doubles.
 *  - Every array argument may be a host pointer or a device pointer of the
 *    context's device; the library checks with cudaPointerGetAttributes and
 *    copies host data in and results out inside the call.  The lpq of
 *    qx_evgw and qx_get_sigma_diag is not copied when it is page-locked
 *    host memory: the setup kernels read the pairs they need from it in
 *    place (with every orbital a target, its upper triangle p <= q).
 *  - Every call returns a qx_status; on failure qx_last_error(ctx) holds a
 *    message.  No exceptions cross the ABI and no device code traps.
 *  - A context owns one CUDA stream and a cached device workspace; calls on
 *    one context are serialised by the caller (one thread at a time).
 */
#ifndef QX_GW_H
#define QX_GW_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Mirrors QuasixError (quasix_core/src/common/mod.rs:18-70). */
typedef enum {
  QX_OK = 0,
  QX_ERR_INVALID_INPUT = 1,      /* QuasixError::InvalidInput */
  QX_ERR_DIMENSION_MISMATCH = 2, /* QuasixError::DimensionMismatch */
  QX_ERR_NUMERICAL = 3,          /* QuasixError::NumericalError (non-finite, singular) */
  QX_ERR_CONVERGENCE = 4,        /* QuasixError::ConvergenceError */
  QX_ERR_NOT_IMPLEMENTED = 5,    /* QuasixError::NotImplemented */
  QX_ERR_CUDA = 6,               /* CUDA runtime / launch failure */
  QX_ERR_NO_DEVICE = 7           /* no usable sm_100 device */
} qx_status;

/* Arithmetic form of the dense contractions (P0, Sigma_c pair contraction).
 * FP64: the plain path.  BF16X3 / FP16X3: tcgen05 tensor cores, each FP64
 * operand split into hi + lo (bf16, or fp16 after a per-matrix power-of-two
 * scale), three products hi*hi + hi*lo + lo*hi accumulated in FP32 in TMEM;
 * the factorisation of eps, Pade and QP stay FP64.  Relative error per product
 * ~2^-17 (BF16X3) or ~2^-22 (FP16X3). */
typedef enum { QX_PREC_FP64 = 0, QX_PREC_BF16X3 = 1, QX_PREC_FP16X3 = 2 } qx_precision;

typedef struct qx_ctx qx_ctx;

/* ---- context -------------------------------------------------------------- */
qx_status qx_ctx_create(qx_ctx** ctx, int device);
qx_status qx_ctx_destroy(qx_ctx* ctx);
const char* qx_last_error(const qx_ctx* ctx);
/* Run on a caller stream (cudaStream_t as void*); NULL restores the context's own. */
qx_status qx_ctx_set_stream(qx_ctx* ctx, void* stream);
/* Milliseconds of device time of the last call, per stage (P0, inversion,
 * contraction, sigma assembly, QP), measured with CUDA events. */
qx_status qx_ctx_last_timings(const qx_ctx* ctx, double* ms_p0, double* ms_inv, double* ms_contract,
                              double* ms_sigma, double* ms_qp);
/* Number of kernel launches issued by the last call. */
int64_t qx_ctx_last_launches(const qx_ctx* ctx);
/* eps inversions of the last call that ran guarded (eps >= I not certain),
 * and how many of those were re-inverted with pivoting (no reference
 * counterpart).  Either pointer may be NULL. */
qx_status qx_ctx_last_guard_stats(const qx_ctx* ctx, int64_t* guarded, int64_t* reinverted);
/* Form of the split-precision P0 (FP16X3 / BF16X3; no reference
 * counterpart): QX_P0_MATERIALISED writes the hi/lo split of B_ov chi'(w) s_w
 * for every frequency (4 nw naux nov bytes) and reads it back by TMA;
 * QX_P0_PAIR reads the same operands with tiles on CTA pairs (tcgen05
 * cta_group::2, two 128-row tiles per MMA of M = 256); QX_P0_CONVERTER
 * applies chi'(w) while the B operand is staged in shared memory, so that
 * nothing chi-scaled goes to memory; QX_P0_AUTO (default) materialises up to
 * 6 GiB of such operands and converts beyond. */
enum { QX_P0_AUTO = 0, QX_P0_MATERIALISED = 1, QX_P0_CONVERTER = 2, QX_P0_PAIR = 3 };
qx_status qx_ctx_set_p0_form(qx_ctx* ctx, int form);
/* Tiles of the split-precision pair contraction Sigma_c needs (v = B W' B^T
 * row by row; no reference counterpart): QX_CONTRACT_SINGLE one 128-row pair
 * block per CTA; QX_CONTRACT_PAIR two pair blocks per CTA pair (tcgen05
 * cta_group::2, M = 256), each CTA staging half of the W' tile;
 * QX_CONTRACT_AUTO (default) takes the pair form. */
enum { QX_CONTRACT_AUTO = 0, QX_CONTRACT_SINGLE = 1, QX_CONTRACT_PAIR = 2 };
qx_status qx_ctx_set_contraction_form(qx_ctx* ctx, int form);
/* Library version string. */
const char* qx_version(void);

/* ---- freq ----------------------------------------------------------------- */
/* get_scaled_legendre_roots (quasix_core/src/selfenergy/correlation_ac.rs:94-114):
 * GL rule on [-1,1] mapped by w = x0 (1+t)/(1-t); host-only, no context. */
qx_status qx_get_scaled_legendre_roots(int nw, double x0, double* freqs, double* wts);

/* ---- gw: polarizability / screening ---------------------------------------- */
/* get_rho_response for nfreq imaginary frequencies at once
 * (correlation_ac.rs:184-211; S3-2 compute_polarizability_p0,
 * quasix_core/src/dielectric/polarizability.rs:169-275).
 * lpq_ov: [naux][nocc][nvir]; mo_energy: [nocc+nvir]; pi: [nfreq][naux][naux]. */
qx_status qx_get_rho_response(qx_ctx* ctx, int nfreq, const double* freqs, const double* mo_energy,
                              const double* lpq_ov, int naux, int nocc, int nvir, int precision,
                              double* pi);

/* Wc = (I - Pi)^-1 - I for nfreq matrices (correlation_ac.rs:377-401).
 * pi, wc: [nfreq][naux][naux] (may alias).  The reference inverts eps by
 * Cholesky, then by LU with partial pivoting, then substitutes the identity;
 * here a block Gauss-Jordan sweep runs first, guarded: a matrix with a pivot
 * below 1e-6 max|eps|, element growth above 1e4 max|eps|, or a probe-vector
 * backward error max|eps X v - v| / (n max|eps| max|X|) above 1e-15 is
 * inverted again by Gauss-Jordan elimination with partial pivoting, and one
 * that is singular there gets Wc = 0 (with a warning on stderr). */
qx_status qx_screened_interaction(qx_ctx* ctx, int nfreq, int naux, const double* pi, double* wc);

/* 1 when eps(w) = I + B diag(chi'(w)) B^T >= I is guaranteed for these
 * orbital energies at every real shift |w| <= wmax (wmax = 0: the imaginary
 * axis): every occupied level lies below every virtual one and wmax is below
 * that gap, so every chi' > 0.  The library's own inversions skip the guard
 * of qx_screened_interaction exactly then.  No reference counterpart (the
 * reference tries Cholesky first and falls back on failure); host-only. */
int qx_eps_at_least_identity(const double* mo_energy, int nocc, int nvir, double wmax);

/* compute_screened_interaction(P0, v_aux, freqs) (quasix_core/src/dielectric/
 * screening.rs:164-236, the S3-3 form used by the CD path): per frequency
 * W = v^1/2 (I - v^1/2 P0 v^1/2)^-1 v^1/2 with the symmetric square root of
 * v_aux, eps and W symmetrised by averaging as the reference does.
 * p0, w: [nfreq][naux][naux]; v_aux: [naux][naux] (host or device; w must
 * not alias p0).  The frequencies themselves are not needed (the reference
 * ignores its freqs argument too).  eps^-1 comes from the guarded sweep of
 * qx_screened_interaction.  Errors: QX_ERR_NUMERICAL when v_aux has an
 * eigenvalue at or below 1e-14 (the reference clamps those) or W is not
 * finite. */
qx_status qx_compute_screened_interaction(qx_ctx* ctx, int nfreq, int naux, const double* p0, const double* v_aux,
                                          double* w);

/* qx_screened_interaction without any allocation.  No counterpart in the
 * reference: it exists for callers that must not allocate device memory
 * inside the call (e.g. a pre-sized serving process).  pi and wc must be
 * device pointers of the context's device ([nfreq][naux][naux], may alias);
 * all scratch lives in one file-scope device array of
 * QX_NOALLOC_SCRATCH_BYTES, shared by every call on a device.  Limits:
 * naux <= QX_NOALLOC_MAX_NAUX, nfreq <= QX_NOALLOC_MAX_NFREQ; larger sizes
 * return QX_ERR_INVALID_INPUT.  The first call on each device resolves the
 * scratch address and sets kernel attributes: make it before any stream
 * capture.  Calls on one device that overlap in time (other threads, contexts
 * or streams) race on the scratch and must be serialised by the caller.
 * Synchronous: returns after wc is written. */
#define QX_NOALLOC_SCRATCH_BYTES (32u << 20)
#define QX_NOALLOC_MAX_NAUX 1024
#define QX_NOALLOC_MAX_NFREQ 4096
qx_status qx_screened_interaction_noalloc(qx_ctx* ctx, int nfreq, int naux, const double* pi, double* wc);

/* ---- selfenergy ------------------------------------------------------------ */
/* get_sigma_diag (correlation_ac.rs:241-449).  lpq: [naux][nmo][nmo] (symmetric
 * in the MO pair), orbs: [norbs].  Outputs sigma, omega: complex
 * [norbs][nw_sigma_max]; *nw_sigma receives the grid length
 * (1 + #{GL frequencies < iw_cutoff}).  nw_sigma_max must be >= nw + 1. */
qx_status qx_get_sigma_diag(qx_ctx* ctx, const double* mo_energy, const double* lpq, const int* orbs,
                            int norbs, int nmo, int nocc, int naux, int nw, double iw_cutoff, double x0,
                            int precision, double* sigma, double* omega, int nw_sigma_max,
                            int* nw_sigma);

/* thiele + ac_pade_thiele_diag (correlation_ac.rs:470-509, 587-654), one
 * device thread per orbital.  sigma, omega: complex [norbs][nw_sigma].
 * npade < 0 selects the reference's point rule; npade = k selects 2k points
 * (the [k/k] form, nfit <= 64).  coeff: complex [nfit][norbs], omega_fit:
 * complex [norbs][nfit]; *nfit out. */
qx_status qx_ac_pade_thiele_diag(qx_ctx* ctx, int norbs, int nw_sigma, const double* sigma,
                                 const double* omega, int npade, double* coeff, double* omega_fit,
                                 int nfit_max, int* nfit);

/* pade_thiele (correlation_ac.rs:530-566) at nomega real points for one
 * orbital, on the device: zn, coeff complex [nfit]; out complex [nomega]. */
qx_status qx_pade_thiele(qx_ctx* ctx, int nfit, const double* zn, const double* coeff, int nomega,
                         const double* omega, double* out);

/* NewtonSolverConfig (quasix_core/src/qp/newton_solver.rs:52-103; defaults
 * 50, 1e-8, 1.0, 0.1, 1.0, 1.0, 1e-6, 1, 0.1, 0.999, 1, 30). */
typedef struct {
  int max_iterations;
  double energy_tolerance;
  double initial_damping, min_damping, max_damping;
  double max_step;
  double derivative_delta;
  int use_richardson;
  double z_min, z_max;
  int use_bisection_fallback;
  int max_bisection_iterations;
} qx_newton_config;

/* NewtonQPSolver::new + solve (newton_solver.rs:141-402) for norbs orbitals at
 * once, one device thread each, with the Pade continuation of Sigma_c as the
 * evaluator (the SigmaCEvaluator of newton_solver.rs:133; coeff complex
 * [nfit][norbs] and omega_fit complex [norbs][nfit], the layout
 * qx_ac_pade_thiele_diag writes).  epsilon_hf, sigma_x, vxc, initial_guess:
 * [norbs]; fermi_level shared.  Outputs per orbital: qp_energy, residual
 * |f(E)|, iterations, method (0 Newton, 1 bisection fallback, -1 not
 * converged: the reference's ConvergenceError, with the last Newton iterate
 * in qp_energy), sigma_c complex [norbs], z_factor. */
qx_status qx_newton_qp_solve(qx_ctx* ctx, const qx_newton_config* cfg, int norbs, int nfit, const double* coeff,
                             const double* omega_fit, const double* epsilon_hf, const double* sigma_x,
                             const double* vxc, double fermi_level, const double* initial_guess, double* qp_energy,
                             double* residual, int* iterations, int* method, double* sigma_c, double* z_factor);

/* ---- analysis: spectral functions ------------------------------------------- */
/* SpectralAnalyzer::compute_spectral_function (quasix_core/src/analysis/
 * spectral.rs:235-325, profiles 327-545): weights[q] = sum_i Z_i P(omega[q] -
 * E_i) with P Gaussian (voigt_mixing < 0.01), Lorentzian (> 0.99) or the
 * mixture (1 - a) G + a L.  kind 0: every state; 1: generate_pes_spectrum
 * (states E <= fermi_energy at binding energy fermi_energy - E); 2:
 * generate_ipes_spectrum (states E > fermi_energy at E - fermi_energy)
 * (spectral.rs:557-656).  Rejects Z outside [0, 1], widths <= 0, mixing
 * outside [0, 1] and an empty grid (QX_ERR_INVALID_INPUT), as the reference's
 * validate() does.  total_weight (may be NULL): sum(weights) * (omega[1] -
 * omega[0]), the reference's normalisation figure. */
qx_status qx_spectral_function(qx_ctx* ctx, const double* qp_energies, const double* z_factors, int n_states,
                               double fermi_energy, int kind, const double* omega, int n_omega,
                               double gaussian_width, double lorentzian_width, double voigt_mixing,
                               double* weights, double* total_weight);

/* EvGWResult.spectral_function (quasix/quasix/evgw.py:124-134): per state,
 * A[i][q] = Z_i eta / ((omega[q] - E_i)^2 + eta^2) / pi; A [n_states][n_omega]. */
qx_status qx_spectral_function_states(qx_ctx* ctx, const double* qp_energies, const double* z_factors, int n_states,
                                      const double* omega, int n_omega, double eta, double* A);

/* Spectral function of each orbital from the Pade continuation of its
 * Sigma_c (the fits of qx_ac_pade_thiele_diag; no reference counterpart, the
 * reference broadens the QP peaks only): with S(w) the continued fraction of
 * orbital t at w - ef,
 *   A[t][q] = (1/pi) G / ((w - e_ref[t] - sigma_x[t] + vxc[t] - Re S)^2 + G^2),
 *   G = |Im S| + eta,  w = omega[q].
 * coeff complex [nfit][norbs], omega_fit complex [norbs][nfit]; vxc may be
 * NULL (0); A [norbs][n_omega]. */
qx_status qx_spectral_function_pade(qx_ctx* ctx, int norbs, int nfit, const double* coeff, const double* omega_fit,
                                    const double* e_ref, const double* sigma_x, const double* vxc, double ef,
                                    const double* omega, int n_omega, double eta, double* A);

/* Exchange self-energy diagonal (qp/evgw.rs:1167-1193):
 * sigma_x[p] = -sum_{i,R} lpq[R][p][i]^2. */
qx_status qx_compute_exchange_diag(qx_ctx* ctx, const double* lpq, int naux, int nmo, int nocc,
                                   double* sigma_x);

/* ---- qp: evGW driver -------------------------------------------------------- */
/* EvGWConfig (quasix_core/src/qp/evgw.rs:161-316) with the fields the driver uses. */
typedef struct {
  int max_iterations;          /* 12 */
  double energy_tolerance;     /* 1e-4 */
  double damping_factor;       /* 0.5 */
  double z_min, z_max;         /* 0.1, 0.999 */
  int use_diis;                /* 1 */
  int diis_space_dim;          /* 6 */
  int frontier_convergence;    /* 1 */
  double frontier_window;      /* 1.0 */
  int nfreq;                   /* 100 */
  double iw_cutoff;            /* 5.0 */
  double x0;                   /* 0.5 */
  int use_solved_qp;           /* 0 = linearized, 1 = Newton */
  double newton_energy_tolerance; /* 1e-8 */
  int newton_max_iterations;   /* 50 */
  int npade;                   /* -1 = reference point rule, k = [k/k] */
  int precision;               /* qx_precision */
  int fixed_iterations;        /* >0: run exactly this many iterations (benchmarking) */
} qx_evgw_config;

void qx_evgw_config_default(qx_evgw_config* cfg);

/* EvGWResult (qp/evgw.rs:329-350).  Caller-allocated arrays of nmo entries;
 * history_* arrays hold max_iterations entries (may be NULL). */
typedef struct {
  double* qp_energies;   /* [nmo] */
  double* z_factors;     /* [nmo] */
  double* sigma_x;       /* [nmo] diagonal */
  double* sigma_c;       /* complex [nmo] */
  double* history_energies; /* [max_iterations][nmo] or NULL */
  double* history_max_change; /* [max_iterations] or NULL */
  double* history_rms_change; /* [max_iterations] or NULL */
  int n_iterations;
  int converged;
} qx_evgw_result;

/* EvGWDriver::run_evgw_blocks (qp/evgw.rs:420-1049) on lpq [naux][nmo][nmo]
 * (the driver's permuted mn_full, evgw.rs:539-543); vxc: [nmo]. */
qx_status qx_evgw(qx_ctx* ctx, const double* mo_energy, const double* lpq, const double* vxc, int nmo,
                  int nocc, int naux, const qx_evgw_config* cfg, qx_evgw_result* res);

/* ---- G0W0 by contour deformation -------------------------------------------- */
/* QP solver of the CD entry points.  NEWTON: the step rule of
 * NewtonQPSolver::solve (quasix_core/src/qp/newton_solver.rs:174-280; clipped
 * step, adaptive damping) with the analytic slope of Sigma^CD, up to max_iter
 * evaluations.  LINEARIZED: one evaluation at e_n, E = e_n + Z (Sx + Sigma(e_n)
 * - Vxc) (qp/evgw.rs:784-821).  Z is clipped to [0.1, 0.999] in both. */
typedef enum { QX_QP_NEWTON = 0, QX_QP_LINEARIZED = 1 } qx_qp_solver;

/* Sigma_c(w) = imaginary-axis GL integral + residues at the real shifts
 * |w - e_m| (imaginary-axis integrand of compute_sigma_c_pyscf_cd,
 * quasix_core/src/selfenergy/correlation_pyscf_cd.rs:164-259; residues restated
 * from the full-frequency formulation, no reference implementation), Newton QP
 * root for each target.  Outputs [ntarget]. */
qx_status qx_g0w0_cd(qx_ctx* ctx, const double* mo_energy, const double* lpq, const double* vxc, int nmo,
                     int nocc, int naux, const int* targets, int ntarget, int nw, double x0, double tol,
                     int max_iter, int qp_solver, int precision, double* qp_energies, double* z_factors,
                     double* sigma_c, double* sigma_x);

/* Sigma_c^CD_n(w) and its slope dSigma/dw at caller-given real energies
 * omega[t] for each target (compute_sigma_c_pyscf_cd,
 * correlation_pyscf_cd.rs:164-259, which evaluates the imaginary-axis term at
 * one energy; here with the residues).  sigma_x receives diag(Sigma_x) of the
 * targets (may be NULL, as may dsigma_c). */
qx_status qx_cd_sigma(qx_ctx* ctx, const double* mo_energy, const double* lpq, int nmo, int nocc, int naux,
                      const int* targets, int ntarget, const double* omega, int nw, double x0, int precision,
                      double* sigma_c, double* dsigma_c, double* sigma_x);

/* Many independent G0W0-CD systems of uneven size in one call (no reference
 * counterpart: the reference runs compute_sigma_c_pyscf_cd once per system).
 * Each system is the argument set of qx_g0w0_cd.  nworkers = 0: grouped
 * mode -- the systems advance phase by phase on their own streams and every
 * inversion (the imaginary-axis eps of all systems; the residue eps of all
 * systems at each QP evaluation) runs as one grouped block sweep, in waves of
 * at most 64 systems and ~48 GB of workspace.  nworkers > 0: each system runs
 * whole on one of nworkers worker streams (at most 16), largest P0 cost
 * first; < 0: 4 such streams.  Per-system status is written to
 * systems[i].status; the call returns the first failure (by index). */
typedef struct {
  const double* mo_energy; /* [nmo] */
  const double* lpq;       /* [naux][nmo][nmo] */
  const double* vxc;       /* [nmo] or NULL (0) */
  int nmo, nocc, naux;
  const int* targets;      /* [ntarget] */
  int ntarget;
  double* qp_energies;     /* [ntarget] out */
  double* z_factors;       /* [ntarget] out or NULL */
  double* sigma_c;         /* [ntarget] out or NULL */
  double* sigma_x;         /* [ntarget] out or NULL */
  int status;              /* out: qx_status of this system */
} qx_cd_system;

qx_status qx_g0w0_cd_batch(qx_ctx* ctx, qx_cd_system* systems, int nsys, int nw, double x0, double tol,
                           int max_iter, int qp_solver, int precision, int nworkers);

/* Adjoint of the CD QP roots (no reference counterpart: QuasiX has no
 * derivative code).  Given the roots qp_energies[t] of f_t(E) = E - e_n - Sx_n
 * - Sigma^CD_n(E) + Vxc_n (as returned by qx_g0w0_cd with Newton; Vxc is held
 * fixed) and weights dl_dqp[t], returns the gradient of L = sum_t dl_dqp[t]
 * E_t with respect to mo_energy (grad_energy [nmo]) and the symmetric tensor
 * lpq (grad_lpq [naux][nmo][nmo], symmetric: dL = sum grad_lpq * dlpq for
 * every symmetric dlpq).  Implicit differentiation with Z_t = 1/(1 -
 * dSigma/dE) (unclipped, written to z_raw [ntarget] when non-NULL); P0 and W
 * are rebuilt per frequency, not stored.  precision selects the P0 rebuild
 * (FP64 or the split tcgen05 form); the adjoint GEMMs run in FP64.
 * grad_energy or grad_lpq may be NULL (not both); targets must be distinct. */
qx_status qx_g0w0_cd_grad(qx_ctx* ctx, const double* mo_energy, const double* lpq, int nmo, int nocc, int naux,
                          const int* targets, int ntarget, const double* qp_energies, const double* dl_dqp,
                          int nw, double x0, int precision, double* grad_energy, double* grad_lpq,
                          double* z_raw);

/* ---- df: density-fitting tensors ---------------------------------------------- */
/* transform_mo_3center (quasix_core/src/df/mo_transform.rs:136-282):
 * out[i*nvir + a][P] = sum_{u,v} C_occ[u][i] (uv|P) C_vir[v][a] on FP64 DMMA
 * GEMMs.  j3c_ao [nao][nao][naux] (symmetric in u, v), c_occ [nao][nocc],
 * c_vir [nao][nvir]. */
qx_status qx_transform_mo_3center(qx_ctx* ctx, const double* j3c_ao, const double* c_occ, const double* c_vir,
                                  int nao, int nocc, int nvir, int naux, double* out);

/* J^-1/2 and J^1/2 of the Coulomb metric J = (P|Q) (quasix/quasix/evgw.py:
 * 1014-1046, there by eigh with eigenvalues clamped at thresh_df) by the
 * scaled Denman-Beavers iteration on the device.  A metric with an eigenvalue
 * at or below thresh returns QX_ERR_NUMERICAL (the clamping is not
 * reproduced).  metric, inv_sqrt, sqrt_metric (may be NULL): [naux][naux]. */
qx_status qx_metric_inv_sqrt(qx_ctx* ctx, const double* metric, int naux, double thresh, double* inv_sqrt,
                             double* sqrt_metric);

/* The RI-normalised tensor of the DF tensor build (quasix/quasix/evgw.py:
 * 1007-1100): lpq[P][p][q] = sum_Q J^-1/2[P][Q] sum_{u,v} C[u][p] (uv|Q)
 * C[v][q], the lpq every GW and BSE entry point here takes.  Exactly one of
 * metric (J, then J^-1/2 as qx_metric_inv_sqrt with thresh) and
 * metric_inv_sqrt (J^-1/2 given) is non-NULL; chol_v (J^1/2, the
 * reference's chol_v; may be NULL) needs the metric.  j3c_ao
 * [nao][nao][naux], mo_coeff [nao][nmo], lpq [naux][nmo][nmo]. */
qx_status qx_build_lpq(qx_ctx* ctx, const double* j3c_ao, const double* mo_coeff, const double* metric,
                       const double* metric_inv_sqrt, int nao, int nmo, int naux, double thresh, double* lpq,
                       double* chol_v);

/* ---- bse -------------------------------------------------------------------- */
typedef struct qx_bse qx_bse;
/* BSETDAKernel::new (quasix_core/src/bse/kernel.rs:259-337; PyO3
 * quasix/src/bse.rs:139-200).  delta_qp [nov], df_ia [nov][naux],
 * df_ij [nocc*nocc][naux], df_ab [nvirt*nvirt][naux], w0 [naux][naux].
 * spin: 0 singlet (alpha_x = 2), 1 triplet (alpha_x = 0). */
qx_status qx_bse_create(qx_ctx* ctx, qx_bse** bse, int nocc, int nvirt, int naux, const double* delta_qp,
                        const double* df_ia, const double* df_ij, const double* df_ab, const double* w0,
                        int spin, int precision);
qx_status qx_bse_destroy(qx_bse* bse);
/* apply_tda_hamiltonian_batch (kernel.rs:550-598): x, y [nov][nvec]. */
qx_status qx_bse_apply(qx_bse* bse, const double* x, double* y, int nvec);

/* DavidsonConfig / DavidsonResult (quasix_core/src/bse/davidson.rs:47-145). */
typedef struct {
  int n_roots, max_iter, max_space;
  double tol_residual, lindep_threshold, level_shift;
} qx_davidson_config;
void qx_davidson_config_default(qx_davidson_config* cfg);

/* solve_davidson / davidson_bse (kernel.rs:652-663, davidson.rs:372-508).
 * eigenvalues [n_roots], eigenvectors [nov][n_roots], converged [n_roots],
 * residual_norms [n_roots]. */
qx_status qx_bse_davidson(qx_bse* bse, const qx_davidson_config* cfg, double* eigenvalues,
                          double* eigenvectors, int* converged, double* residual_norms,
                          int* iterations);

/* Operator for qx_davidson: y[v][0..n) = H x[v][0..n) for v < nvec.  x and y
 * are device pointers on the context's device, the vectors rows of stride ld
 * (ld >= n, a multiple of 8).  The callback runs on the thread that called
 * qx_davidson, after the library's work on x is complete; the library
 * synchronises the device after it returns, so y may be written on any
 * stream.  A nonzero return aborts the solve with that status
 * (QX_ERR_INVALID_INPUT when it is not a qx_status value). */
typedef int (*qx_apply_fn)(void* user, const double* x, double* y, int nvec, int ld);

/* davidson_bse(apply_h, qp_gaps, config) (quasix_core/src/bse/davidson.rs:
 * 372-508) with a caller-supplied operator: the same device Davidson as
 * qx_bse_davidson (unit-vector start at the smallest qp_gaps, preconditioner
 * 1 / (qp_gaps - theta + level_shift) with the reference's clamp, double
 * Gram-Schmidt, restart from the Ritz vectors past max_space).
 * qp_gaps: [n] (host or device); outputs as qx_bse_davidson with n in place
 * of nov. */
qx_status qx_davidson(qx_ctx* ctx, int n, const double* qp_gaps, qx_apply_fn apply_h, void* user,
                      const qx_davidson_config* cfg, double* eigenvalues, double* eigenvectors, int* converged,
                      double* residual_norms, int* iterations);

/* Gradient of an eigenvalue Omega of the kernel's matrix (eigenvector x [nov],
 * any norm) with respect to the orbital energies, grad_energy [nocc+nvirt], by
 * Hellmann-Feynman (no reference counterpart).  delta_qp is taken as
 * e_a - e_i.  With mo_energy non-NULL, W0 is taken as (I - Pi(0))^-1 built
 * from mo_energy and df_ia (qx_bse_w0) and its dependence is included; with
 * NULL, W0 is held fixed.  W0 must be symmetric. */
qx_status qx_bse_root_grad(qx_bse* bse, const double* x, const double* mo_energy, double* grad_energy);

/* ---- bse: optical properties ------------------------------------------------- */
/* compute_transition_dipoles (quasix/quasix/bse_driver.py:249-298) with the
 * AO dipole integrals given (the reference takes them from PySCF's
 * int1e_r): mu[i*nvir + a][c] = sum_{m,n} C[m][i] D[c][m][n] C[n][nocc + a].
 * mo_coeff [nao][nmo], ao_dipoles [3][nao][nao], mu [nocc*nvir][3]. */
qx_status qx_compute_transition_dipoles(qx_ctx* ctx, const double* mo_coeff, const double* ao_dipoles, int nao,
                                        int nmo, int nocc, double* mu);

/* compute_oscillator_strengths (quasix_core/src/bse/optical.rs:179-247):
 * d[n][c] = sum_t X[t][n] mu[t][c], f[n] = 2/3 E_n |d_n|^2, f_sum = sum f.
 * eigenvectors [n_trans][n_roots], transition_dipoles [n_trans][3];
 * root_dipoles [n_roots][3] and f_sum may be NULL.  A negative or non-finite
 * eigenvalue returns QX_ERR_NUMERICAL, as the reference does. */
qx_status qx_compute_oscillator_strengths(qx_ctx* ctx, const double* eigenvalues, const double* eigenvectors,
                                          const double* transition_dipoles, int n_trans, int n_roots,
                                          double* oscillator_strengths, double* root_dipoles, double* f_sum);

/* compute_absorption_spectrum (optical.rs:305-385): intensities[q] = sum_n
 * f_n L(E_q - E_n) on E_q = e_min + q (e_max - e_min) / (n_points - 1), L =
 * gamma / (x^2 + gamma^2) (broadening_type 0, Lorentzian) or exp(-x^2 / (2
 * gamma^2)) (1, Gaussian), gamma = broadening in Hartree.  has_range = 0
 * picks the reference's automatic range (eigenvalue span padded by max(0.2
 * span, 5 gamma), clipped at 0). */
qx_status qx_compute_absorption_spectrum(qx_ctx* ctx, const double* eigenvalues, const double* oscillator_strengths,
                                         int n_roots, int broadening_type, double broadening, int has_range,
                                         double e_min, double e_max, int n_points, double* energies,
                                         double* intensities);

/* qx_bse_root_grad with the gradient of Omega with respect to the DF blocks as
 * passed to qx_bse_create (no reference counterpart): grad_ia [nov][naux],
 * grad_ij [nocc*nocc][naux], grad_ab [nvirt*nvirt][naux], each entry the
 * derivative with respect to that input entry (Hellmann-Feynman on the
 * normalised x):
 *   d/dB_ia^P = 2 alpha_x x_ia (B_ia^T x)_P [+ 8/Delta_ia (G B_ia)_P],
 *   d/dB_ij^P = -(T W0)_(ij)P, T^Q_ij = sum_ab x_ia B_ab^Q x_jb,
 *   d/dB_ab^Q = -sum_ij x_ia (B_ij W0)^Q_ij x_jb,
 * the bracket (G = W0 sym(M) W0, M_PQ = sum_ij B_ij^P T^Q_ij) when mo_energy is
 * given and W0 = (I - Pi(0))^-1 is taken to follow df_ia and the energies.
 * Any output may be NULL (not all). */
qx_status qx_bse_root_grad_b(qx_bse* bse, const double* x, const double* mo_energy, double* grad_energy,
                             double* grad_ia, double* grad_ij, double* grad_ab);

/* W(w=0) = (I - Pi(0))^-1 for the screened-direct kernel, from lpq_ov [naux][nocc][nvir]. */
qx_status qx_bse_w0(qx_ctx* ctx, const double* mo_energy, const double* lpq_ov, int naux, int nocc,
                    int nvir, double* w0);

#ifdef __cplusplus
}
#endif
#endif /* QX_GW_H */
