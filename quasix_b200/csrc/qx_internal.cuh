// Internal declarations shared by the CUDA translation units of libqxgpu.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <cmath>
#include <complex>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <stdexcept>
#include <string>
#include <vector>

#include "../../include/qx_gw.h"

namespace qx {

// Error carried to the C ABI boundary as a qx_status plus message.
struct Error : public std::runtime_error {
  qx_status status;
  Error(qx_status s, const std::string& m) : std::runtime_error(m), status(s) {}
};

inline std::string fmt(const char* f, ...) {
  char buf[1024];
  va_list ap;
  va_start(ap, f);
  vsnprintf(buf, sizeof(buf), f, ap);
  va_end(ap);
  return std::string(buf);
}

#define QX_CUDA(call)                                                                    \
  do {                                                                                   \
    cudaError_t e_ = (call);                                                             \
    if (e_ != cudaSuccess)                                                               \
      throw ::qx::Error(QX_ERR_CUDA, ::qx::fmt("%s failed: %s (%s:%d)", #call,          \
                                               cudaGetErrorString(e_), __FILE__, __LINE__)); \
  } while (0)

#define QX_REQUIRE(cond, status, ...)                       \
  do {                                                      \
    if (!(cond)) throw ::qx::Error(status, ::qx::fmt(__VA_ARGS__)); \
  } while (0)

// Device buffer owned by a context; grows, never shrinks, reused across calls.
struct DevBuf {
  void* ptr = nullptr;
  size_t bytes = 0;
  void reserve(size_t n) {
    if (n <= bytes) return;
    if (ptr) cudaFree(ptr);
    ptr = nullptr;
    bytes = 0;
    QX_CUDA(cudaMalloc(&ptr, n));
    bytes = n;
  }
  template <class T>
  T* as() const { return reinterpret_cast<T*>(ptr); }
  ~DevBuf() {
    if (ptr) cudaFree(ptr);
  }
};

// Grow-only page-locked host buffer: device-to-host copies into it stay
// asynchronous (a copy into pageable memory blocks the host until the stream
// reaches it).
struct HostBuf {
  void* ptr = nullptr;
  size_t bytes = 0;
  void reserve(size_t n) {
    if (n <= bytes) return;
    if (ptr) cudaFreeHost(ptr);
    ptr = nullptr;
    bytes = 0;
    QX_CUDA(cudaMallocHost(&ptr, n));
    bytes = n;
  }
  template <class T>
  T* as() const { return reinterpret_cast<T*>(ptr); }
  ~HostBuf() {
    if (ptr) cudaFreeHost(ptr);
  }
};

}  // namespace qx

// Stage indices for timing.
enum { QX_ST_P0 = 0, QX_ST_INV, QX_ST_CONTRACT, QX_ST_SIGMA, QX_ST_QP, QX_ST_COUNT };

struct qx_ctx {
  int device = 0;
  int sm_count = 148;
  cudaStream_t own_stream = nullptr;
  cudaStream_t stream = nullptr;
  std::string err;
  int64_t launches = 0;
  double stage_ms[QX_ST_COUNT] = {0, 0, 0, 0, 0};
  cudaEvent_t ev[2 * QX_ST_COUNT] = {};
  // Named workspace slots.
  qx::DevBuf ws[40];
  qx::HostBuf host_stage;  // pinned staging of small device-to-host results
  // Device status words to inspect after the next stream synchronisation:
  // (pointer, count, kind) with kind 0 = tcgen05 pipeline error code,
  // kind 1 = per-frequency singular-eps flags.
  struct Pending {
    const int* dev;
    int count;
    int kind;
  };
  std::vector<Pending> pending;
  // Status words of the pending checks: a fixed arena, never reallocated
  // while checks are pending; reset at every synchronisation.
  qx::DevBuf status_arena;
  int status_used = 0;
  // Streams of the look-ahead inversion (critical chain at high priority,
  // trailing updates at low priority) and their events; created on first use.
  cudaStream_t sweep_hi = nullptr, sweep_lo = nullptr;
  // Side stream of the setup (the rest of the pair gather from host lpq,
  // beside the first P0 and inversion) and its two events: prefix gathered,
  // all pairs gathered; created on first use.
  cudaStream_t side = nullptr;
  cudaEvent_t side_ev[2] = {};
  // Batch workers share the GPU with each other: their look-ahead streams keep
  // the default priority (a high-priority chain there stalls the other
  // workers' kernels while SMs drain for its large-shared-memory CTAs).
  bool worker = false;
  cudaEvent_t sweep_ev[4] = {};
  // Worker contexts of batched calls (own streams and workspaces), owned.
  std::vector<qx_ctx*> workers;
  // Guarded inversions of the last call: matrices checked, and matrices
  // re-inverted with pivoting.
  int64_t guard_matrices = 0, guard_reinverted = 0;
  // Form of the split-precision P0 (QX_P0_AUTO / _MATERIALISED / _CONVERTER);
  // batch workers inherit it from their parent context.
  int p0_form = 0;
  int contraction_form = 0;  // QX_CONTRACT_*: tiles of the split pair contraction
};

namespace qx {

// Workspace slot identifiers.
enum WsSlot {
  WS_LPQ = 0,     // lpq copy when the caller passes host memory
  WS_BPT,         // gathered pair tensor [npair][ldk] FP64
  WS_BOV,         // B_ov [naux][ldov] FP64
  WS_CHI,         // chi' [nw][ldov]
  WS_EPS,         // eps / Wc [nw][naux][ldn]
  WS_PANEL,       // sweep panels
  WS_VPAIR,       // v[w][npair]
  WS_SIGMA,       // sigma [norbs][nws] complex
  WS_SMALL,       // small per-call arrays (energies, grids, indices)
  WS_QPOUT,       // QP outputs
  WS_BPT_HI,      // bf16 split pair tensor
  WS_BPT_LO,
  WS_BOV_HI,
  WS_BOV_LO,
  WS_WC_HI,
  WS_WC_LO,
  WS_BPT_F32,     // FP32 copy of the pair tensor (epilogue operand)
  WS_HOSTIN,      // generic staging
  WS_BSE0, WS_BSE1, WS_BSE2, WS_BSE3, WS_BSE4, WS_BSE5, WS_BSE6, WS_BSE7,
  WS_CD0, WS_CD1, WS_CD2, WS_CD3,
  WS_TCERR,       // tcgen05 pipeline error word
  WS_GRAD0, WS_GRAD1, WS_GRAD2,  // CD adjoint: accumulators, per-frequency chunk, lpq gradient
  WS_SWEEP_SPLIT,  // split sweep panels (two steps in flight)
  WS_GUARD,        // guarded inversion: copies of eps and the pivoted fallback's work arrays
  WS_COUNT
};
static_assert(WS_COUNT <= 40, "workspace slots");

// Runs f once per device (per call site): kernel attributes such as the
// dynamic shared-memory limit are set per device, with that device current.
struct PerDeviceOnce {
  static constexpr int kMaxDevices = 64;
  std::once_flag flags[kMaxDevices];
  template <class F>
  void operator()(int device, F&& f) {
    QX_REQUIRE(device >= 0 && device < kMaxDevices, QX_ERR_INVALID_INPUT, "device %d out of range", device);
    std::call_once(flags[device], std::forward<F>(f));
  }
};

// Is p a device-accessible pointer of the current device?
bool is_device_ptr(const void* p);

// Make a device copy of a caller array when it is host memory; returns the
// device pointer to read.
const void* device_view(qx_ctx* ctx, int slot, const void* p, size_t bytes);

// As device_view, but page-locked host memory with a device mapping is not
// copied: the kernels read it in place over the host link, so only the bytes
// they touch cross it (the setup gathers read lpq's upper triangle, half of
// it).  For arrays that are read once, by kernels that touch part of them.
// *in_place (when given) tells whether the result is such host memory.
const void* mapped_view(qx_ctx* ctx, int slot, const void* p, size_t bytes, bool* in_place = nullptr);

inline int ceil_div(int a, int b) { return (a + b - 1) / b; }
inline int round_up(int a, int b) { return ceil_div(a, b) * b; }

inline void check_launch(qx_ctx* ctx) {
  ctx->launches++;
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) throw Error(QX_ERR_CUDA, fmt("kernel launch failed: %s", cudaGetErrorString(e)));
}

// Synchronise the context stream and act on the pending device status words.
void sync_and_check(qx_ctx* ctx);

// n status words (int) from the context's arena, valid until the next
// sync_and_check (which this call performs first when the arena is full).
int* status_words(qx_ctx* ctx, int n);

// Forget pending checks (and the guard counts) at the start of an entry point.
inline void reset_pending(qx_ctx* ctx) {
  ctx->pending.clear();
  ctx->status_used = 0;
  ctx->guard_matrices = 0;
  ctx->guard_reinverted = 0;
}

// Stage timer (CUDA events on the context stream).
struct StageTimer {
  qx_ctx* ctx;
  int st;
  StageTimer(qx_ctx* c, int s) : ctx(c), st(s) { cudaEventRecord(ctx->ev[2 * s], ctx->stream); }
  ~StageTimer() { cudaEventRecord(ctx->ev[2 * st + 1], ctx->stream); }
};

// ---------------------------------------------------------------------------
// Host-side numerics shared by the drivers.
// ---------------------------------------------------------------------------
void scaled_legendre_roots(int nw, double x0, double* freqs, double* wts);

// ---------------------------------------------------------------------------
// Kernel launchers (defined in the .cu files).
// ---------------------------------------------------------------------------
// chi'[w][k] = -4 e_k / (f_w^2 + e_k^2) (imaginary axis) or -4 e_k / (e_k^2 - f_w^2)
// (real axis), e_k = e_i - e_a over the ov pairs in row-major (i, a) order.
void launch_chi(qx_ctx* ctx, const double* energies, int nocc, int nvir, const double* freqs, int nw,
                int real_axis, double* chi, int ldov);

// eps[w] = I + B_ov diag(chi'[w]) B_ov^T for nw frequencies (FP64).
void launch_eps_fp64(qx_ctx* ctx, const double* bov, int ldov, int naux, int nov, const double* chi, int nw,
                     double* eps, int ldn, size_t eps_stride);

// ---------------------------------------------------------------------------
// Guarded inversion (k_pivot.cu).  The block sweep has no pivoting; when eps
// >= I cannot be shown, each eps is copied aside, the sweep flags a pivot
// below kGuardPivot * max|eps| or an unswept entry above kGuardGrowth *
// max|eps|, and the flagged matrices are inverted again from their copies by
// Gauss-Jordan elimination with partial pivoting.
// ---------------------------------------------------------------------------
constexpr double kGuardPivot = 1e-6;
constexpr double kGuardGrowth = 1e4;
// Probe backward error max|eps X v - v| / (n max|eps| max|X|) above which the
// sweep's inverse is redone with pivoting (a stable inverse gives ~1e-17).
constexpr double kGuardResidual = 1e-15;

// One guarded matrix.  The caller sets M, n, ldn, idx and status;
// guard_layout places bk, ints and rbuf.
struct GuardMat {
  double* M;     // the matrix being inverted ([n][ldn], -eps^-1 after the sweep or the fallback)
  double* bk;    // its copy, worked in place by the fallback
  int n, ldn;
  int idx;       // its index in the sweep (its max|eps| and growth words)
  int unused_;
  int* status;   // the sweep's status word of the matrix (nonzero: singular, Wc = 0)
  int* ints;     // 3 n ints: row state, pivot row of each column, inverse permutation
  double* rbuf;  // [n][32] the current panel's old pivot rows
};
struct GuardSet {
  std::vector<GuardMat> mats;  // the guarded matrices
  int nall = 0;                // matrices in the sweep (length of amax and growth)
  GuardMat* d_tab = nullptr;
  unsigned long long* amax = nullptr;    // [nall] max|eps| as a double's bits (0: not guarded)
  unsigned long long* growth = nullptr;  // [nall] max over the unswept entries met by the sweep
  unsigned long long* xmax = nullptr;    // [nall] max|eps^-1| of the sweep's result
  unsigned long long* rmax = nullptr;    // [nall] probe residual max|eps X v - v|
  int nflagged = 0;                      // matrices re-inverted by the last guard_end
};
// Workspace bytes of count guarded n x ldn matrices (an upper bound).
size_t guard_bytes(int n, int ldn, int count);
// Carve the workspace for gs.mats (and gs.nall words) out of mem.
void guard_layout(GuardSet& gs, void* mem, size_t bytes);
// Before the sweep, on the context stream: copies and max|eps|.
void guard_begin(qx_ctx* ctx, GuardSet& gs);
// After the sweep: synchronises the context stream, reads the flags and
// re-inverts the flagged matrices with pivoting (queued on the context
// stream).  Returns the number re-inverted.
int guard_end(qx_ctx* ctx, GuardSet& gs);

// eps >= I holds for eps = I + B diag(chi') B^T when every chi' >= 0: on the
// imaginary axis when no occupied level lies above a virtual one, on the real
// axis when in addition every shift |w| is below the smallest transition.
// energies: [nocc + nvir] host array; wmax: largest |real shift| (0: imaginary
// axis).  Strict inequalities keep chi' finite.
bool eps_at_least_identity(const double* energies, int nocc, int nvir, double wmax);

// In-place inversion of nw symmetric matrices by the block sweep operator;
// output Wc = eps^-1 - I (FP64).
// guard: the caller cannot show eps >= I (see eps_at_least_identity); the
// sweep then runs guarded, with the pivoted fallback.
// half_lower: return W' = strict-lower(Wc) + diag(Wc)/2 (zeros above) instead of Wc.
// split_update: run the trailing updates on tcgen05 in the FP16X3 form
// (launch_sweep_update_tc); the diagonal blocks and panels stay FP64.
void launch_invert_wc(qx_ctx* ctx, double* eps, int n, int ldn, size_t stride, int nw, int guard,
                      int half_lower = 0, int split_update = 0);

// One matrix of a grouped block sweep: M [n][ldn], symmetric, inverted in
// place.  prow (its first row in the concatenated panel arrays, a multiple of
// 128) is assigned by launch_invert_wc_group; guard as launch_invert_wc.
struct GMat {
  double* M;
  int n;
  int ldn;
  int prow;
  int guard;
};

// Wc = eps^-1 - I in place for G symmetric matrices of different orders (the
// eps of many systems at once): each block step of the sweep is one launch of
// each kernel over all matrices that still have that block, with the
// (matrix, tile) of a CTA found in per-step prefix tables.  half_lower and
// split_update as launch_invert_wc.  Runs on the context stream.
void launch_invert_wc_group(qx_ctx* ctx, const GMat* mats, int G, int half_lower, int split_update);

// The same sweep on caller-provided panels (no workspace, full Wc): Tp and Pp
// hold nw * n * SWEEP_NB doubles each, Dp nw * SWEEP_NB^2, status nw ints that
// must be zero on entry (nonzero on exit = singular eps, Wc set to 0).
// guard_mem (guard_bytes(n, ldn, nw) bytes, or null for an unguarded sweep)
// holds the guarded inversion's copies and work arrays.
// sweep_set_attributes() raises the kernels' dynamic shared-memory limits on
// the current device.
constexpr int kSweepPanelCols = 128;
void sweep_set_attributes();
void launch_invert_wc_panels(qx_ctx* ctx, double* eps, int n, int ldn, size_t stride, int nw, double* Tp,
                             double* Dp, double* Pp, int* status, void* guard_mem, size_t guard_mem_bytes);

// v[w][p] = Bpt[p]^T Wc[w] Bpt[p] for all pairs (FP64), given W' (half-lower form).
void launch_pair_contract_fp64(qx_ctx* ctx, const double* bpt, int ldk, int npair, int naux, const double* wc,
                               int ldn, size_t wc_stride, int nw, double* v, int ldv);

// Gathers.
// bpt[p][P] = lpq[P][pairs[p].x][pairs[p].y] on stream st; max_blocks > 0
// caps the grid (the blocks then walk the tiles).
void launch_gather_pairs(qx_ctx* ctx, cudaStream_t st, const double* lpq, int naux, int nmo, const int2* pairs,
                         int npair, double* bpt, int ldk, int max_blocks = 0);
void launch_gather_ov(qx_ctx* ctx, const double* lpq, int naux, int nmo, int nocc, double* bov, int ldov);
void launch_ov_from_pairs(qx_ctx* ctx, const double* bpt, int ldk, const int* pidx, int naux, int nmo, int nocc,
                          double* bov, int ldov);
void launch_exchange_pairs(qx_ctx* ctx, const double* bpt, int ldk, const int* pidx, int naux, int nmo, int nocc,
                           int norbs, double* sx);
// sx[p] = -sum_{R,i} lpq[R][p][i]^2 for every orbital, or only for the norbs
// orbitals orbs (device array) when given.
void launch_exchange_diag(qx_ctx* ctx, const double* lpq, int naux, int nmo, int nocc, double* sx,
                          const int* orbs = nullptr, int norbs = 0);

// Sigma_c(iw_k) assembly: sigma[t][k] (complex) for each target t.  sigma must
// be the start of the WS_SIGMA slot sized by sigma_workspace_doubles.
size_t sigma_workspace_doubles(int norbs, int nws, int nw, int nmo);
void launch_sigma_assemble(qx_ctx* ctx, const double* v, int ldv, int nw, const int* pair_index, int norbs,
                           int nmo, const int* orbs, int nocc, const double* energies, double ef,
                           const double* freqs, const double* wts, const double* iw, int nws,
                           double* sigma);

// Pade + QP per orbital (see k_qp.cu for the exact semantics).
struct QPParams {
  int norbs;
  int nws;
  int nfit;
  const int* fit_idx;       // [nfit]
  const double* sigma;      // complex [norbs][nws]
  const double* iw;         // [nws]
  const int* orbs;          // [norbs]
  int nocc;
  const double* mo_energy;  // reference (HF) energies [nmo]
  const double* eval_energy;// evaluation energies [nmo] (HF at iteration 0, previous QP after)
  const double* sigma_x;    // [nmo]
  const double* vxc;        // [nmo]
  double ef;
  double z_min, z_max;
  int solved;               // 0 linearized, 1 Newton
  int first_iteration;
  double newton_tol;
  int newton_max_iter;
  double* coeff;            // complex [nfit][norbs]
  double* qp_out;           // [norbs]
  double* z_out;            // [norbs]
  double* sc_out;           // complex [norbs]
};
void launch_pade_qp(qx_ctx* ctx, const QPParams& p);

// Mixed-precision (tcgen05) forms.  An operand is a hi/lo pair of bf16 or
// fp16 arrays plus the device scales (powers of two, one per batch) applied
// before the split.
struct TcOperand {
  void* hi;
  void* lo;
  float* scale;
};
inline bool is_tc_precision(int p) { return p == QX_PREC_BF16X3 || p == QX_PREC_FP16X3; }
// slot selects one of the scratch areas for the scales (0..2; 3..6 belong to
// the sweep, 7 to the B_ov split of P0).
// given_amax: the bounds max|src| per batch ([batch] words, a double's bits)
// are already on the device; no amax pass.
void launch_split(qx_ctx* ctx, const double* src, int rows, int cols, int ld_src, void* hi, void* lo, int ld_dst,
                  size_t src_stride, size_t dst_stride, int batch, int fp16, int slot, float** scale_out,
                  const unsigned long long* given_amax = nullptr);
// The amax words of split slot `slot` (1024, for kernels that accumulate a
// bound before the split).
unsigned long long* split_amax_words(qx_ctx* ctx, int slot);
// The amax words of split slot `slot` set to a known bound for n sources (in
// place of a pass over them), on the context stream.
unsigned long long* split_bound_words(qx_ctx* ctx, int slot, int n, double bound);
// reuse_a: B_ov is the one split by the previous call on this context; its
// hi/lo split is reused (unless the operand buffer has to grow).
void launch_eps_tc(qx_ctx* ctx, const double* bov, int ldov, int naux, int nov, const double* chi, int nw,
                   double* eps, int ldn, size_t eps_stride, int fp16, int reuse_a = 0);
void launch_gemm_tc(qx_ctx* ctx, const TcOperand& A, int M, int lda, const TcOperand& B, int N, int ldb, int K,
                    int nbatch, double* out, int ldo, size_t out_stride, int fp16);
void launch_pair_contract_tc(qx_ctx* ctx, const TcOperand& A, const float* bpt_f32, int ldk, int npair, int naux,
                             const TcOperand& W, int ldw, size_t wc_stride, int nw, double* v, int ldv, int fp16);
bool tc_supported(qx_ctx* ctx);

// Block sweep in the FP16X3 form: split the step's panels (buffer half buf of
// base, 2 * 4 * nw * n * 128 * 2 bytes in all; the bounds max|T|, max|P| per
// matrix must be in the amax words of split slots 3 + 2 buf and 4 + 2 buf),
// then the tcgen05 trailing update on stream st (mode / next_blk as
// k_sweep_update; err: one zeroed status word).
struct SweepSplit {
  TcOperand T, P;
};
SweepSplit launch_sweep_split(qx_ctx* ctx, cudaStream_t st, const double* Tp, const double* Pp, int n, int kb,
                              int nw, int buf, void* base);
void launch_sweep_update_tc(qx_ctx* ctx, cudaStream_t st, double* eps, int n, int ldn, size_t stride, int nw,
                            int kblk, const SweepSplit& sp, int mode, int next_blk, int* err);
// Grouped form: lower 128 x 128 tiles of the count matrices of d_mats (prefix
// table d_pre of tile counts, ntiles in all) minus the split panels T, P
// ([rows][128], one scale each), skipping tile row/column `step`.
void launch_gsweep_update_tc(qx_ctx* ctx, const GMat* d_mats, const int* d_pre, int count, int ntiles, int step,
                             const TcOperand& T, const TcOperand& P, int rows, int* err);


}  // namespace qx
