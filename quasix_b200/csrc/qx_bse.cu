// BSE-TDA on the GPU: the matrix-free Hamiltonian of BSETDAKernel
// (quasix_core/src/bse/kernel.rs:501-598) as batched GEMMs, and the block
// Davidson of davidson_bse (quasix_core/src/bse/davidson.rs:372-508) with the
// subspace, Rayleigh-Ritz (parallel Jacobi) and re-orthonormalisation on the
// device; the host only steers (convergence flags, subspace size).
#include <cuda_bf16.h>
#include <cuda_fp16.h>

#include <algorithm>
#include <cmath>
#include <functional>
#include <numeric>

#include "qx_blas.cuh"
#include "qx_internal.cuh"
#include "split_round.cuh"

namespace qx {

// out[b][c][r] = in[b][r][c]   (rows x cols per batch)
__global__ void k_transpose(const double* __restrict__ in, int rows, int cols, int ldi, size_t si,
                            double* __restrict__ out, int ldo, size_t so) {
  __shared__ double t[32][33];
  const int b = blockIdx.z;
  const int r0 = blockIdx.y * 32, c0 = blockIdx.x * 32;
  for (int y = threadIdx.y; y < 32; y += blockDim.y) {
    const int r = r0 + y, c = c0 + threadIdx.x;
    t[y][threadIdx.x] = (r < rows && c < cols) ? in[(size_t)b * si + (size_t)r * ldi + c] : 0.0;
  }
  __syncthreads();
  for (int y = threadIdx.y; y < 32; y += blockDim.y) {
    const int c = c0 + y, r = r0 + threadIdx.x;
    if (c < cols && r < rows) out[(size_t)b * so + (size_t)c * ldo + r] = t[threadIdx.x][y];
  }
}

void transpose(qx_ctx* ctx, const double* in, int rows, int cols, int ldi, size_t si, double* out, int ldo,
               size_t so, int batch) {
  dim3 grid(ceil_div(cols, 32), ceil_div(rows, 32), batch);
  k_transpose<<<grid, dim3(32, 8), 0, ctx->stream>>>(in, rows, cols, ldi, si, out, ldo, so);
  check_launch(ctx);
}

// Xp[(v, j)][b] = X[v][j * nvir + b] (rows padded to ldvp).
__global__ void k_pack_x(const double* __restrict__ X, int ldx, int nvec, int nocc, int nvir,
                         double* __restrict__ Xp, int ldvp) {
  const size_t total = (size_t)nvec * nocc * ldvp;
  for (size_t idx = (size_t)blockIdx.x * blockDim.x + threadIdx.x; idx < total;
       idx += (size_t)gridDim.x * blockDim.x) {
    const int b = (int)(idx % ldvp);
    const size_t row = idx / ldvp;
    const int v = (int)(row / nocc), j = (int)(row % nocc);
    Xp[idx] = (b < nvir) ? X[(size_t)v * ldx + (size_t)j * nvir + b] : 0.0;
  }
}

// Y[v][ia] = delta[ia] X[v][ia] + ax Yx[v][ia] - Yd[i][a * nvec + v]
__global__ void k_bse_combine(const double* __restrict__ X, const double* __restrict__ delta,
                              const double* __restrict__ Yx, const double* __restrict__ Yd, int nvec, int nocc,
                              int nvir, int ldx, double ax, double* __restrict__ Y) {
  const int nov = nocc * nvir;
  const size_t total = (size_t)nvec * ldx;
  for (size_t idx = (size_t)blockIdx.x * blockDim.x + threadIdx.x; idx < total;
       idx += (size_t)gridDim.x * blockDim.x) {
    const int v = (int)(idx / ldx), ia = (int)(idx % ldx);
    double y = 0.0;
    if (ia < nov) {
      const int i = ia / nvir, a = ia % nvir;
      y = delta[ia] * X[idx] - Yd[(size_t)i * nvir * nvec + (size_t)a * nvec + v];
      if (ax != 0.0) y += ax * Yx[idx];
    }
    Y[idx] = y;
  }
}

// R[r] = AX[r] - theta[r] X[r]; nrm2[r] = |R[r]|^2
__global__ void k_residual(const double* __restrict__ AX, const double* __restrict__ X, const double* __restrict__ theta,
                           int ld, int n, double* __restrict__ R, double* __restrict__ nrm2) {
  const int r = blockIdx.y;
  double s = 0.0;
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x) {
    const double v = AX[(size_t)r * ld + k] - theta[r] * X[(size_t)r * ld + k];
    R[(size_t)r * ld + k] = v;
    s += v * v;
  }
  for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
  __shared__ double red[32];
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = s;
  __syncthreads();
  if (threadIdx.x == 0) {
    double t = 0.0;
    for (int i = 0; i < (int)(blockDim.x >> 5); ++i) t += red[i];
    atomicAdd(nrm2 + r, t);
  }
}

// t = r / (delta - theta + shift) with the reference's clamp (davidson.rs:194-225); nrm2 += |t|^2
__global__ void k_precond(const double* __restrict__ R, const double* __restrict__ delta, double theta, double shift,
                          int n, double* __restrict__ t, double* __restrict__ nrm2) {
  double s = 0.0;
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x) {
    double den = delta[k] - theta + shift;
    if (fabs(den) < 1e-8) den = (den >= 0.0) ? 1e-8 : -1e-8;
    const double v = R[k] / den;
    t[k] = v;
    s += v * v;
  }
  for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
  __shared__ double red[32];
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = s;
  __syncthreads();
  if (threadIdx.x == 0) {
    double tt = 0.0;
    for (int i = 0; i < (int)(blockDim.x >> 5); ++i) tt += red[i];
    atomicAdd(nrm2, tt);
  }
}

// x[k] *= 1/sqrt(nrm2[0]) when sqrt(nrm2) > thr (thr < 0: always)
__global__ void k_normalize(double* __restrict__ x, int n, const double* __restrict__ nrm2, double thr) {
  const double nr = sqrt(nrm2[0]);
  if (!(nr > thr)) return;
  const double inv = 1.0 / nr;
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x) x[k] *= inv;
}

__global__ void k_norm2(const double* __restrict__ x, int n, double* __restrict__ nrm2) {
  double s = 0.0;
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x) s += x[k] * x[k];
  for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
  __shared__ double red[32];
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = s;
  __syncthreads();
  if (threadIdx.x == 0) {
    double t = 0.0;
    for (int i = 0; i < (int)(blockDim.x >> 5); ++i) t += red[i];
    atomicAdd(nrm2, t);
  }
}

// M <- (M + M^T) / 2 for an n x n matrix (ld).
__global__ void k_symmetrize(double* __restrict__ M, int n, int ld) {
  for (int idx = blockIdx.x * blockDim.x + threadIdx.x; idx < n * n; idx += gridDim.x * blockDim.x) {
    const int r = idx / n, c = idx % n;
    if (c < r) {
      const double v = 0.5 * (M[(size_t)r * ld + c] + M[(size_t)c * ld + r]);
      M[(size_t)r * ld + c] = v;
      M[(size_t)c * ld + r] = v;
    }
  }
}

// s[k] = sum_Q U[k][Q] D[k][Q]   (one warp per row)
__global__ void k_rowdot(const double* __restrict__ U, const double* __restrict__ D, int rows, int n, int ld,
                         double* __restrict__ s) {
  const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
  if (warp >= rows) return;
  double acc = 0.0;
  for (int q = lane; q < n; q += 32) acc += U[(size_t)warp * ld + q] * D[(size_t)warp * ld + q];
  for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
  if (lane == 0) s[warp] = acc;
}

}  // namespace qx

using namespace qx;

// max|x| over n doubles (a double's bits; x >= 0 compares as its pattern).
__global__ void k_absmax(const double* __restrict__ x, size_t n, unsigned long long* __restrict__ out) {
  double m = 0.0;
  for (size_t k = (size_t)blockIdx.x * blockDim.x + threadIdx.x; k < n; k += (size_t)gridDim.x * blockDim.x)
    m = fmax(m, fabs(x[k]));
  for (int o = 16; o > 0; o >>= 1) m = fmax(m, __shfl_xor_sync(0xffffffffu, m, o));
  __shared__ double red[32];
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = m;
  __syncthreads();
  if (threadIdx.x < 32) {
    m = threadIdx.x < (blockDim.x >> 5) ? red[threadIdx.x] : 0.0;
    for (int o = 16; o > 0; o >>= 1) m = fmax(m, __shfl_xor_sync(0xffffffffu, m, o));
    if (threadIdx.x == 0) atomicMax(out, __double_as_longlong(m));
  }
}

// Row (i,a) of the direct kernel K^d[(i,a)][(j,b)] = C[(i,j)][(a,b)], scaled
// by s and split into hi/lo (fp16 or bf16, the rounding of the other splits),
// row stride ldg, zero past nov.  One block per row.
template <bool FP16>
__global__ void k_kd_split(const double* __restrict__ C, int nocc, int nvir, int ldg, double s,
                           uint16_t* __restrict__ hi, uint16_t* __restrict__ lo) {
  const int row = blockIdx.x, i = row / nvir, a = row % nvir;
  const size_t ldc = (size_t)nvir * nvir;
  const int nov = nocc * nvir;
  for (int c = threadIdx.x; c < ldg; c += blockDim.x) {
    double v = 0.0;
    if (c < nov) {
      const int j = c / nvir, b = c % nvir;
      v = C[(size_t)(i * nocc + j) * ldc + (size_t)a * nvir + b] * s;
    }
    uint16_t h, l;
    split_round<FP16>(v, h, l);
    hi[(size_t)row * ldg + c] = h;
    lo[(size_t)row * ldg + c] = l;
  }
}

struct DevArr {
  double* p = nullptr;
  size_t n = 0;
  void alloc(size_t count) {
    if (count <= n) return;
    if (p) cudaFree(p);
    p = nullptr;
    n = 0;
    QX_CUDA(cudaMalloc(&p, count * sizeof(double)));
    n = count;
  }
  ~DevArr() {
    if (p) cudaFree(p);
  }
};

// Davidson subspace and scratch (grown on demand, reused across solves).
struct DavWork {
  DevArr V, AV, X, AX, R, heff, jv, Z2, small, eigi;
};

struct qx_bse {
  qx_ctx* ctx;
  int nocc, nvir, naux, nov, precision;
  int ldq, ldvp, ldov;
  double alpha_x;
  DevArr delta, dia, diaT, ijw, dabT;
  DevArr w0T, dij;                   // kept for the root gradient (W0 term)
  DevArr dab_split, dab_scale;       // split forms: hi/lo of dabT [a][Q][ldvp], scale per a
  // Split forms, when it fits: the direct kernel K^d [nov][ldg] as hi/lo with
  // one scale, so that a matvec's direct term is one GEMM.
  DevArr kd_split, kd_scale;
  int ldg = 0;
  bool kd = false;
  DevArr x_split;                    // split forms: hi/lo of the packed vectors
  DevArr xp, T, Yd, Z, Yx, Xr, Yr;  // matvec scratch
  DevArr gTt, gTp, gTpT, gdijT, gM, gG1, gG, gU;  // root-gradient scratch
  DevArr gGrad;                                     // root-gradient scratch of the DF blocks
  DavWork dav;
  std::vector<double> h_delta;
};

// y[v] = H x[v] for nvec vectors in row layout [nvec][ldov] (device).
// need_T: take the factored direct term even when K^d is held (the root
// gradient reads its first step T).
static void bse_apply_rows(qx_bse* B, const double* X, double* Y, int nvec, bool need_T = false) {
  qx_ctx* ctx = B->ctx;
  const int nocc = B->nocc, nvir = B->nvir, naux = B->naux;
  B->Yd.alloc((size_t)nocc * nvir * nvec);
  if (B->kd && !need_T) {
    // Direct term as one GEMM: Yd[(i,a)][v] = sum_(j,b) K^d[(i,a)][(j,b)] X[v][(j,b)]
    // (the layout Yd[i][(a,v)] of the factored form).
    const int fp16 = B->precision == QX_PREC_FP16X3;
    const size_t xe = (size_t)nvec * B->ldov;
    const size_t xhalf = ((xe * 2 + 255) / 256) * 256;
    B->x_split.alloc((2 * xhalf + 7) / 8 + 64);
    uint8_t* xs = reinterpret_cast<uint8_t*>(B->x_split.p);
    TcOperand Xo{xs, xs + xhalf, nullptr};
    launch_split(ctx, X, nvec, B->nov, B->ldov, Xo.hi, Xo.lo, B->ldov, 0, 0, 1, fp16, 0, &Xo.scale);
    const size_t ge = (size_t)B->nov * B->ldg;
    uint8_t* gs = reinterpret_cast<uint8_t*>(B->kd_split.p);
    TcOperand Go{gs, gs + ((ge * 2 + 255) / 256) * 256, reinterpret_cast<float*>(B->kd_scale.p)};
    launch_gemm_tc(ctx, Go, B->nov, B->ldg, Xo, nvec, B->ldov, B->nov, 1, B->Yd.p, nvec, 0, fp16);
  } else {
  // Direct term, step 1: T[a][(v,j)][Q] = sum_b X[v][j,b] dab[a][b][Q].
  B->xp.alloc((size_t)nvec * nocc * B->ldvp);
  {
    const size_t tot = (size_t)nvec * nocc * B->ldvp;
    k_pack_x<<<(unsigned)std::min<size_t>((tot + 255) / 256, 4096), 256, 0, ctx->stream>>>(X, B->ldov, nvec, nocc, nvir,
                                                                                          B->xp.p, B->ldvp);
    check_launch(ctx);
  }
  const size_t tslab = (size_t)nvec * nocc * B->ldq;
  if (B->T.n < tslab * nvir) {
    B->T.alloc(tslab * nvir);
    QX_CUDA(cudaMemsetAsync(B->T.p, 0, tslab * nvir * sizeof(double), ctx->stream));  // Q padding stays zero
  }
  if (is_tc_precision(B->precision)) {
    // T on tcgen05: split packed X (one scale), dabT split at create.
    const int fp16 = B->precision == QX_PREC_FP16X3;
    const size_t xe = (size_t)nvec * nocc * B->ldvp;
    B->x_split.alloc((xe * 2 * 2 + 7) / 8 + 64);
    uint8_t* xs = reinterpret_cast<uint8_t*>(B->x_split.p);
    TcOperand A{xs, xs + ((xe * 2 + 255) / 256) * 256, nullptr};
    launch_split(ctx, B->xp.p, nvec * nocc, nvir, B->ldvp, A.hi, A.lo, B->ldvp, 0, 0, 1, fp16, 0, &A.scale);
    const size_t de = (size_t)nvir * naux * B->ldvp;
    uint8_t* ds = reinterpret_cast<uint8_t*>(B->dab_split.p);
    TcOperand Bo{ds, ds + ((de * 2 + 255) / 256) * 256, reinterpret_cast<float*>(B->dab_scale.p)};
    launch_gemm_tc(ctx, A, nvec * nocc, B->ldvp, Bo, naux, B->ldvp, nvir, nvir, B->T.p, B->ldq, tslab, fp16);
  } else {
    GemmNT g{};
    g.M = nvec * nocc;
    g.N = naux;
    g.K = nvir;
    g.A = B->xp.p;
    g.lda = B->ldvp;
    g.sA = 0;
    g.B = B->dabT.p;
    g.ldb = B->ldvp;
    g.sB = (size_t)naux * B->ldvp;
    g.C = B->T.p;
    g.ldc = B->ldq;
    g.sC = tslab;
    g.batch = nvir;
    g.alpha = 1.0;
    g.beta = 0.0;
    g.splitk = 1;
    gemm_nt_f64(ctx, g);
  }
  // Step 2: Yd[i][(a,v)] = sum_{(j,Q)} ijw[i][(j,Q)] T[a][v][(j,Q)].
  {
    GemmNT g{};
    g.M = nocc;
    g.N = nvir * nvec;
    g.K = nocc * B->ldq;
    g.A = B->ijw.p;
    g.lda = nocc * B->ldq;
    g.B = B->T.p;
    g.ldb = nocc * B->ldq;
    g.C = B->Yd.p;
    g.ldc = nvir * nvec;
    g.batch = 1;
    g.alpha = 1.0;
    g.beta = 0.0;
    g.splitk = 0;
    gemm_nt_f64(ctx, g);
  }
  }
  // Exchange: Z[v][Q] = sum_ia X[v][ia] dia[ia][Q]; Yx[v][ia] = sum_Q Z[v][Q] dia[ia][Q].
  if (B->alpha_x != 0.0) {
    B->Z.alloc((size_t)nvec * B->ldq);
    B->Yx.alloc((size_t)nvec * B->ldov);
    GemmNT g{};
    g.M = nvec;
    g.N = naux;
    g.K = B->nov;
    g.A = X;
    g.lda = B->ldov;
    g.B = B->diaT.p;
    g.ldb = B->ldov;
    g.C = B->Z.p;
    g.ldc = B->ldq;
    g.batch = 1;
    g.alpha = 1.0;
    g.splitk = 0;
    gemm_nt_f64(ctx, g);
    GemmNT h{};
    h.M = nvec;
    h.N = B->nov;
    h.K = naux;
    h.A = B->Z.p;
    h.lda = B->ldq;
    h.B = B->dia.p;
    h.ldb = B->ldq;
    h.C = B->Yx.p;
    h.ldc = B->ldov;
    h.batch = 1;
    h.alpha = 1.0;
    h.splitk = 1;
    gemm_nt_f64(ctx, h);
  }
  const size_t tot = (size_t)nvec * B->ldov;
  k_bse_combine<<<(unsigned)std::min<size_t>((tot + 255) / 256, 4096), 256, 0, ctx->stream>>>(
      X, B->delta.p, B->alpha_x != 0.0 ? B->Yx.p : nullptr, B->Yd.p, nvec, nocc, nvir, B->ldov, B->alpha_x, Y);
  check_launch(ctx);
}

template <class F>
static qx_status bse_guard(qx_ctx* ctx, F&& f) {
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

static void upload(qx_ctx* ctx, double* dst, const double* src, size_t n) {
  QX_CUDA(cudaMemcpyAsync(dst, src, n * sizeof(double), cudaMemcpyDefault, ctx->stream));
}

extern "C" {

void qx_davidson_config_default(qx_davidson_config* c) {
  c->n_roots = 3;
  c->max_iter = 100;
  c->max_space = 60;
  c->tol_residual = 1e-5;
  c->lindep_threshold = 1e-12;
  c->level_shift = 0.001;
}

qx_status qx_bse_create(qx_ctx* ctx, qx_bse** out, int nocc, int nvirt, int naux, const double* delta_qp,
                        const double* df_ia, const double* df_ij, const double* df_ab, const double* w0, int spin,
                        int precision) {
  if (!ctx || !out) return QX_ERR_INVALID_INPUT;
  *out = nullptr;
  qx_bse* B = new qx_bse();
  qx_status st = bse_guard(ctx, [&] {
    QX_REQUIRE(nocc > 0 && nvirt > 0 && naux > 0, QX_ERR_DIMENSION_MISMATCH, "nocc=%d nvirt=%d naux=%d must be positive",
               nocc, nvirt, naux);
    QX_REQUIRE(delta_qp && df_ia && df_ij && df_ab && w0, QX_ERR_INVALID_INPUT, "null BSE input");
    QX_REQUIRE(spin == 0 || spin == 1, QX_ERR_INVALID_INPUT, "Unknown spin type %d", spin);
    QX_REQUIRE(precision == QX_PREC_FP64 || is_tc_precision(precision), QX_ERR_INVALID_INPUT, "bad precision %d",
               precision);
    QX_REQUIRE(!is_tc_precision(precision) || nvirt <= 1024, QX_ERR_INVALID_INPUT,
               "split forms support nvirt <= 1024 (one scale per virtual orbital)");
    B->ctx = ctx;
    B->nocc = nocc;
    B->nvir = nvirt;
    B->naux = naux;
    B->nov = nocc * nvirt;
    B->precision = precision;
    B->ldq = round_up(naux, 8);
    B->ldvp = round_up(nvirt, 8);
    B->ldov = round_up(B->nov, 8);
    B->alpha_x = spin == 0 ? 2.0 : 0.0;  // SpinType::exchange_prefactor (kernel.rs:67-79)
    const int nov = B->nov;
    B->h_delta.resize(nov);
    QX_CUDA(cudaMemcpy(B->h_delta.data(), delta_qp, nov * sizeof(double), cudaMemcpyDefault));
    for (double d : B->h_delta) QX_REQUIRE(std::isfinite(d), QX_ERR_NUMERICAL, "delta_qp contains NaN or Inf");
    B->delta.alloc(B->ldov);
    QX_CUDA(cudaMemsetAsync(B->delta.p, 0, B->ldov * sizeof(double), ctx->stream));
    upload(ctx, B->delta.p, B->h_delta.data(), nov);
    // Staging for unpadded inputs.
    DevArr stage;
    stage.alloc(std::max({(size_t)nvirt * nvirt * naux, (size_t)nov * naux, (size_t)naux * naux,
                          (size_t)nocc * nocc * naux}));
    // df_ia -> dia [nov][ldq] and diaT [naux][ldov].
    upload(ctx, stage.p, df_ia, (size_t)nov * naux);
    B->dia.alloc((size_t)nov * B->ldq);
    QX_CUDA(cudaMemsetAsync(B->dia.p, 0, (size_t)nov * B->ldq * sizeof(double), ctx->stream));
    QX_CUDA(cudaMemcpy2DAsync(B->dia.p, B->ldq * sizeof(double), stage.p, naux * sizeof(double), naux * sizeof(double),
                              nov, cudaMemcpyDeviceToDevice, ctx->stream));
    B->diaT.alloc((size_t)naux * B->ldov);
    QX_CUDA(cudaMemsetAsync(B->diaT.p, 0, (size_t)naux * B->ldov * sizeof(double), ctx->stream));
    transpose(ctx, stage.p, nov, naux, naux, 0, B->diaT.p, B->ldov, 0, 1);
    // w0^T [Q][P] (ldq), df_ij [nocc^2][ldq]; ijw = df_ij w0 (kernel.rs:286-291).
    DevArr& w0T = B->w0T;
    DevArr& dij = B->dij;
    upload(ctx, stage.p, w0, (size_t)naux * naux);
    w0T.alloc((size_t)naux * B->ldq);
    QX_CUDA(cudaMemsetAsync(w0T.p, 0, (size_t)naux * B->ldq * sizeof(double), ctx->stream));
    transpose(ctx, stage.p, naux, naux, naux, 0, w0T.p, B->ldq, 0, 1);
    QX_CUDA(cudaStreamSynchronize(ctx->stream));
    upload(ctx, stage.p, df_ij, (size_t)nocc * nocc * naux);
    dij.alloc((size_t)nocc * nocc * B->ldq);
    QX_CUDA(cudaMemsetAsync(dij.p, 0, (size_t)nocc * nocc * B->ldq * sizeof(double), ctx->stream));
    QX_CUDA(cudaMemcpy2DAsync(dij.p, B->ldq * sizeof(double), stage.p, naux * sizeof(double), naux * sizeof(double),
                              (size_t)nocc * nocc, cudaMemcpyDeviceToDevice, ctx->stream));
    B->ijw.alloc((size_t)nocc * nocc * B->ldq);
    QX_CUDA(cudaMemsetAsync(B->ijw.p, 0, (size_t)nocc * nocc * B->ldq * sizeof(double), ctx->stream));
    {
      GemmNT g{};
      g.M = nocc * nocc;
      g.N = naux;
      g.K = naux;
      g.A = dij.p;
      g.lda = B->ldq;
      g.B = w0T.p;
      g.ldb = B->ldq;
      g.C = B->ijw.p;
      g.ldc = B->ldq;
      g.batch = 1;
      g.alpha = 1.0;
      g.splitk = 0;
      gemm_nt_f64(ctx, g);
    }
    // df_ab [a][b][Q] -> dabT [a][Q][b] (ldvp).
    QX_CUDA(cudaStreamSynchronize(ctx->stream));
    upload(ctx, stage.p, df_ab, (size_t)nvirt * nvirt * naux);
    // Split forms: hold K^d[(i,a)][(j,b)] = sum_Q ijw[(i,j)][Q] B_ab[(a,b)][Q]
    // (kernel.rs:391-462 contracted once) when its FP64 build (nov^2 doubles,
    // freed after the split) fits 16 GB: every matvec's direct term is then
    // one GEMM that streams the 4 nov^2 bytes of hi/lo, instead of the
    // 2 nov nvir naux-FLOP factored product per vector.
    if (is_tc_precision(precision) && (size_t)nov * nov * sizeof(double) <= ((size_t)16 << 30)) {
      const int fp16 = precision == QX_PREC_FP16X3;
      DevArr cmat;
      cmat.alloc((size_t)nov * nov);
      GemmNT g{};
      g.M = nocc * nocc;
      g.N = nvirt * nvirt;
      g.K = naux;
      g.A = B->ijw.p;
      g.lda = B->ldq;
      g.B = stage.p;
      g.ldb = naux;
      g.C = cmat.p;
      g.ldc = nvirt * nvirt;
      g.batch = 1;
      g.alpha = 1.0;
      g.beta = 0.0;
      g.splitk = 0;
      gemm_nt_f64(ctx, g);
      DevArr amax;
      amax.alloc(1);
      QX_CUDA(cudaMemsetAsync(amax.p, 0, sizeof(double), ctx->stream));
      k_absmax<<<1184, 256, 0, ctx->stream>>>(cmat.p, (size_t)nov * nov,
                                              reinterpret_cast<unsigned long long*>(amax.p));
      check_launch(ctx);
      double bound = 0.0;
      QX_CUDA(cudaMemcpyAsync(&bound, amax.p, sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
      QX_CUDA(cudaStreamSynchronize(ctx->stream));
      // Power-of-two scale as in the other fp16 splits (largest entry in [2^14, 2^15)).
      const double s = (fp16 && bound > 0.0 && std::isfinite(bound)) ? std::exp2(std::floor(std::log2(32768.0 / bound)))
                                                                     : 1.0;
      B->ldg = round_up(nov, 8);
      const size_t ge = (size_t)nov * B->ldg;
      const size_t ghalf = ((ge * 2 + 255) / 256) * 256;
      B->kd_split.alloc((2 * ghalf + 7) / 8 + 64);
      uint16_t* gs = reinterpret_cast<uint16_t*>(B->kd_split.p);
      if (fp16)
        k_kd_split<true><<<nov, 256, 0, ctx->stream>>>(cmat.p, nocc, nvirt, B->ldg, s, gs, gs + ghalf / 2);
      else
        k_kd_split<false><<<nov, 256, 0, ctx->stream>>>(cmat.p, nocc, nvirt, B->ldg, s, gs, gs + ghalf / 2);
      check_launch(ctx);
      const float sf = (float)s;
      B->kd_scale.alloc(1);
      QX_CUDA(cudaMemcpyAsync(B->kd_scale.p, &sf, sizeof(float), cudaMemcpyHostToDevice, ctx->stream));
      QX_CUDA(cudaStreamSynchronize(ctx->stream));  // cmat is freed on return
      B->kd = true;
    }
    B->dabT.alloc((size_t)nvirt * naux * B->ldvp);
    QX_CUDA(cudaMemsetAsync(B->dabT.p, 0, (size_t)nvirt * naux * B->ldvp * sizeof(double), ctx->stream));
    transpose(ctx, stage.p, nvirt, naux, naux, (size_t)nvirt * naux, B->dabT.p, B->ldvp, (size_t)naux * B->ldvp,
              nvirt);
    if (is_tc_precision(precision)) {
      // hi/lo of dabT with a power-of-two scale per virtual orbital a (kept).
      const size_t de = (size_t)nvirt * naux * B->ldvp;
      const size_t half = ((de * 2 + 255) / 256) * 256;
      B->dab_split.alloc((2 * half + 7) / 8 + 64);
      B->dab_scale.alloc((nvirt + 1) / 2 + 1);
      uint8_t* ds = reinterpret_cast<uint8_t*>(B->dab_split.p);
      float* sc = nullptr;
      launch_split(ctx, B->dabT.p, naux, nvirt, B->ldvp, ds, ds + half, B->ldvp, (size_t)naux * B->ldvp,
                   (size_t)naux * B->ldvp, nvirt, precision == QX_PREC_FP16X3, 2, &sc);
      QX_CUDA(cudaMemcpyAsync(B->dab_scale.p, sc, nvirt * sizeof(float), cudaMemcpyDeviceToDevice, ctx->stream));
    }
    sync_and_check(ctx);
  });
  if (st != QX_OK) {
    delete B;
    return st;
  }
  *out = B;
  return QX_OK;
}

qx_status qx_bse_destroy(qx_bse* B) {
  if (!B) return QX_OK;
  cudaSetDevice(B->ctx->device);
  cudaStreamSynchronize(B->ctx->stream);
  delete B;
  return QX_OK;
}

qx_status qx_bse_apply(qx_bse* B, const double* x, double* y, int nvec) {
  if (!B) return QX_ERR_INVALID_INPUT;
  return bse_guard(B->ctx, [&] {
    QX_REQUIRE(x && y && nvec > 0, QX_ERR_INVALID_INPUT, "invalid arguments to apply");
    qx_ctx* ctx = B->ctx;
    const int nov = B->nov;
    // x, y are [nov][nvec] (apply_tda_hamiltonian_batch layout).
    std::vector<double> hx((size_t)nov * nvec), hr((size_t)nvec * B->ldov, 0.0);
    QX_CUDA(cudaMemcpy(hx.data(), x, hx.size() * sizeof(double), cudaMemcpyDefault));
    for (double v : hx) QX_REQUIRE(std::isfinite(v), QX_ERR_NUMERICAL, "input vector contains NaN or Inf");
    for (int k = 0; k < nov; ++k)
      for (int v = 0; v < nvec; ++v) hr[(size_t)v * B->ldov + k] = hx[(size_t)k * nvec + v];
    B->Xr.alloc(hr.size());
    B->Yr.alloc(hr.size());
    QX_CUDA(cudaMemcpyAsync(B->Xr.p, hr.data(), hr.size() * sizeof(double), cudaMemcpyHostToDevice, ctx->stream));
    bse_apply_rows(B, B->Xr.p, B->Yr.p, nvec);
    QX_CUDA(cudaMemcpyAsync(hr.data(), B->Yr.p, hr.size() * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
    sync_and_check(ctx);
    for (int k = 0; k < nov; ++k)
      for (int v = 0; v < nvec; ++v) hx[(size_t)k * nvec + v] = hr[(size_t)v * B->ldov + k];
    for (double v : hx)
      QX_REQUIRE(std::isfinite(v), QX_ERR_NUMERICAL, "BSE Hamiltonian application produced non-finite values");
    QX_CUDA(cudaMemcpy(y, hx.data(), hx.size() * sizeof(double), cudaMemcpyDefault));
  });
}

// Davidson of davidson_bse (davidson.rs:372-508) on an n-dimensional operator
// whose vectors are rows of stride ld on the device: apply_rows(x, y, count)
// writes y[v] = H x[v] on the context stream; d_delta / h_delta are the QP
// gaps (the preconditioner's diagonal and the initial subspace's order).
static void davidson_run(qx_ctx* ctx, DavWork& W, int n, int ld, const double* d_delta,
                         const std::vector<double>& h_delta,
                         const std::function<void(const double*, double*, int)>& apply_rows,
                         const qx_davidson_config& cfg, double* eigenvalues, double* eigenvectors, int* converged_out,
                         double* residual_norms, int* iterations) {
  const int nroots = std::min(cfg.n_roots, n);
  const int max_space = std::min(cfg.max_space, n);
  QX_REQUIRE(nroots > 0 && eigenvalues && eigenvectors, QX_ERR_INVALID_INPUT, "invalid Davidson arguments");
  QX_REQUIRE(max_space <= 1024, QX_ERR_INVALID_INPUT, "max_space %d exceeds 1024", max_space);
  const int cap = std::max(max_space, nroots) + nroots + 1;
  W.V.alloc((size_t)cap * ld);
  W.AV.alloc((size_t)cap * ld);
  W.X.alloc((size_t)nroots * ld);
  W.AX.alloc((size_t)nroots * ld);
  W.R.alloc((size_t)nroots * ld);
  W.heff.alloc((size_t)cap * cap);
  W.jv.alloc(eigh_lowest_work_doubles(cap, cap));
  W.eigi.alloc(((size_t)cap * cap + 1) / 2 + 1);
  W.Z2.alloc((size_t)cap * cap);
  W.small.alloc((size_t)4 * cap + 64);
  double* d_theta = W.small.p;
  double* d_nrm = d_theta + cap;
  double* d_c = d_nrm + cap;
  QX_CUDA(cudaMemsetAsync(W.V.p, 0, (size_t)cap * ld * sizeof(double), ctx->stream));
  auto apply = [&](int first, int count) { apply_rows(W.V.p + (size_t)first * ld, W.AV.p + (size_t)first * ld, count); };
  auto rr = [&](int nv, int k) {
    // heff = V AV^T, then the lowest k eigenpairs of its symmetric part ->
    // theta, Z2 (columns).
    GemmNT g{};
    g.M = nv;
    g.N = nv;
    g.K = n;
    g.A = W.V.p;
    g.lda = ld;
    g.B = W.AV.p;
    g.ldb = ld;
    g.C = W.heff.p;
    g.ldc = nv;
    g.batch = 1;
    g.alpha = 1.0;
    g.splitk = 0;
    gemm_nt_f64(ctx, g);
    eigh_lowest(ctx, W.heff.p, nv, nv, k, d_theta, W.Z2.p, nv, W.jv.p, reinterpret_cast<int*>(W.eigi.p));
  };
  const int nthreads = 256, nblk = std::min(ceil_div(n, nthreads), 2 * ctx->sm_count);
  // The norm reductions run in one block of 1024 threads each, so that their
  // summation order (and the Davidson path) is the same on every run.
  constexpr int kRedThreads = 1024;
  // Trivial case (davidson.rs:384-387, 510-540): the full matrix.
  if (n <= nroots) {
    std::vector<double> id((size_t)n * ld, 0.0);
    for (int i = 0; i < n; ++i) id[(size_t)i * ld + i] = 1.0;
    QX_CUDA(cudaMemcpyAsync(W.V.p, id.data(), id.size() * sizeof(double), cudaMemcpyHostToDevice, ctx->stream));
    apply(0, n);
    rr(n, n);
    std::vector<double> th(n), zz((size_t)n * n);
    QX_CUDA(cudaMemcpyAsync(th.data(), d_theta, n * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
    QX_CUDA(cudaMemcpyAsync(zz.data(), W.Z2.p, zz.size() * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
    sync_and_check(ctx);
    std::vector<double> ev((size_t)n * nroots);
    for (int k = 0; k < n; ++k)
      for (int r = 0; r < nroots; ++r) ev[(size_t)k * nroots + r] = zz[(size_t)k * n + r];
    QX_CUDA(cudaMemcpy(eigenvalues, th.data(), nroots * sizeof(double), cudaMemcpyDefault));
    QX_CUDA(cudaMemcpy(eigenvectors, ev.data(), ev.size() * sizeof(double), cudaMemcpyDefault));
    if (converged_out)
      for (int r = 0; r < nroots; ++r) converged_out[r] = 1;
    if (residual_norms)
      for (int r = 0; r < nroots; ++r) residual_norms[r] = 0.0;
    if (iterations) *iterations = 1;
    return;
  }
  // Initial subspace: unit vectors at the smallest gaps (davidson.rs:157-176).
  std::vector<int> order(n);
  std::iota(order.begin(), order.end(), 0);
  std::stable_sort(order.begin(), order.end(), [&](int a, int b) { return h_delta[a] < h_delta[b]; });
  {
    std::vector<double> init((size_t)nroots * ld, 0.0);
    for (int i = 0; i < nroots; ++i) init[(size_t)i * ld + order[i]] = 1.0;
    QX_CUDA(cudaMemcpyAsync(W.V.p, init.data(), init.size() * sizeof(double), cudaMemcpyHostToDevice, ctx->stream));
  }
  int nv = nroots;
  apply(0, nv);
  std::vector<double> evals(nroots, 0.0), rnorm(nroots, std::numeric_limits<double>::max());
  std::vector<int> conv(nroots, 0);
  DevArr evecs;  // converged eigenvectors [nroots][ld]
  evecs.alloc((size_t)nroots * ld);
  QX_CUDA(cudaMemsetAsync(evecs.p, 0, (size_t)nroots * ld * sizeof(double), ctx->stream));
  int iter = 0;
  bool all = false;
  std::vector<double> th(cap), nr(cap);
  for (iter = 0; iter < cfg.max_iter; ++iter) {
    const int nr_ = std::min(nroots, nv);
    rr(nv, nr_);
    // Ritz vectors X = V Y, AX = AV Y.
    combine_rows(ctx, W.V.p, ld, nv, W.Z2.p, nv, nr_, n, W.X.p, ld, 1.0, 0.0);
    combine_rows(ctx, W.AV.p, ld, nv, W.Z2.p, nv, nr_, n, W.AX.p, ld, 1.0, 0.0);
    QX_CUDA(cudaMemsetAsync(d_nrm, 0, nr_ * sizeof(double), ctx->stream));
    k_residual<<<dim3(1, nr_), kRedThreads, 0, ctx->stream>>>(W.AX.p, W.X.p, d_theta, ld, n, W.R.p, d_nrm);
    check_launch(ctx);
    QX_CUDA(cudaMemcpyAsync(th.data(), d_theta, nr_ * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
    QX_CUDA(cudaMemcpyAsync(nr.data(), d_nrm, nr_ * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
    sync_and_check(ctx);
    std::vector<int> newr;
    for (int j = 0; j < nroots; ++j) {
      if (j >= nr_ || conv[j]) continue;
      const double res = std::sqrt(nr[j]);
      rnorm[j] = res;
      if (res < cfg.tol_residual) {
        conv[j] = 1;
        evals[j] = th[j];
        QX_CUDA(cudaMemcpyAsync(evecs.p + (size_t)j * ld, W.X.p + (size_t)j * ld, ld * sizeof(double),
                                cudaMemcpyDeviceToDevice, ctx->stream));
        continue;
      }
      newr.push_back(j);
    }
    all = std::all_of(conv.begin(), conv.end(), [](int c) { return c != 0; });
    if (all) {
      ++iter;
      break;
    }
    if (newr.empty()) continue;
    // Preconditioned residuals t_j (davidson.rs:444-449), staged after V.
    const int nnew = (int)newr.size();
    for (int q = 0; q < nnew; ++q) {
      const int j = newr[q];
      double* t = W.V.p + (size_t)(nv + q) * ld;
      QX_CUDA(cudaMemsetAsync(d_c, 0, sizeof(double), ctx->stream));
      k_precond<<<1, kRedThreads, 0, ctx->stream>>>(W.R.p + (size_t)j * ld, d_delta, th[j], cfg.level_shift, n,
                                                    t, d_c);
      check_launch(ctx);
      k_normalize<<<nblk, nthreads, 0, ctx->stream>>>(t, n, d_c, 1e-14);
      check_launch(ctx);
    }
    if (nv + nnew > max_space) {
      // Restart from the Ritz vectors, re-orthonormalised (davidson.rs:298-307).
      QX_CUDA(cudaMemcpyAsync(W.V.p, W.X.p, (size_t)nr_ * ld * sizeof(double), cudaMemcpyDeviceToDevice,
                              ctx->stream));
      for (int i = 0; i < nr_; ++i) {
        double* v = W.V.p + (size_t)i * ld;
        for (int pass = 0; pass < 2 && i > 0; ++pass) {
          GemmNT g{};
          g.M = i;
          g.N = 1;
          g.K = n;
          g.A = W.V.p;
          g.lda = ld;
          g.B = v;
          g.ldb = ld;
          g.C = d_c;
          g.ldc = 1;
          g.batch = 1;
          g.alpha = 1.0;
          g.splitk = 0;
          gemm_nt_f64(ctx, g);
          combine_rows(ctx, W.V.p, ld, i, d_c, 1, 1, n, v, ld, -1.0, 1.0);
        }
        QX_CUDA(cudaMemsetAsync(d_nrm, 0, sizeof(double), ctx->stream));
        k_norm2<<<1, kRedThreads, 0, ctx->stream>>>(v, n, d_nrm);
        check_launch(ctx);
        k_normalize<<<nblk, nthreads, 0, ctx->stream>>>(v, n, d_nrm, -1.0);
        check_launch(ctx);
      }
      nv = nr_;
      QX_CUDA(cudaMemsetAsync(W.V.p + (size_t)nv * ld, 0, (size_t)(cap - nv) * ld * sizeof(double), ctx->stream));
      apply(0, nv);
      continue;
    }
    // Double Gram-Schmidt of each candidate against the subspace (davidson.rs:240-285).
    int added = 0;
    for (int q = 0; q < nnew; ++q) {
      double* src = W.V.p + (size_t)(nv + q) * ld;
      double* dst = W.V.p + (size_t)(nv + added) * ld;
      if (src != dst)
        QX_CUDA(cudaMemcpyAsync(dst, src, ld * sizeof(double), cudaMemcpyDeviceToDevice, ctx->stream));
      const int cur = nv + added;
      for (int pass = 0; pass < 2; ++pass) {
        GemmNT g{};
        g.M = cur;
        g.N = 1;
        g.K = n;
        g.A = W.V.p;
        g.lda = ld;
        g.B = dst;
        g.ldb = ld;
        g.C = d_c;
        g.ldc = 1;
        g.batch = 1;
        g.alpha = 1.0;
        g.splitk = 0;
        gemm_nt_f64(ctx, g);
        combine_rows(ctx, W.V.p, ld, cur, d_c, 1, 1, n, dst, ld, -1.0, 1.0);
      }
      QX_CUDA(cudaMemsetAsync(d_nrm, 0, sizeof(double), ctx->stream));
      k_norm2<<<1, kRedThreads, 0, ctx->stream>>>(dst, n, d_nrm);
      check_launch(ctx);
      double h2 = 0.0;
      QX_CUDA(cudaMemcpyAsync(&h2, d_nrm, sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
      sync_and_check(ctx);
      if (std::sqrt(h2) < cfg.lindep_threshold) continue;
      k_normalize<<<nblk, nthreads, 0, ctx->stream>>>(dst, n, d_nrm, -1.0);
      check_launch(ctx);
      ++added;
    }
    QX_CUDA(cudaMemsetAsync(W.V.p + (size_t)(nv + added) * ld, 0, (size_t)(cap - nv - added) * ld * sizeof(double),
                            ctx->stream));
    if (added > 0) apply(nv, added);
    nv += added;
  }
  // Not converged: the latest Ritz approximation for roots never stored
  // (davidson.rs:480-496).
  if (!all) {
    const int nr_ = std::min(nroots, nv);
    rr(nv, nr_);
    combine_rows(ctx, W.V.p, ld, nv, W.Z2.p, nv, nr_, n, W.X.p, ld, 1.0, 0.0);
    QX_CUDA(cudaMemcpyAsync(th.data(), d_theta, nr_ * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
    sync_and_check(ctx);
    for (int j = 0; j < nr_; ++j)
      if (!conv[j]) {
        evals[j] = th[j];
        QX_CUDA(cudaMemcpyAsync(evecs.p + (size_t)j * ld, W.X.p + (size_t)j * ld, ld * sizeof(double),
                                cudaMemcpyDeviceToDevice, ctx->stream));
      }
    iter = cfg.max_iter;
  }
  std::vector<double> hv((size_t)nroots * ld), ev((size_t)n * nroots);
  QX_CUDA(cudaMemcpyAsync(hv.data(), evecs.p, hv.size() * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
  sync_and_check(ctx);
  for (int k = 0; k < n; ++k)
    for (int r = 0; r < nroots; ++r) ev[(size_t)k * nroots + r] = hv[(size_t)r * ld + k];
  QX_CUDA(cudaMemcpy(eigenvalues, evals.data(), nroots * sizeof(double), cudaMemcpyDefault));
  QX_CUDA(cudaMemcpy(eigenvectors, ev.data(), ev.size() * sizeof(double), cudaMemcpyDefault));
  if (converged_out)
    for (int r = 0; r < nroots; ++r) converged_out[r] = conv[r];
  if (residual_norms)
    for (int r = 0; r < nroots; ++r) residual_norms[r] = rnorm[r];
  if (iterations) *iterations = iter;
}

qx_status qx_bse_davidson(qx_bse* B, const qx_davidson_config* cfgp, double* eigenvalues, double* eigenvectors,
                          int* converged_out, double* residual_norms, int* iterations) {
  if (!B || !cfgp) return QX_ERR_INVALID_INPUT;
  return bse_guard(B->ctx, [&] {
    davidson_run(B->ctx, B->dav, B->nov, B->ldov, B->delta.p, B->h_delta,
                 [&](const double* x, double* y, int count) { bse_apply_rows(B, x, y, count); }, *cfgp, eigenvalues,
                 eigenvectors, converged_out, residual_norms, iterations);
  });
}

qx_status qx_davidson(qx_ctx* ctx, int n, const double* qp_gaps, qx_apply_fn apply_h, void* user,
                      const qx_davidson_config* cfgp, double* eigenvalues, double* eigenvectors, int* converged_out,
                      double* residual_norms, int* iterations) {
  if (!ctx || !cfgp || !apply_h) return QX_ERR_INVALID_INPUT;
  return bse_guard(ctx, [&] {
    QX_REQUIRE(n > 0 && qp_gaps, QX_ERR_INVALID_INPUT, "davidson needs n > 0 (got %d) and qp_gaps", n);
    const int ld = round_up(n, 8);
    std::vector<double> h(n);
    QX_CUDA(cudaMemcpy(h.data(), qp_gaps, n * sizeof(double), cudaMemcpyDefault));
    for (double v : h) QX_REQUIRE(std::isfinite(v), QX_ERR_INVALID_INPUT, "qp_gaps contains NaN or Inf");
    DevArr d;
    d.alloc(ld);
    QX_CUDA(cudaMemsetAsync(d.p, 0, ld * sizeof(double), ctx->stream));
    upload(ctx, d.p, h.data(), n);
    DavWork W;
    davidson_run(ctx, W, n, ld, d.p, h,
                 [&](const double* x, double* y, int count) {
                   sync_and_check(ctx);
                   const int rc = apply_h(user, x, y, count, ld);
                   QX_CUDA(cudaDeviceSynchronize());
                   QX_REQUIRE(rc == 0, (rc > 0 && rc <= (int)QX_ERR_NO_DEVICE) ? (qx_status)rc : QX_ERR_INVALID_INPUT,
                              "apply_h returned %d", rc);
                 },
                 *cfgp, eigenvalues, eigenvectors, converged_out, residual_norms, iterations);
  });
}

static void gemm_nt(qx_ctx* ctx, int M, int N, int K, const double* A, int lda, const double* Bm, int ldb, double* C,
                    int ldc) {
  GemmNT g{};
  g.M = M;
  g.N = N;
  g.K = K;
  g.A = A;
  g.lda = lda;
  g.B = Bm;
  g.ldb = ldb;
  g.C = C;
  g.ldc = ldc;
  g.batch = 1;
  g.alpha = 1.0;
  g.beta = 0.0;
  g.splitk = 0;
  gemm_nt_f64(ctx, g);
}

}  // extern "C"

// grad_ia[ia][P] = 2 alpha_x x_ia u_P - c_ia U[ia][P], u = B_ia^T x; c_ia = 8 / e_ia
// (e_ia = e_i - e_a) when W0's dependence on B_ia is included, else 0.
__global__ void k_grad_ia(const double* __restrict__ x, const double* __restrict__ u,
                          const double* __restrict__ U, int ldu, const double* __restrict__ c, int nov, int naux,
                          double alpha_x, double* __restrict__ out) {
  for (size_t k = (size_t)blockIdx.x * blockDim.x + threadIdx.x; k < (size_t)nov * naux;
       k += (size_t)gridDim.x * blockDim.x) {
    const int ia = (int)(k / naux), P = (int)(k % naux);
    double g = 2.0 * alpha_x * x[ia] * u[P];
    if (c) g -= c[ia] * U[(size_t)ia * ldu + P];
    out[k] = g;
  }
}

// out[r][c] = in[r][c] for c < cols (drops the row padding).
__global__ void k_unpad(const double* __restrict__ in, size_t rows, int cols, int ld, double* __restrict__ out) {
  for (size_t k = (size_t)blockIdx.x * blockDim.x + threadIdx.x; k < rows * cols; k += (size_t)gridDim.x * blockDim.x)
    out[k] = in[(k / cols) * ld + k % cols];
}

// Gradients of a root Omega = x^T H x (|x| = 1, Hellmann-Feynman) of the
// kernel's matrix with respect to the orbital energies and, when requested,
// to the DF blocks df_ia, df_ij, df_ab as given to qx_bse_create:
//   H = diag(Delta) + alpha_x B_ia B_ia^T - K^d,  K^d_(ia)(jb) = sum_PQ B_ij^P W0_PQ B_ab^Q.
// With T'^Q_ij = sum_ab x_ia B_ab^Q x_jb and M_PQ = sum_ij B_ij^P T'^Q_ij:
//   dOmega/dB_ij^P = -(T' W0)_(ij)P,
//   dOmega/dB_ab^Q = -sum_ij x_ia (B_ij W0)^Q_ij x_jb,
//   dOmega/dB_ia^P = 2 alpha_x x_ia (B_ia^T x)_P [- 8 / e_ia (B_ia G)_P],
// the bracket (with G = W0 sym(M) W0) when W0 = (I - Pi(0))^-1 follows B_ia
// (mo_energy given), as for the energies: dW0 = W0 dPi W0, Pi(0) = 4 sum_ia
// B_ia B_ia^T / e_ia.
static void bse_root_grad_impl(qx_bse* B, const double* x, const double* mo_energy, double* grad_energy,
                               double* grad_ia, double* grad_ij, double* grad_ab) {
  {
    qx_ctx* ctx = B->ctx;
    const int nocc = B->nocc, nvir = B->nvir, naux = B->naux, nov = B->nov, ldq = B->ldq, ldvp = B->ldvp;
    std::vector<double> hx(nov);
    QX_CUDA(cudaMemcpy(hx.data(), x, nov * sizeof(double), cudaMemcpyDefault));
    double n2 = 0.0;
    for (double v : hx) n2 += v * v;
    QX_REQUIRE(n2 > 0.0 && std::isfinite(n2), QX_ERR_NUMERICAL, "eigenvector has zero or non-finite norm");
    for (double& v : hx) v /= std::sqrt(n2);
    // Delta_ia = e_a - e_i.
    std::vector<double> g(nocc + nvir, 0.0);
    for (int i = 0; i < nocc; ++i)
      for (int a = 0; a < nvir; ++a) {
        const double w = hx[(size_t)i * nvir + a] * hx[(size_t)i * nvir + a];
        g[i] -= w;
        g[nocc + a] += w;
      }
    const bool want_b = grad_ia || grad_ij || grad_ab;
    const int nq = nocc * ldq, n2o = nocc * nocc, ld2 = round_up(n2o, 8);
    std::vector<double> e;
    if (mo_energy) {
      e.resize(nocc + nvir);
      QX_CUDA(cudaMemcpy(e.data(), mo_energy, e.size() * sizeof(double), cudaMemcpyDefault));
    }
    if (mo_energy || want_b) {
      // T[a][j][Q] = sum_b x[j][b] B_ab^Q: the first step of the matvec (nvec = 1).
      std::vector<double> hr(B->ldov, 0.0);
      std::copy(hx.begin(), hx.end(), hr.begin());
      B->Xr.alloc(B->ldov);
      B->Yr.alloc(B->ldov);
      QX_CUDA(cudaMemcpyAsync(B->Xr.p, hr.data(), B->ldov * sizeof(double), cudaMemcpyHostToDevice, ctx->stream));
      bse_apply_rows(B, B->Xr.p, B->Yr.p, 1, /*need_T=*/true);
      // T'[(i,j)][Q] = sum_a x[i][a] T[a][(j,Q)]
      B->gTt.alloc((size_t)nq * ldvp);
      QX_CUDA(cudaMemsetAsync(B->gTt.p, 0, (size_t)nq * ldvp * sizeof(double), ctx->stream));
      transpose(ctx, B->T.p, nvir, nq, nq, 0, B->gTt.p, ldvp, 0, 1);
      B->gTp.alloc((size_t)n2o * ldq);
      gemm_nt(ctx, nocc, nq, nvir, B->xp.p, ldvp, B->gTt.p, ldvp, B->gTp.p, nq);
    }
    if (mo_energy) {
      // M[P][Q] = sum_(ij) B_ij^P T'[(ij)][Q]
      B->gdijT.alloc((size_t)naux * ld2);
      B->gTpT.alloc((size_t)ldq * ld2);
      QX_CUDA(cudaMemsetAsync(B->gdijT.p, 0, (size_t)naux * ld2 * sizeof(double), ctx->stream));
      QX_CUDA(cudaMemsetAsync(B->gTpT.p, 0, (size_t)ldq * ld2 * sizeof(double), ctx->stream));
      transpose(ctx, B->dij.p, n2o, naux, ldq, 0, B->gdijT.p, ld2, 0, 1);
      transpose(ctx, B->gTp.p, n2o, naux, ldq, 0, B->gTpT.p, ld2, 0, 1);
      B->gM.alloc((size_t)naux * ldq);
      gemm_nt(ctx, naux, naux, n2o, B->gdijT.p, ld2, B->gTpT.p, ld2, B->gM.p, ldq);
      k_symmetrize<<<std::min(ceil_div(naux * naux, 256), 4096), 256, 0, ctx->stream>>>(B->gM.p, naux, ldq);
      check_launch(ctx);
      // G = W0 sym(M) W0 (W0 symmetric, stored as its transpose)
      B->gG1.alloc((size_t)naux * ldq);
      B->gG.alloc((size_t)naux * ldq);
      gemm_nt(ctx, naux, naux, naux, B->w0T.p, ldq, B->gM.p, ldq, B->gG1.p, ldq);
      gemm_nt(ctx, naux, naux, naux, B->gG1.p, ldq, B->w0T.p, ldq, B->gG.p, ldq);
      // s_ia = b_ia^T G b_ia
      B->gU.alloc((size_t)nov * ldq + nov);
      gemm_nt(ctx, nov, naux, naux, B->dia.p, ldq, B->gG.p, ldq, B->gU.p, ldq);
      double* d_s = B->gU.p + (size_t)nov * ldq;
      k_rowdot<<<ceil_div(nov * 32, 256), 256, 0, ctx->stream>>>(B->gU.p, B->dia.p, nov, naux, ldq, d_s);
      check_launch(ctx);
      std::vector<double> sv(nov);
      QX_CUDA(cudaMemcpyAsync(sv.data(), d_s, nov * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
      sync_and_check(ctx);
      for (int i = 0; i < nocc; ++i)
        for (int a = 0; a < nvir; ++a) {
          const double d = e[nocc + a] - e[i];
          const double gd = sv[(size_t)i * nvir + a] * (-4.0 / (d * d));
          g[i] -= gd;
          g[nocc + a] += gd;
        }
    }
    if (grad_energy) QX_CUDA(cudaMemcpy(grad_energy, g.data(), g.size() * sizeof(double), cudaMemcpyDefault));
    if (!want_b) return;
    // Scratch for the block gradients: u, c, the padded ij and ab results.
    const int ldo8 = round_up(nocc, 8);
    DevArr& gs = B->gGrad;
    const size_t n_u = ldq, n_c = B->ldov, n_ij = (size_t)n2o * ldq, n_xt = (size_t)nvir * ldo8,
                 n_ut = (size_t)nocc * naux * ldo8, n_v = (size_t)nocc * nvir * ldq, n_vt = (size_t)nvir * ldq * ldo8,
                 n_ab = (size_t)nvir * nvir * ldq, n_out = std::max({(size_t)nov, (size_t)n2o, (size_t)nvir * nvir}) * naux;
    gs.alloc(n_u + n_c + n_ij + n_xt + n_ut + n_v + n_vt + n_ab + n_out + 64);
    double* u = gs.p;
    double* cia = u + n_u;
    double* gij = cia + n_c;
    double* xt = gij + n_ij;
    double* ut = xt + n_xt;
    double* v = ut + n_ut;
    double* vt = v + n_v;
    double* gab = vt + n_vt;
    double* outb = gab + n_ab;
    auto copy_out = [&](const double* src, size_t rows, int ld, double* dst) {
      const double* s = src;
      if (ld != naux) {
        k_unpad<<<(unsigned)std::min<size_t>((rows * naux + 255) / 256, 8192), 256, 0, ctx->stream>>>(src, rows, naux,
                                                                                                     ld, outb);
        check_launch(ctx);
        s = outb;
      }
      QX_CUDA(cudaMemcpyAsync(dst, s, rows * naux * sizeof(double), cudaMemcpyDefault, ctx->stream));
      sync_and_check(ctx);  // outb is reused by the next block
    };
    if (grad_ia) {
      // u[P] = sum_ia x_ia B_ia^P.
      GemmNT gu{};
      gu.M = 1;
      gu.N = naux;
      gu.K = nov;
      gu.A = B->Xr.p;
      gu.lda = B->ldov;
      gu.B = B->diaT.p;
      gu.ldb = B->ldov;
      gu.C = u;
      gu.ldc = ldq;
      gu.batch = 1;
      gu.alpha = 1.0;
      gu.splitk = 0;
      gemm_nt_f64(ctx, gu);
      const double* cptr = nullptr;
      if (mo_energy) {
        std::vector<double> hc(nov);
        for (int i = 0; i < nocc; ++i)
          for (int a = 0; a < nvir; ++a) hc[(size_t)i * nvir + a] = 8.0 / (e[i] - e[nocc + a]);
        QX_CUDA(cudaMemcpyAsync(cia, hc.data(), nov * sizeof(double), cudaMemcpyHostToDevice, ctx->stream));
        cptr = cia;
      }
      k_grad_ia<<<(unsigned)std::min<size_t>(((size_t)nov * naux + 255) / 256, 8192), 256, 0, ctx->stream>>>(
          B->Xr.p, u, B->gU.p, ldq, cptr, nov, naux, B->alpha_x, outb);
      check_launch(ctx);
      QX_CUDA(cudaMemcpyAsync(grad_ia, outb, (size_t)nov * naux * sizeof(double), cudaMemcpyDefault, ctx->stream));
      sync_and_check(ctx);
    }
    if (grad_ij) {
      // grad_ij[(ij)][P] = -sum_Q T'[(ij)][Q] W0[Q][P]  (w0T rows are W0's columns).
      GemmNT gg{};
      gg.M = n2o;
      gg.N = naux;
      gg.K = naux;
      gg.A = B->gTp.p;
      gg.lda = ldq;
      gg.B = B->w0T.p;
      gg.ldb = ldq;
      gg.C = gij;
      gg.ldc = ldq;
      gg.batch = 1;
      gg.alpha = -1.0;
      gg.splitk = 0;
      gemm_nt_f64(ctx, gg);
      copy_out(gij, n2o, ldq, grad_ij);
    }
    if (grad_ab) {
      // x^T [b][j] and U^T[i][Q][j] with U = ijw = B_ij W0 ([(i,j)][Q]).
      QX_CUDA(cudaMemsetAsync(xt, 0, n_xt * sizeof(double), ctx->stream));
      QX_CUDA(cudaMemsetAsync(ut, 0, n_ut * sizeof(double), ctx->stream));
      transpose(ctx, B->xp.p, nocc, nvir, ldvp, 0, xt, ldo8, 0, 1);
      transpose(ctx, B->ijw.p, nocc, naux, ldq, (size_t)nocc * ldq, ut, ldo8, (size_t)naux * ldo8, nocc);
      // V[i][b][Q] = sum_j x[j][b] U[(i,j)][Q]
      GemmNT ga{};
      ga.M = nvir;
      ga.N = naux;
      ga.K = nocc;
      ga.A = xt;
      ga.lda = ldo8;
      ga.sA = 0;
      ga.B = ut;
      ga.ldb = ldo8;
      ga.sB = (size_t)naux * ldo8;
      ga.C = v;
      ga.ldc = ldq;
      ga.sC = (size_t)nvir * ldq;
      ga.batch = nocc;
      ga.alpha = 1.0;
      ga.splitk = 1;
      gemm_nt_f64(ctx, ga);
      // grad_ab[a][(b,Q)] = -sum_i x[i][a] V[i][(b,Q)]
      QX_CUDA(cudaMemsetAsync(vt, 0, n_vt * sizeof(double), ctx->stream));
      transpose(ctx, v, nocc, nvir * ldq, nvir * ldq, 0, vt, ldo8, 0, 1);
      GemmNT gb{};
      gb.M = nvir;
      gb.N = nvir * ldq;
      gb.K = nocc;
      gb.A = xt;
      gb.lda = ldo8;
      gb.B = vt;
      gb.ldb = ldo8;
      gb.C = gab;
      gb.ldc = nvir * ldq;
      gb.batch = 1;
      gb.alpha = -1.0;
      gb.splitk = 1;
      gemm_nt_f64(ctx, gb);
      copy_out(gab, (size_t)nvir * nvir, ldq, grad_ab);
    }
  }
}

extern "C" {

qx_status qx_bse_root_grad(qx_bse* B, const double* x, const double* mo_energy, double* grad_energy) {
  if (!B) return QX_ERR_INVALID_INPUT;
  return bse_guard(B->ctx, [&] {
    QX_REQUIRE(x && grad_energy, QX_ERR_INVALID_INPUT, "invalid arguments to bse_root_grad");
    bse_root_grad_impl(B, x, mo_energy, grad_energy, nullptr, nullptr, nullptr);
  });
}

qx_status qx_bse_root_grad_b(qx_bse* B, const double* x, const double* mo_energy, double* grad_energy,
                             double* grad_ia, double* grad_ij, double* grad_ab) {
  if (!B) return QX_ERR_INVALID_INPUT;
  return bse_guard(B->ctx, [&] {
    QX_REQUIRE(x && (grad_energy || grad_ia || grad_ij || grad_ab), QX_ERR_INVALID_INPUT,
               "invalid arguments to bse_root_grad_b");
    bse_root_grad_impl(B, x, mo_energy, grad_energy, grad_ia, grad_ij, grad_ab);
  });
}

qx_status qx_bse_w0(qx_ctx* ctx, const double* mo_energy, const double* lpq_ov, int naux, int nocc, int nvir,
                    double* w0) {
  if (!ctx) return QX_ERR_INVALID_INPUT;
  return bse_guard(ctx, [&] {
    QX_REQUIRE(mo_energy && lpq_ov && w0 && naux > 0 && nocc > 0 && nvir > 0, QX_ERR_INVALID_INPUT,
               "invalid arguments to bse_w0");
    const int nov = nocc * nvir, ldov = round_up(nov, 8), ldn = round_up(naux, 8);
    const double* d_lov = (const double*)device_view(ctx, WS_LPQ, lpq_ov, (size_t)naux * nov * sizeof(double));
    ctx->ws[WS_SMALL].reserve((nocc + nvir + 8) * sizeof(double));
    double* d_e = ctx->ws[WS_SMALL].as<double>();
    double* d_f = d_e + nocc + nvir;
    QX_CUDA(cudaMemcpyAsync(d_e, mo_energy, (nocc + nvir) * sizeof(double), cudaMemcpyDefault, ctx->stream));
    QX_CUDA(cudaMemsetAsync(d_f, 0, sizeof(double), ctx->stream));
    ctx->ws[WS_BOV].reserve((size_t)naux * ldov * sizeof(double));
    double* bov = ctx->ws[WS_BOV].as<double>();
    QX_CUDA(cudaMemcpy2DAsync(bov, ldov * sizeof(double), d_lov, nov * sizeof(double), nov * sizeof(double), naux,
                              cudaMemcpyDeviceToDevice, ctx->stream));
    if (ldov > nov)
      QX_CUDA(cudaMemset2DAsync(bov + nov, ldov * sizeof(double), 0, (ldov - nov) * sizeof(double), naux, ctx->stream));
    ctx->ws[WS_CHI].reserve((size_t)ldov * sizeof(double));
    double* chi = ctx->ws[WS_CHI].as<double>();
    const size_t stride = (size_t)naux * ldn;
    ctx->ws[WS_EPS].reserve(stride * sizeof(double));
    double* eps = ctx->ws[WS_EPS].as<double>();
    launch_chi(ctx, d_e, nocc, nvir, d_f, 1, 0, chi, ldov);
    launch_eps_fp64(ctx, bov, ldov, naux, nov, chi, 1, eps, ldn, stride);
    std::vector<double> he(nocc + nvir);
    QX_CUDA(cudaMemcpy(he.data(), mo_energy, (nocc + nvir) * sizeof(double), cudaMemcpyDefault));
    launch_invert_wc(ctx, eps, naux, ldn, stride, 1, !eps_at_least_identity(he.data(), nocc, nvir, 0.0));
    std::vector<double> h(stride);
    QX_CUDA(cudaMemcpyAsync(h.data(), eps, stride * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
    sync_and_check(ctx);
    std::vector<double> out((size_t)naux * naux);
    for (int r = 0; r < naux; ++r)
      for (int c = 0; c < naux; ++c) out[(size_t)r * naux + c] = h[(size_t)r * ldn + c] + (r == c ? 1.0 : 0.0);
    QX_CUDA(cudaMemcpy(w0, out.data(), out.size() * sizeof(double), cudaMemcpyDefault));
  });
}

}  // extern "C"
