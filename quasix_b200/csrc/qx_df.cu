// Density-fitting tensors on the device: the MO transform of the
// three-centre integrals and the RI normalisation by the inverse square root
// of the Coulomb metric, producing lpq[P][p][q] -- the tensor every GW and BSE
// entry point of this library takes.
//
// Reference: quasix/quasix/evgw.py:1007-1100 (J^-1/2 from eigh(metric) with
// eigenvalues clamped at thresh_df, then C^T (uv|P) C per P) and the Rust
// transform_mo_3center (quasix_core/src/df/mo_transform.rs:136-282, the ov
// block [nocc*nvir][naux]).
//
// Layout and order.  The caller's (uv|P) is [nao][nao][naux] (P fastest, the
// layout of PySCF's aux_e2 reshaped and of the Rust j3c_ao).  It is first
// transposed to X[P][u][v] (rows padded to 8 doubles), so that both MO
// transforms are batched FP64 DMMA GEMMs over P with the contraction index
// contiguous:
//   T[P][p][v]  = sum_u C[u][p] X[P][v][u]      (X[P] symmetric in u, v)
//   L'[P][p][q] = sum_v T[P][p][v] C[v][q]
// The metric step lpq[P][pq] = sum_Q J^-1/2[P][Q] L'[Q][pq] is one GEMM with
// L' transposed to [pq][Q].  The MO transform runs before the metric step
// (the reference does it after): the two are linear and commute, and this
// order contracts the metric over nmo^2 instead of nao^2 columns.
//
// J^-1/2 and J^1/2 come from the scaled Denman-Beavers iteration (product
// form, see metric_inv_sqrt: one SPD inverse by the block sweep refined by a
// Newton-Schulz step, and four DMMA GEMMs per step, 5-8 steps); it equals the
// eigendecomposition form of the reference whenever no eigenvalue of J lies
// below thresh_df.  That is checked with lambda_min(J) >= 1 / trace(J^-1)
// and, when this bound is inconclusive, by power iteration on J^-1/2 (the
// reference's clamping of such eigenvalues is not reproduced: those metrics
// are rejected with QX_ERR_NUMERICAL).
#include <algorithm>

#include "qx_blas.cuh"
#include "qx_internal.cuh"

namespace qx {
namespace {

size_t a256(size_t b) { return (b + 255) & ~size_t(255); }

// X[P][u][v] (row stride ldx, zero padding) = j3c[u][v][P] through 32 x 32
// shared-memory tiles of the (uv) x P matrix.  grid (ceil(naux/32), y).
__global__ void k_aux_major(const double* __restrict__ j3c, int nao, int naux, double* __restrict__ X, int ldx) {
  __shared__ double t[32][33];
  const long long rows = (long long)nao * nao;
  const int c0 = blockIdx.x * 32;
  for (long long r0 = (long long)blockIdx.y * 32; r0 < rows; r0 += (long long)gridDim.y * 32) {
    __syncthreads();
    for (int y = threadIdx.y; y < 32; y += blockDim.y) {
      const long long r = r0 + y;
      const int c = c0 + threadIdx.x;
      t[y][threadIdx.x] = (r < rows && c < naux) ? j3c[r * naux + c] : 0.0;
    }
    __syncthreads();
    for (int y = threadIdx.y; y < 32; y += blockDim.y) {
      const int c = c0 + y;
      const long long r = r0 + threadIdx.x;
      if (c < naux && r < rows) {
        const int u = (int)(r / nao), v = (int)(r % nao);
        X[(size_t)c * nao * ldx + (size_t)u * ldx + v] = t[threadIdx.x][y];
      }
    }
  }
}

// out[P][q] (row stride ldo) = in[q][P] for a [rows][cols] input with row
// stride ldi: the generic tile transpose with grid-stride rows.
__global__ void k_transpose_gs(const double* __restrict__ in, long long rows, int cols, int ldi,
                               double* __restrict__ out, long long ldo) {
  __shared__ double t[32][33];
  const int c0 = blockIdx.x * 32;
  for (long long r0 = (long long)blockIdx.y * 32; r0 < rows; r0 += (long long)gridDim.y * 32) {
    __syncthreads();
    for (int y = threadIdx.y; y < 32; y += blockDim.y) {
      const long long r = r0 + y;
      const int c = c0 + threadIdx.x;
      t[y][threadIdx.x] = (r < rows && c < cols) ? in[r * ldi + c] : 0.0;
    }
    __syncthreads();
    for (int y = threadIdx.y; y < 32; y += blockDim.y) {
      const int c = c0 + y;
      const long long r = r0 + threadIdx.x;
      if (c < cols && r < rows) out[(size_t)c * ldo + r] = t[threadIdx.x][y];
    }
  }
}

void transpose_gs(qx_ctx* ctx, const double* in, long long rows, int cols, int ldi, double* out, long long ldo) {
  const long long rb = (rows + 31) / 32;
  dim3 grid(ceil_div(cols, 32), (unsigned)std::min<long long>(rb, 16384));
  k_transpose_gs<<<grid, dim3(32, 8), 0, ctx->stream>>>(in, rows, cols, ldi, out, ldo);
  check_launch(ctx);
}

// out = s * in (+ t I) over the n x n part (row stride ld); padding untouched.
__global__ void k_axpi(const double* __restrict__ in, int n, int ldi, double s, double t, double* __restrict__ out,
                       int ldo) {
  for (size_t e = (size_t)blockIdx.x * blockDim.x + threadIdx.x; e < (size_t)n * n;
       e += (size_t)gridDim.x * blockDim.x) {
    const size_t r = e / n, c = e % n;
    out[r * ldo + c] = s * in[r * ldi + c] + (r == c ? t : 0.0);
  }
}

// M <- (I + (a M + b Mi) / 2) / 2, symmetrised (each thread owns the pair
// (r, c), (c, r) with c <= r), and *res = max |M - I| (bits).
__global__ void k_db_m(double* __restrict__ M, const double* __restrict__ Mi, int n, int ld, double a, double b,
                       unsigned long long* __restrict__ res) {
  double m = 0.0;
  for (size_t e = (size_t)blockIdx.x * blockDim.x + threadIdx.x; e < (size_t)n * n;
       e += (size_t)gridDim.x * blockDim.x) {
    const size_t r = e / n, c = e % n;
    if (c > r) continue;
    const double id = (r == c) ? 1.0 : 0.0;
    const double v1 = 0.5 * (id + 0.5 * (a * M[r * ld + c] + b * Mi[r * ld + c]));
    const double v2 = 0.5 * (id + 0.5 * (a * M[c * ld + r] + b * Mi[c * ld + r]));
    const double v = 0.5 * (v1 + v2);
    M[r * ld + c] = v;
    M[c * ld + r] = v;
    m = fmax(m, isfinite(v) ? fabs(v - id) : INFINITY);
  }
  for (int o = 16; o > 0; o >>= 1) m = fmax(m, __shfl_xor_sync(0xffffffffu, m, o));
  if ((threadIdx.x & 31) == 0) atomicMax(res, (unsigned long long)__double_as_longlong(m));
}

// One Newton-Schulz step of an approximate inverse Mi of M: Mi <- 2 Mi - X
// with X = Mi M Mi, symmetrised (each thread owns the pair (r, c), (c, r)).
__global__ void k_ns_step(double* __restrict__ Mi, const double* __restrict__ X, int n, int ld) {
  for (size_t e = (size_t)blockIdx.x * blockDim.x + threadIdx.x; e < (size_t)n * n;
       e += (size_t)gridDim.x * blockDim.x) {
    const size_t r = e / n, c = e % n;
    if (c > r) continue;
    const double v = 0.5 * ((2.0 * Mi[r * ld + c] - X[r * ld + c]) + (2.0 * Mi[c * ld + r] - X[c * ld + r]));
    Mi[r * ld + c] = v;
    Mi[c * ld + r] = v;
  }
}

// sum of squares (one atomic per warp into a double via bits is not
// order-free; a fixed two-pass reduction is used instead): part[b] per block.
__global__ void k_sumsq(const double* __restrict__ J, int n, int ldj, double* __restrict__ part) {
  double s = 0.0;
  for (size_t e = (size_t)blockIdx.x * blockDim.x + threadIdx.x; e < (size_t)n * n;
       e += (size_t)gridDim.x * blockDim.x) {
    const double v = J[(e / n) * ldj + e % n];
    s += v * v;
  }
  __shared__ double red[256];
  red[threadIdx.x] = s;
  __syncthreads();
  for (int o = 128; o > 0; o >>= 1) {
    if (threadIdx.x < o) red[threadIdx.x] += red[threadIdx.x + o];
    __syncthreads();
  }
  if (threadIdx.x == 0) part[blockIdx.x] = red[0];
}

// y = A x, one warp per row (power iteration on the symmetric J^-1/2).
__global__ void k_matvec(const double* __restrict__ A, int n, int ld, const double* __restrict__ x,
                         double* __restrict__ y) {
  const int lane = threadIdx.x & 31, nwarp = blockDim.x >> 5;
  for (int i = blockIdx.x * nwarp + (threadIdx.x >> 5); i < n; i += gridDim.x * nwarp) {
    double s = 0.0;
    for (int j = lane; j < n; j += 32) s += A[(size_t)i * ld + j] * x[j];
    for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    if (lane == 0) y[i] = s;
  }
}

// out[0] = x.y / x.x (the Rayleigh quotient of x with y = A x), x = y / |y|.
// One block of 1024 threads.
__global__ void k_power_norm(double* __restrict__ x, const double* __restrict__ y, int n, double* __restrict__ out) {
  __shared__ double r0[1024], r1[1024], r2[1024];
  double xx = 0.0, xy = 0.0, yy = 0.0;
  for (int i = threadIdx.x; i < n; i += blockDim.x) {
    xx += x[i] * x[i];
    xy += x[i] * y[i];
    yy += y[i] * y[i];
  }
  r0[threadIdx.x] = xx;
  r1[threadIdx.x] = xy;
  r2[threadIdx.x] = yy;
  __syncthreads();
  for (int o = blockDim.x / 2; o > 0; o >>= 1) {
    if (threadIdx.x < o) {
      r0[threadIdx.x] += r0[threadIdx.x + o];
      r1[threadIdx.x] += r1[threadIdx.x + o];
      r2[threadIdx.x] += r2[threadIdx.x + o];
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) out[0] = r1[0] / r0[0];
  const double inv = 1.0 / sqrt(r2[0]);
  for (int i = threadIdx.x; i < n; i += blockDim.x) x[i] = y[i] * inv;
}

// out = (in + in^T) / 2 over n x n (row stride ld).
__global__ void k_symmetrize(const double* __restrict__ in, int n, int ld, double* __restrict__ out) {
  for (size_t e = (size_t)blockIdx.x * blockDim.x + threadIdx.x; e < (size_t)n * n;
       e += (size_t)gridDim.x * blockDim.x) {
    const size_t r = e / n, c = e % n;
    out[r * ld + c] = 0.5 * (in[r * ld + c] + in[c * ld + r]);
  }
}

__global__ void k_scale_copy(const double* __restrict__ in, int n, int ldi, double s, double* __restrict__ out,
                             int ldo) {
  for (size_t e = (size_t)blockIdx.x * blockDim.x + threadIdx.x; e < (size_t)n * n;
       e += (size_t)gridDim.x * blockDim.x) {
    const size_t r = e / n, c = e % n;
    out[r * ldo + c] = s * in[r * ldi + c];
  }
}

void gemm(qx_ctx* ctx, int M, int N, int K, const double* A, int lda, size_t sA, const double* B, int ldb, size_t sB,
          double* C, int ldc, size_t sC, int batch) {
  GemmNT g{M, N, K, A, lda, sA, B, ldb, sB, C, ldc, sC, batch, 1.0, 0.0, 0};
  gemm_nt_f64(ctx, g);
}

// Frobenius norm of an n x n matrix (row stride ld), deterministic.
double frob(qx_ctx* ctx, const double* A, int n, int ld, double* part, int blocks) {
  k_sumsq<<<blocks, 256, 0, ctx->stream>>>(A, n, ld, part);
  check_launch(ctx);
  std::vector<double> h(blocks);
  QX_CUDA(cudaMemcpyAsync(h.data(), part, blocks * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
  QX_CUDA(cudaStreamSynchronize(ctx->stream));
  double s = 0.0;
  for (double v : h) s += v;
  return std::sqrt(s);
}

// J^-1/2 and J^1/2 ([n][ld] each, symmetrised) of the SPD metric J ([n][ldj],
// device), by the scaled product form of the Denman-Beavers iteration:
//   Mi = M^-1,  mu = (||Mi||_F / ||M||_F)^(1/4),  X = (I + Mi / mu^2) / 2,
//   Y <- mu Y X,  Z <- mu Z X,  M <- (I + (mu^2 M + Mi / mu^2) / 2) / 2,
// from M = Y = J, Z = I; M -> I, Y -> J^1/2, Z -> J^-1/2 (numerically stable;
// M stays SPD, so its inverse is the unguarded block sweep).  Returns a lower
// bound on the smallest eigenvalue of J that is tight whenever it is near
// thresh (1 / ||J^-1/2||_F^2, else the power iteration's
// 1 / lambda_max(J^-1/2)^2).
double metric_inv_sqrt(qx_ctx* ctx, const double* J, int n, int ldj, double* Jm, double* Jp, int ld, double* work,
                       double thresh) {
  const size_t nn = (size_t)n * ld;
  double* M = work;
  double* Mi = work + nn;
  double* X = work + 2 * nn;
  double* small = work + 3 * nn;  // [512] block partials | residual word | power vectors
  double* Y = Jp;
  double* Z = Jm;
  const int blocks = std::min<int>((int)((nn + 255) / 256), 2 * ctx->sm_count);
  QX_CUDA(cudaMemsetAsync(M, 0, 3 * nn * sizeof(double), ctx->stream));
  QX_CUDA(cudaMemsetAsync(Jm, 0, nn * sizeof(double), ctx->stream));
  QX_CUDA(cudaMemsetAsync(Jp, 0, nn * sizeof(double), ctx->stream));
  k_axpi<<<blocks, 256, 0, ctx->stream>>>(J, n, ldj, 1.0, 0.0, M, ld);
  check_launch(ctx);
  k_axpi<<<blocks, 256, 0, ctx->stream>>>(J, n, ldj, 1.0, 0.0, Y, ld);
  check_launch(ctx);
  k_axpi<<<blocks, 256, 0, ctx->stream>>>(J, n, ldj, 0.0, 1.0, Z, ld);
  check_launch(ctx);
  const double fj = frob(ctx, J, n, ldj, small, blocks);
  QX_REQUIRE(std::isfinite(fj) && fj > 0.0, QX_ERR_NUMERICAL, "metric is zero or not finite");
  unsigned long long* res = reinterpret_cast<unsigned long long*>(small + 512);
  // Scratch for the products: the work buffer after small.
  double* T = small + 520 + 2 * ((size_t)n + 8) + 64;
  bool done = false;
  double fmi0 = 0.0;  // ||J^-1||_F, from the first step
  for (int it = 0; it < 100 && !done; ++it) {
    // Mi = M^-1 (the sweep leaves M^-1 - I in place; M is SPD).
    QX_CUDA(cudaMemcpyAsync(Mi, M, nn * sizeof(double), cudaMemcpyDeviceToDevice, ctx->stream));
    launch_invert_wc(ctx, Mi, n, ld, nn, 1, /*guard=*/0);
    k_axpi<<<blocks, 256, 0, ctx->stream>>>(Mi, n, ld, 1.0, 1.0, Mi, ld);
    check_launch(ctx);
    // The block sweep applies explicit inverses of its 128-wide diagonal
    // blocks, which costs accuracy as kappa(M) grows (at kappa 1e6 the
    // iteration's J^-1/2 moved ~1e-10 from LAPACK's); one Newton-Schulz step
    // Mi <- 2 Mi - Mi M Mi brings the inverse back to ~kappa u.
    gemm(ctx, n, n, n, Mi, ld, 0, M, ld, 0, T, ld, 0, 1);   // T = Mi M
    gemm(ctx, n, n, n, Mi, ld, 0, T, ld, 0, X, ld, 0, 1);   // X = Mi (Mi M)^T = Mi M Mi
    k_ns_step<<<blocks, 256, 0, ctx->stream>>>(Mi, X, n, ld);
    check_launch(ctx);
    const double fmi = frob(ctx, Mi, n, ld, small, blocks);
    if (it == 0) fmi0 = fmi;
    const double mu = std::pow(fmi / frob(ctx, M, n, ld, small, blocks), 0.25);
    QX_REQUIRE(std::isfinite(mu) && mu > 0.0, QX_ERR_NUMERICAL, "Denman-Beavers iteration of the metric diverged");
    // X = (I + Mi / mu^2) / 2;  Y <- mu Y X,  Z <- mu Z X (X symmetric: its rows are its columns).
    k_axpi<<<blocks, 256, 0, ctx->stream>>>(Mi, n, ld, 0.5 / (mu * mu), 0.5, X, ld);
    check_launch(ctx);
    gemm(ctx, n, n, n, Y, ld, 0, X, ld, 0, T, ld, 0, 1);
    k_axpi<<<blocks, 256, 0, ctx->stream>>>(T, n, ld, mu, 0.0, Y, ld);
    check_launch(ctx);
    gemm(ctx, n, n, n, Z, ld, 0, X, ld, 0, T, ld, 0, 1);
    k_axpi<<<blocks, 256, 0, ctx->stream>>>(T, n, ld, mu, 0.0, Z, ld);
    check_launch(ctx);
    QX_CUDA(cudaMemsetAsync(res, 0, sizeof(unsigned long long), ctx->stream));
    k_db_m<<<blocks, 256, 0, ctx->stream>>>(M, Mi, n, ld, mu * mu, 1.0 / (mu * mu), res);
    check_launch(ctx);
    unsigned long long h = 0;
    QX_CUDA(cudaMemcpyAsync(&h, res, sizeof h, cudaMemcpyDeviceToHost, ctx->stream));
    sync_and_check(ctx);
    double r;
    memcpy(&r, &h, sizeof r);
    QX_REQUIRE(std::isfinite(r), QX_ERR_NUMERICAL, "Denman-Beavers iteration of the metric diverged");
    if (r < 1e-14) done = true;
  }
  // A metric this ill-conditioned has eigenvalues far below any useful
  // thresh_df: report it as such, with 1 / ||J^-1||_F (<= lambda_min).
  QX_REQUIRE(done, QX_ERR_NUMERICAL,
             "Denman-Beavers iteration of the metric did not converge: lambda_min(J) ~ %.3e (1 / ||J^-1||_F; "
             "thresh_df %.1e): remove the linear dependencies of the auxiliary basis first",
             fmi0 > 0.0 ? 1.0 / fmi0 : 0.0, thresh);
  // Symmetrised results (the products keep them symmetric only to rounding).
  k_symmetrize<<<blocks, 256, 0, ctx->stream>>>(Z, n, ld, T);
  check_launch(ctx);
  QX_CUDA(cudaMemcpyAsync(Jm, T, nn * sizeof(double), cudaMemcpyDeviceToDevice, ctx->stream));
  k_symmetrize<<<blocks, 256, 0, ctx->stream>>>(Y, n, ld, T);
  check_launch(ctx);
  QX_CUDA(cudaMemcpyAsync(Jp, T, nn * sizeof(double), cudaMemcpyDeviceToDevice, ctx->stream));
  // lambda_min(J) >= 1 / ||J^-1/2||_F^2 (= 1 / trace J^-1).
  const double fz = frob(ctx, Jm, n, ld, small, blocks);
  if (1.0 / (fz * fz) > thresh) return 1.0 / (fz * fz);
  // Otherwise 1 / lambda_max(J^-1/2)^2 by power iteration from a fixed start.
  double* x = small + 520;
  double* y = x + n + 8;
  std::vector<double> x0(n);
  for (int i = 0; i < n; ++i) x0[i] = 1.0 + 0.5 * std::sin(1.0 + 0.37 * i);
  QX_CUDA(cudaMemcpyAsync(x, x0.data(), n * sizeof(double), cudaMemcpyHostToDevice, ctx->stream));
  const int mv_blocks = std::min(ceil_div(n, 8), 4 * ctx->sm_count);
  for (int it = 0; it < 100; ++it) {
    k_matvec<<<mv_blocks, 256, 0, ctx->stream>>>(Jm, n, ld, x, y);
    check_launch(ctx);
    k_power_norm<<<1, 1024, 0, ctx->stream>>>(x, y, n, small + 516);
    check_launch(ctx);
  }
  double lam = 0.0;
  QX_CUDA(cudaMemcpyAsync(&lam, small + 516, sizeof lam, cudaMemcpyDeviceToHost, ctx->stream));
  QX_CUDA(cudaStreamSynchronize(ctx->stream));
  return 1.0 / (lam * lam);
}

size_t metric_work_doubles(int n, int ld) { return 4 * (size_t)n * ld + 520 + 2 * ((size_t)n + 8) + 64; }

// out[b] = s (in[b] + in[b]^T) / 2 + t I over n x n matrices (row stride ld,
// batch stride st; in and out distinct).  grid (x, batch).
__global__ void k_sym_batch(const double* __restrict__ in, int n, int ld, size_t st, double s, double t,
                            double* __restrict__ out) {
  const double* a = in + blockIdx.y * st;
  double* o = out + blockIdx.y * st;
  for (size_t e = (size_t)blockIdx.x * blockDim.x + threadIdx.x; e < (size_t)n * n;
       e += (size_t)gridDim.x * blockDim.x) {
    const size_t r = e / n, c = e % n;
    o[r * ld + c] = s * (0.5 * (a[r * ld + c] + a[c * ld + r])) + (r == c ? t : 0.0);
  }
}

// A[b] += t I in place.  grid (x, batch).
__global__ void k_add_diag_batch(double* __restrict__ A, int n, int ld, size_t st, double t) {
  double* a = A + blockIdx.y * st;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) a[(size_t)i * ld + i] += t;
}

// Any non-finite entry of the n x n matrices (row stride ld) sets *flag.
__global__ void k_nonfinite(const double* __restrict__ A, int n, int ld, size_t st, int* __restrict__ flag) {
  const double* a = A + blockIdx.y * st;
  for (size_t e = (size_t)blockIdx.x * blockDim.x + threadIdx.x; e < (size_t)n * n;
       e += (size_t)gridDim.x * blockDim.x)
    if (!isfinite(a[(e / n) * ld + e % n])) *flag = 1;
}
}  // namespace
}  // namespace qx

using namespace qx;

template <class F>
static qx_status run_df(qx_ctx* ctx, F&& f) {
  if (!ctx) return QX_ERR_INVALID_INPUT;
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

extern "C" {

qx_status qx_metric_inv_sqrt(qx_ctx* ctx, const double* metric, int naux, double thresh, double* inv_sqrt,
                             double* sqrt_metric) {
  return run_df(ctx, [&] {
    QX_REQUIRE(metric && inv_sqrt && naux > 0, QX_ERR_INVALID_INPUT, "invalid arguments to metric_inv_sqrt");
    const int ld = round_up(naux, 8);
    const size_t nn = (size_t)naux * ld;
    const double* d_j = (const double*)device_view(ctx, WS_LPQ, metric, (size_t)naux * naux * sizeof(double));
    DevBuf& wb = ctx->ws[WS_BSE2];
    wb.reserve((2 * nn + metric_work_doubles(naux, ld)) * sizeof(double));
    double* jm = wb.as<double>();
    double* jp = jm + nn;
    const double lmin = metric_inv_sqrt(ctx, d_j, naux, naux, jm, jp, ld, jp + nn, thresh);
    QX_REQUIRE(lmin > thresh, QX_ERR_NUMERICAL,
               "metric has an eigenvalue (%.3e) at or below thresh_df %.1e: remove the linear dependencies of the "
               "auxiliary basis first", lmin, thresh);
    QX_CUDA(cudaMemcpy2DAsync(inv_sqrt, naux * sizeof(double), jm, ld * sizeof(double), naux * sizeof(double), naux,
                              cudaMemcpyDefault, ctx->stream));
    if (sqrt_metric)
      QX_CUDA(cudaMemcpy2DAsync(sqrt_metric, naux * sizeof(double), jp, ld * sizeof(double), naux * sizeof(double),
                                naux, cudaMemcpyDefault, ctx->stream));
    sync_and_check(ctx);
  });
}

// The S3-3 screened interaction W(w) = v^1/2 (I - v^1/2 P0(w) v^1/2)^-1 v^1/2
// (quasix_core/src/dielectric/screening.rs:164-236 compute_screened_interaction,
// :334-410 compute_W_single_frequency, :580-639 compute_metric_sqrt).
// v^1/2 is the symmetric square root (the Denman-Beavers iterate, equal to
// the reference's eigendecomposition form when no eigenvalue of v lies at or
// below its clamp 1e-14; such metrics are rejected).  Per frequency, as the
// reference: eps = I - v^1/2 P0 v^1/2, symmetrised by averaging; eps^-1 by
// the guarded block sweep (pivoted fallback where the reference would fall
// from Cholesky to LU); W = v^1/2 eps^-1 v^1/2, symmetrised.  All products
// are FP64 DMMA GEMMs, batched over the frequencies of a chunk.
qx_status qx_compute_screened_interaction(qx_ctx* ctx, int nfreq, int naux, const double* p0, const double* v_aux,
                                          double* w) {
  return run_df(ctx, [&] {
    QX_REQUIRE(p0 && v_aux && w && nfreq > 0 && naux > 0, QX_ERR_INVALID_INPUT,
               "invalid arguments to compute_screened_interaction (nfreq=%d naux=%d)", nfreq, naux);
    const int ld = round_up(naux, 8);
    const size_t nn = (size_t)naux * ld, dense = (size_t)naux * naux;
    const double* d_v = (const double*)device_view(ctx, WS_LPQ, v_aux, dense * sizeof(double));
    DevBuf& mb = ctx->ws[WS_BSE2];
    mb.reserve((2 * nn + metric_work_doubles(naux, ld)) * sizeof(double));
    double* vm = mb.as<double>();
    double* vs = vm + nn;
    const double clamp = 1e-14;
    const double lmin = metric_inv_sqrt(ctx, d_v, naux, naux, vm, vs, ld, vs + nn, clamp);
    QX_REQUIRE(lmin > clamp, QX_ERR_NUMERICAL,
               "v_aux has an eigenvalue (%.3e) at or below %.0e: it is not positive definite", lmin, clamp);
    const double* d_p = (const double*)device_view(ctx, WS_BSE4, p0, (size_t)nfreq * dense * sizeof(double));
    // Three [fc][naux][ld] buffers per chunk of fc frequencies, at most ~3 GB.
    const size_t cap = std::max<size_t>(1, ((size_t)3 << 30) / (3 * nn * sizeof(double)));
    const int fc = (int)std::min<size_t>({(size_t)nfreq, cap, (size_t)65535});
    DevBuf& wb = ctx->ws[WS_BSE3];
    wb.reserve((3 * (size_t)fc * nn + 64) * sizeof(double));
    double* A = wb.as<double>();
    double* B = A + (size_t)fc * nn;
    double* E = B + (size_t)fc * nn;
    int* flag = reinterpret_cast<int*>(E + (size_t)fc * nn);
    QX_CUDA(cudaMemsetAsync(A, 0, (3 * (size_t)fc * nn + 64) * sizeof(double), ctx->stream));
    const int blocks = std::max(1, std::min<int>((int)((dense + 255) / 256), 2 * ctx->sm_count / std::max(1, fc) + 1));
    for (int f0 = 0; f0 < nfreq; f0 += fc) {
      const int nb = std::min(fc, nfreq - f0);
      // A = P0^T; B = v^1/2 P0; A = M = v^1/2 P0 v^1/2; E = eps = I - sym(M).
      transpose(ctx, d_p + (size_t)f0 * dense, naux, naux, naux, dense, A, ld, nn, nb);
      gemm(ctx, naux, naux, naux, vs, ld, 0, A, ld, nn, B, ld, nn, nb);
      gemm(ctx, naux, naux, naux, B, ld, nn, vs, ld, 0, A, ld, nn, nb);
      k_sym_batch<<<dim3(blocks, nb), 256, 0, ctx->stream>>>(A, naux, ld, nn, -1.0, 1.0, E);
      check_launch(ctx);
      // The sweep leaves eps^-1 - I in place.
      launch_invert_wc(ctx, E, naux, ld, nn, nb, /*guard=*/1);
      k_add_diag_batch<<<dim3(ceil_div(naux, 256), nb), 256, 0, ctx->stream>>>(E, naux, ld, nn, 1.0);
      check_launch(ctx);
      // B = v^1/2 eps^-T; A = v^1/2 eps^-T v^1/2; E = W = sym(A) (= sym(v^1/2 eps^-1 v^1/2)).
      gemm(ctx, naux, naux, naux, vs, ld, 0, E, ld, nn, B, ld, nn, nb);
      gemm(ctx, naux, naux, naux, B, ld, nn, vs, ld, 0, A, ld, nn, nb);
      k_sym_batch<<<dim3(blocks, nb), 256, 0, ctx->stream>>>(A, naux, ld, nn, 1.0, 0.0, E);
      check_launch(ctx);
      k_nonfinite<<<dim3(blocks, nb), 256, 0, ctx->stream>>>(E, naux, ld, nn, flag);
      check_launch(ctx);
      QX_CUDA(cudaMemcpy2DAsync(w + (size_t)f0 * dense, naux * sizeof(double), E, ld * sizeof(double),
                                naux * sizeof(double), (size_t)nb * naux, cudaMemcpyDefault, ctx->stream));
    }
    int hf = 0;
    QX_CUDA(cudaMemcpyAsync(&hf, flag, sizeof hf, cudaMemcpyDeviceToHost, ctx->stream));
    sync_and_check(ctx);
    QX_REQUIRE(hf == 0, QX_ERR_NUMERICAL, "W contains NaN or Inf values");
  });
}

qx_status qx_build_lpq(qx_ctx* ctx, const double* j3c_ao, const double* mo_coeff, const double* metric,
                       const double* metric_inv_sqrt_in, int nao, int nmo, int naux, double thresh, double* lpq,
                       double* chol_v) {
  return run_df(ctx, [&] {
    QX_REQUIRE(j3c_ao && mo_coeff && lpq && nao > 0 && nmo > 0 && naux > 0 && nmo <= nao, QX_ERR_INVALID_INPUT,
               "invalid arguments to build_lpq (nao=%d nmo=%d naux=%d)", nao, nmo, naux);
    QX_REQUIRE((metric != nullptr) != (metric_inv_sqrt_in != nullptr), QX_ERR_INVALID_INPUT,
               "build_lpq takes exactly one of metric and metric_inv_sqrt");
    QX_REQUIRE(!chol_v || metric, QX_ERR_INVALID_INPUT, "chol_v needs the metric");
    QX_REQUIRE(naux <= 65535, QX_ERR_INVALID_INPUT, "naux %d exceeds 65535", naux);
    const int ldx = round_up(nao, 8), ldj = round_up(naux, 8);
    const long long npq = (long long)nmo * nmo;
    const size_t nX = (size_t)naux * nao * ldx, nT = (size_t)naux * nmo * ldx, nL = (size_t)naux * npq;
    const size_t nLt = (size_t)npq * ldj, nC = (size_t)nmo * ldx, nJ = (size_t)naux * ldj;
    const double* d_j3 = (const double*)device_view(ctx, WS_LPQ, j3c_ao, (size_t)nao * nao * naux * sizeof(double));
    // Workspace: X (later reused for L'^T), T, L', C^T, J^-1/2, J^1/2, metric work.
    DevBuf& wb = ctx->ws[WS_BSE3];
    const size_t nXL = std::max(nX, nLt);
    const bool own_out = !is_device_ptr(lpq);
    wb.reserve((nXL + nT + nL + nC + 2 * nJ + (metric ? metric_work_doubles(naux, ldj) : 0)) * sizeof(double) +
               8 * 256);
    double* X = wb.as<double>();
    double* T = X + nXL;
    double* L = T + nT;
    double* Ct = L + nL;
    double* Jm = Ct + nC;
    double* Jp = Jm + nJ;
    double* mwork = Jp + nJ;
    // C [nao][nmo] -> C^T [nmo][ldx]: the A operand of the first GEMM and the
    // B operand ([q][v], v contiguous) of the second.
    const double* d_c = (const double*)device_view(ctx, WS_BSE6, mo_coeff, (size_t)nao * nmo * sizeof(double));
    QX_CUDA(cudaMemsetAsync(Ct, 0, nC * sizeof(double), ctx->stream));
    transpose_gs(ctx, d_c, nao, nmo, nmo, Ct, ldx);
    // Metric step operand.
    if (metric) {
      const double* d_m = (const double*)device_view(ctx, WS_BSE5, metric, (size_t)naux * naux * sizeof(double));
      const double lmin = metric_inv_sqrt(ctx, d_m, naux, naux, Jm, Jp, ldj, mwork, thresh);
      QX_REQUIRE(lmin > thresh, QX_ERR_NUMERICAL,
                 "metric has an eigenvalue (%.3e) at or below thresh_df %.1e: remove the linear dependencies of the "
                 "auxiliary basis first", lmin, thresh);
    } else {
      QX_CUDA(cudaMemcpy2DAsync(Jm, ldj * sizeof(double), metric_inv_sqrt_in, naux * sizeof(double),
                                naux * sizeof(double), naux, cudaMemcpyDefault, ctx->stream));
    }
    // (uv|P) -> X[P][u][v].
    QX_CUDA(cudaMemsetAsync(X, 0, nX * sizeof(double), ctx->stream));
    {
      const long long rb = ((long long)nao * nao + 31) / 32;
      dim3 grid(ceil_div(naux, 32), (unsigned)std::min<long long>(rb, 4096));
      k_aux_major<<<grid, dim3(32, 8), 0, ctx->stream>>>(d_j3, nao, naux, X, ldx);
      check_launch(ctx);
    }
    // T[P][p][v] = sum_u C^T[p][u] X[P][v][u];  L'[P][p][q] = sum_v T[P][p][v] C^T[q][v].
    gemm(ctx, nmo, nao, nao, Ct, ldx, 0, X, ldx, (size_t)nao * ldx, T, ldx, (size_t)nmo * ldx, naux);
    gemm(ctx, nmo, nmo, nao, T, ldx, (size_t)nmo * ldx, Ct, ldx, 0, L, nmo, (size_t)npq, naux);
    // lpq[P][pq] = sum_Q J^-1/2[P][Q] L'^T[pq][Q].
    double* Lt = X;
    transpose_gs(ctx, L, naux, (int)std::min<long long>(npq, INT32_MAX), (int)npq, Lt, ldj);
    double* out = lpq;
    if (own_out) {
      ctx->ws[WS_BSE4].reserve(nL * sizeof(double));
      out = ctx->ws[WS_BSE4].as<double>();
    }
    QX_REQUIRE(npq < INT32_MAX, QX_ERR_INVALID_INPUT, "nmo %d too large", nmo);
    gemm(ctx, naux, (int)npq, naux, Jm, ldj, 0, Lt, ldj, 0, out, (int)npq, 0, 1);
    if (own_out) QX_CUDA(cudaMemcpyAsync(lpq, out, nL * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
    if (chol_v)
      QX_CUDA(cudaMemcpy2DAsync(chol_v, naux * sizeof(double), Jp, ldj * sizeof(double), naux * sizeof(double), naux,
                                cudaMemcpyDefault, ctx->stream));
    sync_and_check(ctx);
  });
}

qx_status qx_transform_mo_3center(qx_ctx* ctx, const double* j3c_ao, const double* c_occ, const double* c_vir,
                                  int nao, int nocc, int nvir, int naux, double* out) {
  return run_df(ctx, [&] {
    QX_REQUIRE(j3c_ao && c_occ && c_vir && out && nao > 0 && nocc > 0 && nvir > 0 && naux > 0, QX_ERR_INVALID_INPUT,
               "invalid arguments to transform_mo_3center");
    QX_REQUIRE(naux <= 65535, QX_ERR_INVALID_INPUT, "naux %d exceeds 65535", naux);
    const int ldx = round_up(nao, 8), nov = nocc * nvir, ldj = round_up(naux, 8);
    const size_t nX = (size_t)naux * nao * ldx, nT = (size_t)naux * nocc * ldx, nL = (size_t)naux * nov;
    const double* d_j3 = (const double*)device_view(ctx, WS_LPQ, j3c_ao, (size_t)nao * nao * naux * sizeof(double));
    DevBuf& wb = ctx->ws[WS_BSE3];
    wb.reserve((nX + nT + nL + (size_t)nocc * ldx + (size_t)nvir * ldx + (size_t)nov * ldj) * sizeof(double) + 1024);
    double* X = wb.as<double>();
    double* T = X + nX;
    double* L = T + nT;
    double* Co = L + nL;
    double* Cv = Co + (size_t)nocc * ldx;
    double* Lt = Cv + (size_t)nvir * ldx;
    const double* d_co = (const double*)device_view(ctx, WS_BSE5, c_occ, (size_t)nao * nocc * sizeof(double));
    QX_CUDA(cudaMemsetAsync(Co, 0, ((size_t)nocc + nvir) * ldx * sizeof(double), ctx->stream));
    transpose_gs(ctx, d_co, nao, nocc, nocc, Co, ldx);
    const double* d_cv = (const double*)device_view(ctx, WS_BSE6, c_vir, (size_t)nao * nvir * sizeof(double));
    transpose_gs(ctx, d_cv, nao, nvir, nvir, Cv, ldx);
    QX_CUDA(cudaMemsetAsync(X, 0, nX * sizeof(double), ctx->stream));
    {
      const long long rb = ((long long)nao * nao + 31) / 32;
      dim3 grid(ceil_div(naux, 32), (unsigned)std::min<long long>(rb, 4096));
      k_aux_major<<<grid, dim3(32, 8), 0, ctx->stream>>>(d_j3, nao, naux, X, ldx);
      check_launch(ctx);
    }
    // T[P][i][v] = sum_u C_occ^T[i][u] X[P][v][u];  L[P][i][a] = sum_v T[P][i][v] C_vir^T[a][v].
    gemm(ctx, nocc, nao, nao, Co, ldx, 0, X, ldx, (size_t)nao * ldx, T, ldx, (size_t)nocc * ldx, naux);
    gemm(ctx, nocc, nvir, nao, T, ldx, (size_t)nocc * ldx, Cv, ldx, 0, L, nvir, (size_t)nov, naux);
    // [P][(i,a)] -> the reference's [(i,a)][P].
    transpose_gs(ctx, L, naux, nov, nov, Lt, ldj);
    QX_CUDA(cudaMemcpy2DAsync(out, naux * sizeof(double), Lt, ldj * sizeof(double), naux * sizeof(double), nov,
                              cudaMemcpyDefault, ctx->stream));
    sync_and_check(ctx);
  });
}

}  // extern "C"
