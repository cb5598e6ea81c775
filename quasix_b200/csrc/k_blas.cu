// Generic FP64 building blocks on the DMMA mainloop: a batched "NT" GEMM with
// split-K, small combination kernels and a one-CTA parallel Jacobi
// eigensolver for the Davidson Rayleigh-Ritz step.
#include <mutex>

#include "gemm_f64.cuh"
#include "qx_internal.cuh"
#include "qx_blas.cuh"

namespace qx {

using GemmTile = F64Tile<64, 64, 2, 2, 3>;

// C[b][m][n] (or the split-K partial) = sum_{k in split} A[b][m][k] B[b][n][k]
__global__ void __launch_bounds__(GemmTile::THREADS) k_gemm_nt(GemmNT g, double* __restrict__ part) {
  using T = GemmTile;
  extern __shared__ double smem[];
  const int nsplit = g.splitk;
  const int b = blockIdx.z / nsplit, sk = blockIdx.z % nsplit;
  const int m0 = blockIdx.y * T::BM, n0 = blockIdx.x * T::BN;
  const int kchunk = ((g.K + nsplit - 1) / nsplit + T::BK - 1) / T::BK * T::BK;
  const int kbeg = sk * kchunk;
  const int klen = max(0, min(g.K - kbeg, kchunk));
  double acc[T::MI][T::NJ][2];
#pragma unroll
  for (int i = 0; i < T::MI; ++i)
#pragma unroll
    for (int j = 0; j < T::NJ; ++j) acc[i][j][0] = acc[i][j][1] = 0.0;
  if (klen > 0)
    f64_mainloop<T>(acc, smem, g.A + (size_t)b * g.sA + (size_t)m0 * g.lda + kbeg, g.lda, g.M - m0,
                    g.B + (size_t)b * g.sB + (size_t)n0 * g.ldb + kbeg, g.ldb, g.N - n0, nullptr, klen);
#pragma unroll
  for (int i = 0; i < T::MI; ++i)
#pragma unroll
    for (int j = 0; j < T::NJ; ++j)
#pragma unroll
      for (int e = 0; e < 2; ++e) {
        const int m = m0 + f64_row<T>(i), n = n0 + f64_col<T>(j, e);
        if (m >= g.M || n >= g.N) continue;
        if (nsplit == 1) {
          double* c = g.C + (size_t)b * g.sC + (size_t)m * g.ldc + n;
          *c = g.alpha * acc[i][j][e] + (g.beta != 0.0 ? g.beta * *c : 0.0);
        } else {
          part[((size_t)sk * g.batch + b) * g.M * g.N + (size_t)m * g.N + n] = acc[i][j][e];
        }
      }
}

__global__ void k_splitk_reduce(GemmNT g, const double* __restrict__ part) {
  const size_t mn = (size_t)g.M * g.N;
  for (size_t idx = (size_t)blockIdx.x * blockDim.x + threadIdx.x; idx < mn * g.batch;
       idx += (size_t)gridDim.x * blockDim.x) {
    const int b = (int)(idx / mn);
    const size_t r = idx % mn;
    const int m = (int)(r / g.N), n = (int)(r % g.N);
    double s = 0.0;
    for (int k = 0; k < g.splitk; ++k) s += part[((size_t)k * g.batch + b) * mn + r];
    double* c = g.C + (size_t)b * g.sC + (size_t)m * g.ldc + n;
    *c = g.alpha * s + (g.beta != 0.0 ? g.beta * *c : 0.0);
  }
}

void gemm_nt_f64(qx_ctx* ctx, GemmNT g) {
  using T = GemmTile;
  QX_REQUIRE(g.lda % 2 == 0 && g.ldb % 2 == 0 && (reinterpret_cast<uintptr_t>(g.A) & 15) == 0 &&
                 (reinterpret_cast<uintptr_t>(g.B) & 15) == 0 && g.sA % 2 == 0 && g.sB % 2 == 0,
             QX_ERR_INVALID_INPUT, "gemm_nt_f64: operands must be 16-byte aligned with even leading dimensions");
  if (g.M <= 0 || g.N <= 0 || g.batch <= 0) return;
  static PerDeviceOnce attr_once;
  attr_once(ctx->device, [&] {
    QX_CUDA(cudaFuncSetAttribute(k_gemm_nt, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)T::SMEM));
  });
  if (g.splitk < 1) {
    // Enough CTAs to fill the GPU about twice.
    const long tiles = (long)ceil_div(g.M, T::BM) * ceil_div(g.N, T::BN) * g.batch;
    int s = 1;
    while (tiles * s < 2L * ctx->sm_count * 3 && g.K / (s * 2) >= 4 * T::BK && s < 64) s *= 2;
    g.splitk = s;
  }
  double* part = nullptr;
  if (g.splitk > 1) {
    DevBuf& pb = ctx->ws[WS_HOSTIN];
    pb.reserve((size_t)g.splitk * g.batch * g.M * g.N * sizeof(double));
    part = pb.as<double>();
  }
  dim3 grid(ceil_div(g.N, T::BN), ceil_div(g.M, T::BM), g.batch * g.splitk);
  k_gemm_nt<<<grid, T::THREADS, T::SMEM, ctx->stream>>>(g, part);
  check_launch(ctx);
  if (g.splitk > 1) {
    const size_t n = (size_t)g.M * g.N * g.batch;
    k_splitk_reduce<<<(unsigned)std::min<size_t>((n + 255) / 256, 8192), 256, 0, ctx->stream>>>(g, part);
    check_launch(ctx);
  }
}

// out[r][k] (+)= sum_i coef[i * ldc + r] V[i][k]  for r < nr, k < n.
__global__ void k_combine(const double* __restrict__ V, int ldv, int nv, const double* __restrict__ coef, int ldc,
                          int nr, int n, double* __restrict__ out, int ldo, double beta, double alpha) {
  constexpr int MAXR = 16;
  const int r0 = blockIdx.y * MAXR;
  const int nrb = min(MAXR, nr - r0);
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x) {
    double acc[MAXR];
#pragma unroll
    for (int r = 0; r < MAXR; ++r) acc[r] = 0.0;
    for (int i = 0; i < nv; ++i) {
      const double x = V[(size_t)i * ldv + k];
#pragma unroll
      for (int r = 0; r < MAXR; ++r)
        if (r < nrb) acc[r] += coef[(size_t)i * ldc + r0 + r] * x;
    }
#pragma unroll
    for (int r = 0; r < MAXR; ++r)
      if (r < nrb) {
        double* o = out + (size_t)(r0 + r) * ldo + k;
        *o = alpha * acc[r] + (beta != 0.0 ? beta * *o : 0.0);
      }
  }
}

void combine_rows(qx_ctx* ctx, const double* V, int ldv, int nv, const double* coef, int ldc, int nr, int n,
                  double* out, int ldo, double alpha, double beta) {
  if (nr <= 0 || n <= 0) return;
  dim3 grid(std::min(ceil_div(n, 256), 2 * ctx->sm_count), ceil_div(nr, 16));
  k_combine<<<grid, 256, 0, ctx->stream>>>(V, ldv, nv, coef, ldc, nr, n, out, ldo, beta, alpha);
  check_launch(ctx);
}

// ---------------------------------------------------------------------------
// Parallel cyclic Jacobi (round-robin pairing) for a symmetric n x n matrix,
// one CTA.  A is overwritten (diagonal -> eigenvalues), V receives the
// eigenvectors as columns.  Output sorted ascending into w and Z (columns).
// Converges when the off-diagonal Frobenius norm falls below tol * ||A||_F.
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(1024) k_jacobi(double* __restrict__ A, double* __restrict__ V, int n, int lda,
                                                 double* __restrict__ w, double* __restrict__ Z, int ldz,
                                                 int max_sweeps, int* __restrict__ info) {
  extern __shared__ double sh[];
  const int m = n + (n & 1);  // even number of players (a dummy when n is odd)
  double* cs = sh;            // [m/2] cosines
  double* sn = cs + m / 2;    // [m/2] sines
  int* pp = reinterpret_cast<int*>(sn + m / 2);  // [m/2]
  int* qq = pp + m / 2;                          // [m/2]
  __shared__ double red[32];
  __shared__ int done;
  const int tid = threadIdx.x, nt = blockDim.x;
  // Symmetrize and V = I.
  for (int idx = tid; idx < n * n; idx += nt) {
    const int i = idx / n, j = idx % n;
    if (i < j) {
      const double s = 0.5 * (A[(size_t)i * lda + j] + A[(size_t)j * lda + i]);
      A[(size_t)i * lda + j] = s;
      A[(size_t)j * lda + i] = s;
    }
    V[(size_t)i * lda + j] = (i == j) ? 1.0 : 0.0;
  }
  __syncthreads();
  int sweep = 0;
  for (; sweep < max_sweeps; ++sweep) {
    // Convergence test: off-diagonal norm vs total norm.
    double off = 0.0, tot = 0.0;
    for (int idx = tid; idx < n * n; idx += nt) {
      const int i = idx / n, j = idx % n;
      const double a = A[(size_t)i * lda + j];
      tot += a * a;
      if (i != j) off += a * a;
    }
    for (int o = 16; o > 0; o >>= 1) {
      off += __shfl_xor_sync(0xffffffffu, off, o);
      tot += __shfl_xor_sync(0xffffffffu, tot, o);
    }
    if ((tid & 31) == 0) red[tid >> 5] = off;
    __syncthreads();
    if (tid == 0) {
      double s = 0.0;
      for (int i = 0; i < (nt + 31) / 32; ++i) s += red[i];
      red[31] = s;
    }
    __syncthreads();
    const double offs = red[31];
    __syncthreads();
    if ((tid & 31) == 0) red[tid >> 5] = tot;
    __syncthreads();
    if (tid == 0) {
      double s = 0.0;
      for (int i = 0; i < (nt + 31) / 32; ++i) s += red[i];
      done = (offs <= 1e-30 * s) || (sqrt(offs) <= 1e-15 * sqrt(s));
    }
    __syncthreads();
    if (done) break;
    for (int round = 0; round < m - 1; ++round) {
      // Round-robin pairing: player 0 fixed, others rotate.
      for (int k = tid; k < m / 2; k += nt) {
        int a = (k == 0) ? 0 : 1 + (k - 1 + round) % (m - 1);
        int b = 1 + (m - 2 - k + round) % (m - 1);
        const int p = min(a, b), q = max(a, b);
        pp[k] = p;
        qq[k] = q;
        double c = 1.0, s = 0.0;
        if (q < n) {
          const double apq = A[(size_t)p * lda + q];
          if (fabs(apq) > 1e-300) {
            const double app = A[(size_t)p * lda + p], aqq = A[(size_t)q * lda + q];
            const double theta = (aqq - app) / (2.0 * apq);
            const double t = (theta >= 0.0 ? 1.0 : -1.0) / (fabs(theta) + sqrt(theta * theta + 1.0));
            c = 1.0 / sqrt(t * t + 1.0);
            s = t * c;
          }
        }
        cs[k] = c;
        sn[k] = s;
      }
      __syncthreads();
      // A <- A J (columns p, q of every row), V <- V J.
      for (int idx = tid; idx < (m / 2) * n; idx += nt) {
        const int k = idx / n, r = idx % n;
        const int p = pp[k], q = qq[k];
        if (q >= n) continue;
        const double c = cs[k], s = sn[k];
        const double ap = A[(size_t)r * lda + p], aq = A[(size_t)r * lda + q];
        A[(size_t)r * lda + p] = c * ap - s * aq;
        A[(size_t)r * lda + q] = s * ap + c * aq;
        const double vp = V[(size_t)r * lda + p], vq = V[(size_t)r * lda + q];
        V[(size_t)r * lda + p] = c * vp - s * vq;
        V[(size_t)r * lda + q] = s * vp + c * vq;
      }
      __syncthreads();
      // A <- J^T A (rows p, q).
      for (int idx = tid; idx < (m / 2) * n; idx += nt) {
        const int k = idx / n, col = idx % n;
        const int p = pp[k], q = qq[k];
        if (q >= n) continue;
        const double c = cs[k], s = sn[k];
        const double ap = A[(size_t)p * lda + col], aq = A[(size_t)q * lda + col];
        A[(size_t)p * lda + col] = c * ap - s * aq;
        A[(size_t)q * lda + col] = s * ap + c * aq;
      }
      __syncthreads();
    }
  }
  if (tid == 0) info[0] = sweep;
  __syncthreads();
  // Sort eigenvalues ascending (selection by rank; ties broken by index).
  for (int i = tid; i < n; i += nt) {
    const double di = A[(size_t)i * lda + i];
    int rank = 0;
    for (int j = 0; j < n; ++j) {
      const double dj = A[(size_t)j * lda + j];
      if (dj < di || (dj == di && j < i)) ++rank;
    }
    w[rank] = di;
    for (int r = 0; r < n; ++r) Z[(size_t)r * ldz + rank] = V[(size_t)r * lda + i];
  }
}

void jacobi_eigh(qx_ctx* ctx, double* A, double* V, int n, int lda, double* w, double* Z, int ldz, int* info) {
  const int m = n + (n & 1);
  const size_t sh = (size_t)m * sizeof(double) + (size_t)m * sizeof(int) + 64;
  static PerDeviceOnce attr_once;
  attr_once(ctx->device, [&] {
    QX_CUDA(cudaFuncSetAttribute(k_jacobi, cudaFuncAttributeMaxDynamicSharedMemorySize, 64 * 1024));
  });
  QX_REQUIRE(sh <= 64 * 1024, QX_ERR_INVALID_INPUT, "subspace too large for the Jacobi kernel (%d)", n);
  k_jacobi<<<1, 1024, sh, ctx->stream>>>(A, V, n, lda, w, Z, ldz, 60, info);
  check_launch(ctx);
}

// ---------------------------------------------------------------------------
// Lowest k eigenpairs of a symmetric n x n matrix, one CTA of 1024 threads:
// Householder tridiagonalisation (in place in W, through L2), Sturm-count
// bisection for eigenvalues 0..k-1 (one thread each), inverse iteration on
// the tridiagonal with partial pivoting (the dgttrf/dgttrs elimination),
// modified Gram-Schmidt among the k vectors, and back-transformation with
// the stored reflectors.  A is symmetrised on load ((A + A^T) / 2).
// Work (doubles): n*n + 4n + k*n*5 + k*n; ints: k*n.
// ---------------------------------------------------------------------------
__device__ __forceinline__ double cta_sum(double v, double* red) {
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  __syncthreads();
  if (lane == 0) red[warp] = v;
  __syncthreads();
  double t = 0.0;
  for (int i = 0; i < (int)(blockDim.x >> 5); ++i) t += red[i];
  return t;
}

// Sturm count of T - x I from the diagonal d and the squared off-diagonal e2
// (e2[i] = e[i]^2): the number of eigenvalues of T below x.
__device__ int sturm_count_sq(const double* d, const double* e2, int n, double x, double pivmin) {
  int c = 0;
  double q = d[0] - x;
  if (q < 0.0) ++c;
  for (int i = 1; i < n; ++i) {
    if (fabs(q) < pivmin) q = -pivmin;
    q = d[i] - x - e2[i - 1] / q;
    if (q < 0.0) ++c;
  }
  return c;
}

constexpr int kEighMaxMulti = 64;  // eigenvalues found by multisection (more: bisection per thread)

__global__ void __launch_bounds__(1024) k_eigh_lowest(const double* __restrict__ A, int n, int lda, int k,
                                                      double* __restrict__ W, double* __restrict__ work,
                                                      int* __restrict__ iwork, double* __restrict__ w_out,
                                                      double* __restrict__ Z, int ldz) {
  __shared__ double red[32];
  __shared__ int cnt[1024];
  __shared__ double br_lo[kEighMaxMulti], br_hi[kEighMaxMulti];
  __shared__ int br_done;
  extern __shared__ double sm[];  // u [n], q [n]; then d [n], e^2 [n]
  double* u = sm;
  double* q = sm + n;
  double* tau = work;           // [n]
  double* d = work + n;         // [n]
  double* e = work + 2 * n;     // [n]
  double* lam = work + 3 * n;   // [n]
  double* Y = work + 4 * n;     // [k][n] eigenvectors of T, then of A
  double* LU = Y + (size_t)k * n;  // [5][k][n] per-vector factors
  const int tid = threadIdx.x, nt = blockDim.x;
  const int lane = tid & 31, warp = tid >> 5, nwarp = nt >> 5;
  // Rows and columns by warps and lanes: no index division in the loops.
  for (int r = warp; r < n; r += nwarp)
    for (int c = lane; c < n; c += 32) W[(size_t)r * n + c] = 0.5 * (A[(size_t)r * lda + c] + A[(size_t)c * lda + r]);
  __syncthreads();
  // Tridiagonalisation: H_j = I - tau_j u_j u_j^T on rows/cols j+1..n-1.
  // W stays exactly symmetric (the rank-2 update gives (r, c) and (c, r)
  // the same value), so B u is taken along contiguous rows.
  for (int j = 0; j + 2 < n; ++j) {
    const int m = n - j - 1;
    double s = 0.0;
    for (int i = tid; i < m; i += nt) {
      const double x = W[(size_t)(j + 1 + i) * n + j];
      s += x * x;
    }
    const double alpha = sqrt(cta_sum(s, red));
    const double x0 = W[(size_t)(j + 1) * n + j];
    if (alpha == 0.0) {
      if (tid == 0) {
        tau[j] = 0.0;
        d[j] = W[(size_t)j * n + j];
        e[j] = 0.0;
      }
      __syncthreads();
      continue;
    }
    const double as = (x0 >= 0.0) ? -alpha : alpha;
    const double t = 1.0 / (alpha * (alpha + fabs(x0)));  // 2 / (u^T u)
    for (int i = tid; i < m; i += nt) u[i] = W[(size_t)(j + 1 + i) * n + j] - (i == 0 ? as : 0.0);
    __syncthreads();
    // p = B u: one warp per row of B, lanes along the row.
    for (int i = warp; i < m; i += nwarp) {
      const double* row = W + (size_t)(j + 1 + i) * n + j + 1;
      double acc = 0.0;
      for (int l = lane; l < m; l += 32) acc += row[l] * u[l];
      for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
      if (lane == 0) q[i] = acc;
    }
    __syncthreads();
    double up = 0.0;
    for (int i = tid; i < m; i += nt) up += u[i] * q[i];
    const double K = cta_sum(up, red);
    for (int i = tid; i < m; i += nt) q[i] = t * q[i] - 0.5 * t * t * K * u[i];
    __syncthreads();
    for (int r = warp; r < m; r += nwarp) {
      const double ur = u[r], qr = q[r];
      double* row = W + (size_t)(j + 1 + r) * n + j + 1;
      for (int c = lane; c < m; c += 32) row[c] -= ur * q[c] + qr * u[c];
    }
    // keep u in the column below the diagonal for the back-transformation
    for (int i = tid; i < m; i += nt) W[(size_t)(j + 1 + i) * n + j] = u[i];
    if (tid == 0) {
      tau[j] = t;
      d[j] = W[(size_t)j * n + j];
      e[j] = as;
    }
    __syncthreads();
  }
  if (tid == 0) {
    if (n >= 2) {
      d[n - 2] = W[(size_t)(n - 2) * n + n - 2];
      e[n - 2] = W[(size_t)(n - 1) * n + n - 2];
      tau[n - 2] = 0.0;
    }
    d[n - 1] = W[(size_t)(n - 1) * n + n - 1];
    tau[n - 1] = 0.0;
  }
  __syncthreads();
  // T in shared memory for the Sturm counts: d and e^2.
  double* ds = u;
  double* e2s = q;
  for (int i = tid; i < n; i += nt) {
    ds[i] = d[i];
    e2s[i] = (i + 1 < n) ? e[i] * e[i] : 0.0;
  }
  __syncthreads();
  double lo = 1e300, hi = -1e300, emax = 0.0;
  for (int i = 0; i < n; ++i) {
    const double r0 = (i > 0) ? fabs(e[i - 1]) : 0.0, r1 = (i + 1 < n) ? fabs(e[i]) : 0.0;
    lo = fmin(lo, d[i] - r0 - r1);
    hi = fmax(hi, d[i] + r0 + r1);
    if (i + 1 < n) emax = fmax(emax, fabs(e[i]));
  }
  const double tnorm = fmax(fabs(lo), fabs(hi));
  const double pivmin = fmax(1e-300, 1e-290 * fmax(1.0, emax * emax));
  const double a0 = lo - 1e-14 * tnorm - 1e-300, b0 = hi + 1e-14 * tnorm + 1e-300;
  auto converged = [](double a, double b) { return b - a <= 2.0 * 2.2e-16 * fmax(fabs(a), fabs(b)) + 1e-300; };
  if (k <= kEighMaxMulti && nt / k >= 2) {
    // Multisection for the eigenvalues r = 0..k-1 (ascending): each round
    // cuts every bracket [a_r, b_r] at P interior points, one Sturm count per
    // thread, and keeps the sub-interval holding eigenvalue r (count(a) <= r
    // < count(b)); a bracket shrinks (P + 1)-fold per round.
    const int P = nt / k;
    // Point j (1..P) of a bracket, computed the same way for the count and the update.
    auto point = [P](double a, double b, int j) { return a + (b - a) * ((double)j / (double)(P + 1)); };
    for (int r = tid; r < k; r += nt) {
      br_lo[r] = a0;
      br_hi[r] = b0;
    }
    __syncthreads();
    for (int round = 0; round < 64; ++round) {
      const int r = tid / P, pp = tid - r * P;
      if (r < k) {
        const double a = br_lo[r], b = br_hi[r];
        cnt[tid] = converged(a, b) ? -1 : sturm_count_sq(ds, e2s, n, point(a, b, pp + 1), pivmin);
      }
      __syncthreads();
      if (tid == 0) br_done = 1;
      __syncthreads();
      if (tid < k) {
        const double a = br_lo[tid], b = br_hi[tid];
        if (!converged(a, b)) {
          // First point whose count exceeds r: the eigenvalue lies between it
          // and the point before.
          int pf = P;
          for (int p2 = 0; p2 < P; ++p2)
            if (cnt[tid * P + p2] > tid) {
              pf = p2;
              break;
            }
          const double na = (pf == 0) ? a : point(a, b, pf);
          const double nb = (pf == P) ? b : point(a, b, pf + 1);
          br_lo[tid] = na;
          br_hi[tid] = nb;
          if (!converged(na, nb)) br_done = 0;
        }
      }
      __syncthreads();
      if (br_done) break;
    }
    for (int r = tid; r < k; r += nt) lam[r] = 0.5 * (br_lo[r] + br_hi[r]);
  } else {
    // Bisection, one thread per eigenvalue.
    for (int r = tid; r < k; r += nt) {
      double a = a0, b = b0;
      for (int it = 0; it < 200; ++it) {
        const double mid = 0.5 * (a + b);
        if (converged(a, b)) break;
        if (sturm_count_sq(ds, e2s, n, mid, pivmin) > r)
          b = mid;
        else
          a = mid;
      }
      lam[r] = 0.5 * (a + b);
    }
  }
  __syncthreads();
  // Inverse iteration on T - lam I (partial pivoting), three solves.
  for (int r = tid; r < k; r += nt) {
    double* dl = LU + ((size_t)0 * k + r) * n;
    double* dd = LU + ((size_t)1 * k + r) * n;
    double* du = LU + ((size_t)2 * k + r) * n;
    double* du2 = LU + ((size_t)3 * k + r) * n;
    int* piv = iwork + (size_t)r * n;
    double* y = Y + (size_t)r * n;
    const double lr = lam[r];
    for (int i = 0; i < n; ++i) {
      dd[i] = d[i] - lr;
      if (i + 1 < n) {
        dl[i] = e[i];
        du[i] = e[i];
      }
      du2[i] = 0.0;
    }
    for (int i = 0; i + 1 < n; ++i) {
      if (fabs(dd[i]) >= fabs(dl[i])) {
        piv[i] = i;
        if (dd[i] != 0.0) {
          const double f = dl[i] / dd[i];
          dl[i] = f;
          dd[i + 1] -= f * du[i];
        }
      } else {
        piv[i] = i + 1;
        const double f = dd[i] / dl[i];
        dd[i] = dl[i];
        dl[i] = f;
        const double tmp = du[i];
        du[i] = dd[i + 1];
        dd[i + 1] = tmp - f * dd[i + 1];
        if (i + 2 < n) {
          du2[i] = du[i + 1];
          du[i + 1] = -f * du[i + 1];
        }
      }
    }
    const double tiny = 2.2e-16 * fmax(tnorm, 1e-300);
    for (int i = 0; i < n; ++i)
      if (fabs(dd[i]) < tiny) dd[i] = (dd[i] < 0.0) ? -tiny : tiny;
    for (int i = 0; i < n; ++i) y[i] = 1.0 + 0.01 * sin(0.7 * (i + 1) * (r + 1));
    for (int sweep = 0; sweep < 3; ++sweep) {
      for (int i = 0; i + 1 < n; ++i) {
        if (piv[i] == i) {
          y[i + 1] -= dl[i] * y[i];
        } else {
          const double tmp = y[i];
          y[i] = y[i + 1];
          y[i + 1] = tmp - dl[i] * y[i];
        }
      }
      y[n - 1] /= dd[n - 1];
      if (n >= 2) y[n - 2] = (y[n - 2] - du[n - 2] * y[n - 1]) / dd[n - 2];
      for (int i = n - 3; i >= 0; --i) y[i] = (y[i] - du[i] * y[i + 1] - du2[i] * y[i + 2]) / dd[i];
      double nrm = 0.0;
      for (int i = 0; i < n; ++i) nrm += y[i] * y[i];
      nrm = 1.0 / sqrt(nrm);
      for (int i = 0; i < n; ++i) y[i] *= nrm;
    }
  }
  __syncthreads();
  // Modified Gram-Schmidt among the k vectors (in order of eigenvalue).
  for (int r = 0; r < k; ++r) {
    double* yr = Y + (size_t)r * n;
    for (int s2 = 0; s2 < r; ++s2) {
      const double* ys = Y + (size_t)s2 * n;
      double dp = 0.0;
      for (int i = tid; i < n; i += nt) dp += yr[i] * ys[i];
      const double dot = cta_sum(dp, red);
      for (int i = tid; i < n; i += nt) yr[i] -= dot * ys[i];
      __syncthreads();
    }
    double nn = 0.0;
    for (int i = tid; i < n; i += nt) nn += yr[i] * yr[i];
    const double inv = 1.0 / sqrt(cta_sum(nn, red));
    for (int i = tid; i < n; i += nt) yr[i] *= inv;
    __syncthreads();
  }
  // z = H_0 H_1 ... H_{n-3} y: one warp per vector.
  for (int r = warp; r < k; r += nwarp) {
    double* y = Y + (size_t)r * n;
    for (int j = n - 3; j >= 0; --j) {
      const double tj = tau[j];
      if (tj == 0.0) continue;
      const int m = n - j - 1;
      double dp = 0.0;
      for (int i = lane; i < m; i += 32) dp += W[(size_t)(j + 1 + i) * n + j] * y[j + 1 + i];
      for (int o = 16; o > 0; o >>= 1) dp += __shfl_xor_sync(0xffffffffu, dp, o);
      for (int i = lane; i < m; i += 32) y[j + 1 + i] -= tj * dp * W[(size_t)(j + 1 + i) * n + j];
      __syncwarp();
    }
  }
  __syncthreads();
  for (int r = tid; r < k; r += nt) w_out[r] = lam[r];
  for (int idx = tid; idx < n * k; idx += nt) {
    const int i = idx / k, r = idx % k;
    Z[(size_t)i * ldz + r] = Y[(size_t)r * n + i];
  }
}

size_t eigh_lowest_work_doubles(int n, int k) { return (size_t)n * n + 4 * (size_t)n + 6 * (size_t)k * n + 64; }

void eigh_lowest(qx_ctx* ctx, const double* A, int n, int lda, int k, double* w, double* Z, int ldz, double* work,
                 int* iwork) {
  QX_REQUIRE(n >= 1 && k >= 1 && k <= n && n <= 4096, QX_ERR_INVALID_INPUT, "eigh_lowest: n=%d k=%d", n, k);
  double* W = work;
  double* rest = work + (size_t)n * n;
  const size_t sh = 2 * (size_t)n * sizeof(double);
  static PerDeviceOnce attr_once;
  attr_once(ctx->device, [&] {
    QX_CUDA(cudaFuncSetAttribute(k_eigh_lowest, cudaFuncAttributeMaxDynamicSharedMemorySize, 2 * 4096 * 8));
  });
  k_eigh_lowest<<<1, 1024, sh, ctx->stream>>>(A, n, lda, k, W, rest, iwork, w, Z, ldz);
  check_launch(ctx);
}

}  // namespace qx
