// FP64 kernels of the GW chain: chi weights, eps = I + B chi B^T, block-sweep
// inversion to Wc = eps^-1 - I, pair gathers, exchange diagonal, the Sigma_c
// pair contraction v = B_p^T Wc B_p, and the Sigma_c(iw) assembly.
#include <algorithm>
#include <mutex>
#include <vector>

#include "gemm_f64.cuh"
#include "qx_blas.cuh"
#include "qx_internal.cuh"

namespace qx {

// ---------------------------------------------------------------------------
// chi'[w][k] = -4 e_k / (f_w^2 + e_k^2)  (imaginary axis, e_k = e_i - e_a < 0)
// chi'[w][k] = -4 e_k / (e_k^2 - f_w^2)  (real axis)
// so that eps = I - Pi = I + B diag(chi') B^T  (correlation_ac.rs:184-211).
// ---------------------------------------------------------------------------
__global__ void k_chi(const double* __restrict__ en, int nocc, int nvir, const double* __restrict__ freqs,
                      int real_axis, double* __restrict__ chi, int ldov) {
  const int w = blockIdx.y;
  const int nov = nocc * nvir;
  const double f = freqs[w];
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < ldov; k += gridDim.x * blockDim.x) {
    double v = 0.0;
    if (k < nov) {
      const int i = k / nvir, a = k % nvir;
      const double e = en[i] - en[nocc + a];
      v = real_axis ? (-4.0 * e / (e * e - f * f)) : (-4.0 * e / (f * f + e * e));
    }
    chi[(size_t)w * ldov + k] = v;
  }
}

void launch_chi(qx_ctx* ctx, const double* energies, int nocc, int nvir, const double* freqs, int nw,
                int real_axis, double* chi, int ldov) {
  dim3 grid(ceil_div(ldov, 256), nw);
  k_chi<<<grid, 256, 0, ctx->stream>>>(energies, nocc, nvir, freqs, real_axis, chi, ldov);
  check_launch(ctx);
}

// ---------------------------------------------------------------------------
// eps[w] = I + B_ov diag(chi'[w]) B_ov^T on lower-triangular tile pairs,
// mirrored on store.
// ---------------------------------------------------------------------------
using EpsTile = F64Tile<64, 64, 2, 2, 3>;

__global__ void __launch_bounds__(EpsTile::THREADS) k_eps_f64(const double* __restrict__ bov, int ldov, int naux,
                                                              int nov, const double* __restrict__ chi,
                                                              double* __restrict__ eps, int ldn,
                                                              size_t eps_stride) {
  using T = EpsTile;
  extern __shared__ double smem[];
  // Lower-triangular tile index -> (tm, tn), tm >= tn.
  const int t = blockIdx.x;
  int tm = (int)floor((sqrt(8.0 * t + 1.0) - 1.0) * 0.5);
  while ((tm + 1) * (tm + 2) / 2 <= t) ++tm;
  while (tm * (tm + 1) / 2 > t) --tm;
  const int tn = t - tm * (tm + 1) / 2;
  const int w = blockIdx.y;
  const int m0 = tm * T::BM, n0 = tn * T::BN;
  double acc[T::MI][T::NJ][2];
#pragma unroll
  for (int i = 0; i < T::MI; ++i)
#pragma unroll
    for (int j = 0; j < T::NJ; ++j) acc[i][j][0] = acc[i][j][1] = 0.0;
  f64_mainloop<T>(acc, smem, bov + (size_t)m0 * ldov, ldov, naux - m0, bov + (size_t)n0 * ldov, ldov, naux - n0,
                  chi + (size_t)w * ldov, nov);
  double* E = eps + (size_t)w * eps_stride;
#pragma unroll
  for (int i = 0; i < T::MI; ++i)
#pragma unroll
    for (int j = 0; j < T::NJ; ++j)
#pragma unroll
      for (int e = 0; e < 2; ++e) {
        const int m = m0 + f64_row<T>(i), n = n0 + f64_col<T>(j, e);
        if (m < naux && n < naux) {
          const double v = acc[i][j][e] + (m == n ? 1.0 : 0.0);
          E[(size_t)m * ldn + n] = v;
          if (tm != tn) E[(size_t)n * ldn + m] = v;
        }
      }
}

void launch_eps_fp64(qx_ctx* ctx, const double* bov, int ldov, int naux, int nov, const double* chi, int nw,
                     double* eps, int ldn, size_t eps_stride) {
  using T = EpsTile;
  const int tiles = ceil_div(naux, T::BM);
  dim3 grid(tiles * (tiles + 1) / 2, nw);
  static PerDeviceOnce attr_once;
  attr_once(ctx->device, [&] {
    QX_CUDA(cudaFuncSetAttribute(k_eps_f64, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)T::SMEM));
  });
  k_eps_f64<<<grid, T::THREADS, T::SMEM, ctx->stream>>>(bov, ldov, naux, nov, chi, eps, ldn, eps_stride);
  check_launch(ctx);
}

// ---------------------------------------------------------------------------
// Block sweep inversion.  For a symmetric M and index block K, the sweep
//   D = M_KK^-1;  M_RR -= M_RK D M_KR;  M_RK = M_RK D;  M_KR = D M_KR;  M_KK = -D
// applied to every block in turn leaves -M^-1 (Gauss-Jordan without
// pivoting; stable for SPD, and it still inverts an indefinite eps as long as
// no pivot vanishes).  Per block of SWEEP_NB columns:
//   k_sweep_diag   : D = inverse of the current diagonal block (one CTA per matrix)
//   k_sweep_tpanel : T = M[:, K] D                      (DMMA GEMM, K = nb)
//   k_sweep_write  : P[r] = M[r][K] (old panel), then M[r][K] = M[K][r] = T[r],
//                    M[K][K] = -D
//   k_sweep_update : M[r][c] -= T[r] . P[c]  for r, c outside K, lower tiles
//                    only, mirrored (DMMA GEMM, K = nb)
// Because the update reads the saved panel P, the next block's diagonal and
// panel can be swept while the rest of this block's update still runs: the
// update is split into the tiles that touch the next block (on the critical
// chain) and the others (on a low-priority stream), with T, P, D
// double-buffered.
// ---------------------------------------------------------------------------
constexpr int SWEEP_NB = 128;

// The kb x kb diagonal block, padded with the identity to 128 x 128, is swept
// in four sub-blocks of 32 (the block sweep applied recursively): warp 0 sweeps
// the 32 x 32 sub-block element by element in registers (lane j holds column
// j; pivot rows and columns travel by shuffles, so a pivot step costs no block
// barrier), then the whole CTA applies the rank-32 update to the rest of the
// 128 x 128 block through shared memory.
// A pivot at or below tol (0 unguarded: an exact zero), or a non-finite one,
// sets bad_any.  GUARD: gm also takes max |entry| of the columns not yet
// swept after each pivot step (the element growth of the elimination).
template <bool GUARD>
__device__ __forceinline__ void sweep32_warp(double* S, int q0, int lane, bool& bad_any, double tol, double& gm) {
  // Four pivot steps per loop iteration: at the start of group p4, c[k]
  // holds S[(p4 + k) % 32][lane], so step s's pivot row is c[s] and every
  // register index is a compile-time constant; the array then rotates by four
  // (an unrolled loop of 32 steps measured slower, it misses the instruction
  // cache; one step per iteration spent 64 register moves per pivot on the
  // rotation).  The lanes other than p take c[k] - S[r][p] S[p][lane] / d and
  // lane p takes S[r][p] / d, both as one FMA: fma(ck, b, c[k] * a) with
  // (a, b) = (1, -rj) or (0, inv).
  double c[32];
#pragma unroll
  for (int i = 0; i < 32; ++i) c[i] = S[(q0 + i) * SWEEP_NB + q0 + lane];
  constexpr int UNR = 4;
#pragma unroll 1
  for (int p4 = 0; p4 < 32; p4 += UNR) {
#pragma unroll
    for (int s = 0; s < UNR; ++s) {
      const int p = p4 + s;
      const double d = __shfl_sync(0xffffffffu, c[s], p);
      const bool bad = !(fabs(d) > tol) || !isfinite(d);
      bad_any |= bad;
      const double inv = bad ? 0.0 : 1.0 / d;
      const double rj = c[s] * inv;  // S[p][lane] / d
      const bool piv = (lane == p);
      const double a = piv ? 0.0 : 1.0, b = piv ? inv : -rj;
#pragma unroll
      for (int k = 0; k < 32; ++k) {
        if (k == s) continue;
        const double ck = __shfl_sync(0xffffffffu, c[k], p);  // S[row k][p]
        c[k] = fma(ck, b, c[k] * a);
      }
      c[s] = piv ? -inv : rj;
      // Growth of the columns not yet swept, sampled every eighth pivot (the
      // serial pivot chain is this kernel's bound; the probe backward error of
      // the guard catches any loss between samples).
      if (GUARD && (p & 7) == 7 && lane > p) {
#pragma unroll
        for (int i = 0; i < 32; ++i) gm = fmax(gm, isfinite(c[i]) ? fabs(c[i]) : INFINITY);
      }
    }
    double t[UNR];
#pragma unroll
    for (int i = 0; i < UNR; ++i) t[i] = c[i];
#pragma unroll
    for (int i = 0; i + UNR < 32; ++i) c[i] = c[i + UNR];
#pragma unroll
    for (int i = 0; i < UNR; ++i) c[32 - UNR + i] = t[i];
  }
#pragma unroll
  for (int i = 0; i < 32; ++i) S[(q0 + i) * SWEEP_NB + q0 + lane] = c[i];
}

// D = -(A_KK)^-1 for the kb x kb diagonal block whose first element is at
// Akk (row stride ldn), zero outside kb x kb; *status_w = 1 when a pivot is at
// or below tol (guarded sweep) or vanishes.  growth_w (guarded sweep, else
// null): max |A_KK| of the not-yet-swept block joins it.  512 threads;
// dynamic shared memory (128 * 128 + 128 * 33) doubles.
__device__ __forceinline__ void block_amax(double m, double* red, unsigned long long* out);
template <bool GUARD>
__device__ __forceinline__ void sweep_diag_body(const double* __restrict__ Akk, int ldn, int kb,
                                                double* __restrict__ D, int* __restrict__ status_w, double tol,
                                                unsigned long long* growth_w) {
  static_assert(SWEEP_NB == 128, "thread mapping assumes 128 columns");
  constexpr int TLD = 33;                       // padded row stride of T
  extern __shared__ double S[];                 // [128][128]
  double* Tb = S + SWEEP_NB * SWEEP_NB;         // [128][33]
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int j = tid & 127, r0 = tid >> 7;
  double gm = 0.0;  // GUARD: max |entry| met in the unswept part
  for (int k = 0; k < 32; ++k) {
    const int i = r0 + 4 * k;
    const double v = (i < kb && j < kb) ? Akk[(size_t)i * ldn + j] : (i == j ? 1.0 : 0.0);
    S[i * SWEEP_NB + j] = v;
    if (GUARD) gm = fmax(gm, isfinite(v) ? fabs(v) : INFINITY);
  }
  bool bad_any = false;
  // Sub-blocks past kb are identity padding with no coupling to the block:
  // sweeping them changes nothing inside it (D is zeroed outside kb), so a
  // narrow last block sweeps only ceil(kb / 32) of them.
  const int nsb = (kb + 31) / 32;
  for (int sb = 0; sb < nsb; ++sb) {
    const int q0 = 32 * sb;
    __syncthreads();
    if (warp == 0) sweep32_warp<GUARD>(S, q0, lane, bad_any, tol, gm);
    __syncthreads();
    // Both products below use register tiles (thread = 4 rows x 2 or 8
    // columns), so each shared-memory operand feeds several FMAs.
    const int rt = tid >> 4, ct = tid & 15, rb = 4 * rt;
    // T[r][q] = S[r][Q] D1 = -S[r][Q] Sswept[Q][q] for rows outside Q (0 inside).
    {
      const int cb = 2 * ct;
      double t[4][2];
#pragma unroll
      for (int i = 0; i < 4; ++i) t[i][0] = t[i][1] = 0.0;
#pragma unroll 4
      for (int p = 0; p < 32; ++p) {
        const double b0 = S[(q0 + p) * SWEEP_NB + q0 + cb], b1 = S[(q0 + p) * SWEEP_NB + q0 + cb + 1];
#pragma unroll
        for (int i = 0; i < 4; ++i) {
          const double a = S[(rb + i) * SWEEP_NB + q0 + p];
          t[i][0] -= a * b0;
          t[i][1] -= a * b1;
        }
      }
#pragma unroll
      for (int i = 0; i < 4; ++i) {
        const bool inq = (rb + i >= q0 && rb + i < q0 + 32);
        Tb[(rb + i) * TLD + cb] = inq ? 0.0 : t[i][0];
        Tb[(rb + i) * TLD + cb + 1] = inq ? 0.0 : t[i][1];
      }
    }
    __syncthreads();
    // S[r][c] -= T[r] . S[Q][c]  for r, c outside Q (old S[Q][c]; rows in Q
    // are read, never written here).
    {
      // Columns 32 v + 2 ct + {0, 1}, v = 0..3: a warp's double2 loads are
      // contiguous (conflict-free), and each 32-column group lies wholly
      // inside or outside Q.
      const int cb = 2 * ct;
      double acc[4][8];
#pragma unroll
      for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int c = 0; c < 8; ++c) acc[i][c] = 0.0;
#pragma unroll 2
      for (int p = 0; p < 32; ++p) {
        double bv[8];
        const double* brow = S + (q0 + p) * SWEEP_NB + cb;
#pragma unroll
        for (int v = 0; v < 4; ++v) {
          const double2 x2 = *reinterpret_cast<const double2*>(brow + 32 * v);
          bv[2 * v] = x2.x;
          bv[2 * v + 1] = x2.y;
        }
#pragma unroll
        for (int i = 0; i < 4; ++i) {
          const double a = Tb[(rb + i) * TLD + p];
#pragma unroll
          for (int c = 0; c < 8; ++c) acc[i][c] += a * bv[c];
        }
      }
#pragma unroll
      for (int i = 0; i < 4; ++i) {
        if (rb + i >= q0 && rb + i < q0 + 32) continue;
#pragma unroll
        for (int v = 0; v < 4; ++v) {
          if (32 * v == q0) continue;
          const double s0 = S[(rb + i) * SWEEP_NB + 32 * v + cb] - acc[i][2 * v];
          const double s1 = S[(rb + i) * SWEEP_NB + 32 * v + cb + 1] - acc[i][2 * v + 1];
          S[(rb + i) * SWEEP_NB + 32 * v + cb] = s0;
          S[(rb + i) * SWEEP_NB + 32 * v + cb + 1] = s1;
          // Rows and columns past this sub-block: the Schur complement.
          if (GUARD && rb + i >= q0 + 32 && 32 * v > q0) {
            gm = fmax(gm, isfinite(s0) ? fabs(s0) : INFINITY);
            gm = fmax(gm, isfinite(s1) ? fabs(s1) : INFINITY);
          }
        }
      }
    }
    __syncthreads();
    // S[r][Q] = T[r] (lanes along q) and S[Q][r] = T[r]^T (lanes along r).
    for (int idx = tid; idx < SWEEP_NB * 32; idx += blockDim.x) {
      const int r = idx >> 5, q = idx & 31;
      if (!(r >= q0 && r < q0 + 32)) S[r * SWEEP_NB + q0 + q] = Tb[r * TLD + q];
    }
    for (int idx = tid; idx < SWEEP_NB * 32; idx += blockDim.x) {
      const int q = idx >> 7, r = idx & 127;
      if (!(r >= q0 && r < q0 + 32)) S[(q0 + q) * SWEEP_NB + r] = Tb[r * TLD + q];
    }
  }
  __syncthreads();
  if (lane == 0 && warp == 0 && bad_any) atomicExch(status_w, 1);
  if (GUARD && growth_w) {
    __shared__ double gred[16];
    block_amax(gm, gred, growth_w);
  }
  // D = -S, zero outside the kb x kb block.
  for (int k = 0; k < 32; ++k) {
    const int i = r0 + 4 * k;
    D[(size_t)i * SWEEP_NB + j] = (i < kb && j < kb) ? -S[i * SWEEP_NB + j] : 0.0;
  }
}

// Pivot tolerance of matrix w: kGuardPivot * max|eps_w| in a guarded sweep
// (gamax: the words of the guard's copy kernel), an exact zero otherwise.
__device__ __forceinline__ double guard_tol(const unsigned long long* gamax, int w) {
  return gamax ? kGuardPivot * __longlong_as_double((long long)gamax[w]) : 0.0;
}

template <bool GUARD>
__global__ void __launch_bounds__(512) k_sweep_diag(const double* __restrict__ M, int ldn, size_t stride, int k0,
                                                    int kb, double* __restrict__ Dp, int* __restrict__ status,
                                                    const unsigned long long* __restrict__ gamax,
                                                    unsigned long long* __restrict__ growth) {
  const int w = blockIdx.x;
  sweep_diag_body<GUARD>(M + (size_t)w * stride + (size_t)k0 * ldn + k0, ldn, kb,
                         Dp + (size_t)w * SWEEP_NB * SWEEP_NB, status + w, guard_tol(gamax, w),
                         growth ? growth + w : nullptr);
}

using PanelTile = F64Tile<64, 64, 2, 2, 3>;

// *out = max(*out, max over the block of m) (m >= 0 compares as its bit
// pattern); every thread of the block calls it; red holds one double per warp.
__device__ __forceinline__ void block_amax(double m, double* red, unsigned long long* out) {
  for (int o = 16; o > 0; o >>= 1) m = fmax(m, __shfl_xor_sync(0xffffffffu, m, o));
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = m;
  __syncthreads();
  if (threadIdx.x < 32) {
    m = threadIdx.x < (blockDim.x >> 5) ? red[threadIdx.x] : 0.0;
    for (int o = 16; o > 0; o >>= 1) m = fmax(m, __shfl_xor_sync(0xffffffffu, m, o));
    if (threadIdx.x == 0) atomicMax(out, __double_as_longlong(m));
  }
}

// Tile (m0, n0) of T[r][:] = M[r][K] D (D symmetric: its rows serve as the B
// operand); columns past kb come out zero.  amax (optional): max|T| of the
// tile joins *amax (the bound of a later split of T).
__device__ __forceinline__ void sweep_tpanel_body(const double* __restrict__ M, int n, int ldn, int k0, int kb,
                                                  const double* __restrict__ Dw, double* __restrict__ Tw, int m0,
                                                  int n0, unsigned long long* amax) {
  using T = PanelTile;
  extern __shared__ double smem[];
  double acc[T::MI][T::NJ][2];
#pragma unroll
  for (int i = 0; i < T::MI; ++i)
#pragma unroll
    for (int j = 0; j < T::NJ; ++j) acc[i][j][0] = acc[i][j][1] = 0.0;
  const double* A = M + (size_t)m0 * ldn + k0;
  const double* D = Dw + (size_t)n0 * SWEEP_NB;
  f64_mainloop<T>(acc, smem, A, ldn, n - m0, D, SWEEP_NB, kb - n0, nullptr, kb);
#pragma unroll
  for (int i = 0; i < T::MI; ++i)
#pragma unroll
    for (int j = 0; j < T::NJ; ++j)
#pragma unroll
      for (int e = 0; e < 2; ++e) {
        const int r = m0 + f64_row<T>(i), c = n0 + f64_col<T>(j, e);
        if (r < n && c < SWEEP_NB) Tw[(size_t)r * SWEEP_NB + c] = acc[i][j][e];
      }
  if (amax) {
    // The mainloop has drained its stages: smem is free for the reduction.
    double mx = 0.0;
#pragma unroll
    for (int i = 0; i < T::MI; ++i)
#pragma unroll
      for (int j = 0; j < T::NJ; ++j)
#pragma unroll
        for (int e = 0; e < 2; ++e)
          if (m0 + f64_row<T>(i) < n) mx = fmax(mx, fabs(acc[i][j][e]));
    block_amax(mx, smem, amax);
  }
}

// T[w][r][:] = M[w][r][K] D[w]
__global__ void __launch_bounds__(PanelTile::THREADS) k_sweep_tpanel(const double* __restrict__ M, int n, int ldn,
                                                                     size_t stride, int k0, int kb,
                                                                     const double* __restrict__ Dp,
                                                                     double* __restrict__ Tp, size_t pstride,
                                                                     unsigned long long* amax) {
  const int w = blockIdx.z;
  sweep_tpanel_body(M + (size_t)w * stride, n, ldn, k0, kb, Dp + (size_t)w * SWEEP_NB * SWEEP_NB,
                    Tp + (size_t)w * pstride, blockIdx.x * PanelTile::BM, blockIdx.y * PanelTile::BN,
                    amax ? amax + w : nullptr);
}

using SweepTile = F64Tile<64, 64, 2, 2, 3>;

// M[r][c] -= T[r] . P[c] over the 64 x 64 tile (tm, tn), lower part, mirrored;
// rows and columns of the K block are left alone.  mode 0: any tile; 1: only
// tiles whose rows or columns meet the next block [nk0, nk0 + nkb); 2: only
// the other tiles.
__device__ __forceinline__ void sweep_update_body(double* __restrict__ A, int n, int ldn, int k0, int kb,
                                                  const double* __restrict__ Tw, const double* __restrict__ Pw,
                                                  int tm, int tn, int mode, int nk0, int nkb) {
  using T = SweepTile;
  extern __shared__ double smem[];
  const int m0 = tm * T::BM, n0 = tn * T::BN;
  // Tiles entirely inside the K block rows or columns have nothing to update.
  if ((m0 >= k0 && m0 + T::BM <= k0 + kb) || (n0 >= k0 && n0 + T::BN <= k0 + kb)) return;
  if (mode != 0) {
    const bool touches = (m0 < nk0 + nkb && m0 + T::BM > nk0) || (n0 < nk0 + nkb && n0 + T::BN > nk0);
    if (touches != (mode == 1)) return;
  }
  double acc[T::MI][T::NJ][2];
#pragma unroll
  for (int i = 0; i < T::MI; ++i)
#pragma unroll
    for (int j = 0; j < T::NJ; ++j) acc[i][j][0] = acc[i][j][1] = 0.0;
  f64_mainloop<T>(acc, smem, Tw + (size_t)m0 * SWEEP_NB, SWEEP_NB, n - m0, Pw + (size_t)n0 * SWEEP_NB, SWEEP_NB,
                  n - n0, nullptr, kb);
#pragma unroll
  for (int i = 0; i < T::MI; ++i)
#pragma unroll
    for (int j = 0; j < T::NJ; ++j)
#pragma unroll
      for (int e = 0; e < 2; ++e) {
        const int r = m0 + f64_row<T>(i), c = n0 + f64_col<T>(j, e);
        if (r >= n || c >= n || c > r) continue;
        if ((r >= k0 && r < k0 + kb) || (c >= k0 && c < k0 + kb)) continue;
        const double v = A[(size_t)r * ldn + c] - acc[i][j][e];
        A[(size_t)r * ldn + c] = v;
        if (c != r) A[(size_t)c * ldn + r] = v;
      }
}

// Lower tile index t -> (tm, tn), tn <= tm.
__device__ __forceinline__ void lower_tile(int t, int& tm, int& tn) {
  tm = (int)floor((sqrt(8.0 * t + 1.0) - 1.0) * 0.5);
  while ((tm + 1) * (tm + 2) / 2 <= t) ++tm;
  while (tm * (tm + 1) / 2 > t) --tm;
  tn = t - tm * (tm + 1) / 2;
}

__global__ void __launch_bounds__(SweepTile::THREADS) k_sweep_update(double* __restrict__ M, int n, int ldn,
                                                                     size_t stride, int k0, int kb,
                                                                     const double* __restrict__ Tp,
                                                                     const double* __restrict__ Pp,
                                                                     size_t pstride, int mode, int nk0, int nkb) {
  int tm, tn;
  lower_tile(blockIdx.x, tm, tn);
  const int w = blockIdx.y;
  sweep_update_body(M + (size_t)w * stride, n, ldn, k0, kb, Tp + (size_t)w * pstride, Pp + (size_t)w * pstride, tm,
                    tn, mode, nk0, nkb);
}

// Rows [r0, r0 + 32) of the panel write (256 threads).  P[r][q] = the old
// M[r][k0 + q] for rows outside K and q < kb, zero otherwise (a split of P
// then sees no stale values); for q < kb, M[r][k0 + q] = M[k0 + q][r] =
// T[r][q] outside K and -D inside.  The row-major part runs along q; the
// mirror goes through a shared-memory transpose so that it runs along r.  No
// thread reads what another writes: rows outside K read and write only their
// own row, the mirror writes land in rows inside K, and the rows inside K
// read no old value.  Inside the K block both (r, q) and its mirror write the
// same element: D's lower triangle serves both, so the stored value does not
// depend on which write lands last.
constexpr int kWriteRows = 32;
// growth (guarded sweep, else null): max |P| over the rows not yet swept
// (r >= k0 + kb, entries of the Schur complement) joins it.
__device__ __forceinline__ void sweep_write_tile(double* __restrict__ A, int n, int ldn, int k0, int kb,
                                                 const double* __restrict__ Tw, double* __restrict__ Pw,
                                                 const double* __restrict__ D, int r0, unsigned long long* amax,
                                                 unsigned long long* growth) {
  __shared__ double S[kWriteRows][SWEEP_NB + 1];
  __shared__ double red[8];
  double mx = 0.0;  // max|P| of the tile (amax, optional: the bound of a later split of P)
  double gx = 0.0;  // the same over the unswept rows
  for (int e = threadIdx.x; e < kWriteRows * SWEEP_NB; e += blockDim.x) {
    const int rr = e / SWEEP_NB, q = e % SWEEP_NB, r = r0 + rr;
    if (r >= n) continue;
    if (q >= kb) {
      Pw[(size_t)r * SWEEP_NB + q] = 0.0;
      continue;
    }
    const bool in_k = (r >= k0 && r < k0 + kb);
    const double old = in_k ? 0.0 : A[(size_t)r * ldn + k0 + q];
    Pw[(size_t)r * SWEEP_NB + q] = old;
    mx = fmax(mx, fabs(old));
    if (r >= k0 + kb) gx = fmax(gx, isfinite(old) ? fabs(old) : INFINITY);
    const int a = r - k0;
    const double v = in_k ? -D[max(a, q) * SWEEP_NB + min(a, q)] : Tw[(size_t)r * SWEEP_NB + q];
    A[(size_t)r * ldn + k0 + q] = v;
    S[rr][q] = v;
  }
  __syncthreads();
  for (int e = threadIdx.x; e < kWriteRows * SWEEP_NB; e += blockDim.x) {
    const int q = e / kWriteRows, rr = e % kWriteRows, r = r0 + rr;
    if (q < kb && r < n) A[(size_t)(k0 + q) * ldn + r] = S[rr][q];
  }
  if (amax) block_amax(mx, red, amax);
  if (growth) {
    __syncthreads();  // red is reused
    block_amax(gx, red, growth);
  }
}

__global__ void __launch_bounds__(256) k_sweep_write(double* __restrict__ M, int n, int ldn, size_t stride, int k0,
                                                     int kb, const double* __restrict__ Tp, double* __restrict__ Pp,
                                                     size_t pstride, const double* __restrict__ Dp,
                                                     unsigned long long* amax, unsigned long long* growth) {
  const int w = blockIdx.y;
  sweep_write_tile(M + (size_t)w * stride, n, ldn, k0, kb, Tp + (size_t)w * pstride, Pp + (size_t)w * pstride,
                   Dp + (size_t)w * SWEEP_NB * SWEEP_NB, blockIdx.x * kWriteRows, amax ? amax + w : nullptr,
                   growth ? growth + w : nullptr);
}

// After the last sweep M = -eps^-1; Wc = eps^-1 - I = -M - I.  A frequency
// whose eps was singular gets Wc = 0 (eps^-1 replaced by the identity).  With
// half_lower the output is W' = strict lower triangle of Wc + diag(Wc) / 2 and
// zeros above, so that b^T Wc b = 2 b^T W' b needs only the lower triangle.
// Row r of the finish (one block per row).
// Rows [8 b, 8 b + 8) of the finish, one warp per row with the lanes along it
// (a block per row left each block ~1 KB of work and the launch bound by
// block scheduling).
constexpr int kFinishRows = 8;
__device__ __forceinline__ void finish_wc_rows(double* __restrict__ A, int n, int ldn, bool singular, int half_lower,
                                               int b) {
  const int r = kFinishRows * b + (threadIdx.x >> 5), lane = threadIdx.x & 31;
  if (r >= n) return;
  double* row = A + (size_t)r * ldn;
  for (int c = lane; c < n; c += 32) {
    double v = singular ? 0.0 : -row[c] - (r == c ? 1.0 : 0.0);
    if (half_lower) v = (c < r) ? v : (c == r ? 0.5 * v : 0.0);
    row[c] = v;
  }
}

__global__ void __launch_bounds__(32 * kFinishRows) k_finish_wc(double* __restrict__ M, int n, int ldn, size_t stride,
                                                               const int* __restrict__ status, int half_lower) {
  const int w = blockIdx.y;
  finish_wc_rows(M + (size_t)w * stride, n, ldn, status[w] != 0, half_lower, blockIdx.x);
}

static_assert(kSweepPanelCols == SWEEP_NB, "panel width");

// Grouped forms of the sweep kernels (defined below).
template <bool GUARD>
__global__ void k_gsweep_diag(const GMat* __restrict__ mats, int k0, double* __restrict__ Dp,
                              int* __restrict__ status, const unsigned long long* __restrict__ gamax,
                              unsigned long long* __restrict__ growth);
__global__ void k_gsweep_tpanel(const GMat* __restrict__ mats, const int* __restrict__ pre, int count, int k0,
                                const double* __restrict__ Dp, double* __restrict__ Tcat, unsigned long long* amax);
__global__ void k_gsweep_update(const GMat* __restrict__ mats, const int* __restrict__ pre, int count, int k0,
                                const double* __restrict__ Tcat, const double* __restrict__ Pcat);

void sweep_set_attributes() {
  const int diag_smem = (int)((SWEEP_NB * SWEEP_NB + SWEEP_NB * 33) * sizeof(double));
  QX_CUDA(cudaFuncSetAttribute(k_sweep_diag<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, diag_smem));
  QX_CUDA(cudaFuncSetAttribute(k_sweep_diag<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, diag_smem));
  QX_CUDA(cudaFuncSetAttribute(k_sweep_tpanel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)PanelTile::SMEM));
  QX_CUDA(cudaFuncSetAttribute(k_sweep_update, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)SweepTile::SMEM));
  QX_CUDA(cudaFuncSetAttribute(k_gsweep_diag<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, diag_smem));
  QX_CUDA(cudaFuncSetAttribute(k_gsweep_diag<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, diag_smem));
  QX_CUDA(cudaFuncSetAttribute(k_gsweep_tpanel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)PanelTile::SMEM));
  QX_CUDA(cudaFuncSetAttribute(k_gsweep_update, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)SweepTile::SMEM));
}

static void sweep_attributes_once(int device) {
  static PerDeviceOnce attr_once;
  attr_once(device, [] { sweep_set_attributes(); });
}

// One block step of the sweep on stream st: D, T, then P and the panel write.
// amax_t / amax_p (optional): [nw] words that receive max|T|, max|P| per
// matrix (zeroed here first) for the split of the trailing update.  gs
// (guarded sweep, else null): its max|eps| words set the pivot tolerance and
// its growth words receive the unswept maxima.
static void sweep_front(qx_ctx* ctx, cudaStream_t st, double* eps, int n, int ldn, size_t stride, int nw, int k0,
                        int kb, double* Tp, double* Dp, double* Pp, size_t pstride, int* status,
                        unsigned long long* amax_t = nullptr, unsigned long long* amax_p = nullptr,
                        const GuardSet* gs = nullptr) {
  if (amax_t) QX_CUDA(cudaMemsetAsync(amax_t, 0, nw * sizeof(unsigned long long), st));
  if (amax_p) QX_CUDA(cudaMemsetAsync(amax_p, 0, nw * sizeof(unsigned long long), st));
  const int diag_smem = (SWEEP_NB * SWEEP_NB + SWEEP_NB * 33) * sizeof(double);
  unsigned long long* gamax = gs ? gs->amax : nullptr;
  unsigned long long* growth = gs ? gs->growth : nullptr;
  if (gs)
    k_sweep_diag<true><<<nw, 512, diag_smem, st>>>(eps, ldn, stride, k0, kb, Dp, status, gamax, growth);
  else
    k_sweep_diag<false><<<nw, 512, diag_smem, st>>>(eps, ldn, stride, k0, kb, Dp, status, nullptr, nullptr);
  check_launch(ctx);
  dim3 tg(ceil_div(n, PanelTile::BM), ceil_div(kb, PanelTile::BN), nw);
  k_sweep_tpanel<<<tg, PanelTile::THREADS, PanelTile::SMEM, st>>>(eps, n, ldn, stride, k0, kb, Dp, Tp, pstride,
                                                                   amax_t);
  check_launch(ctx);
  dim3 wg(ceil_div(n, kWriteRows), nw);
  k_sweep_write<<<wg, 256, 0, st>>>(eps, n, ldn, stride, k0, kb, Tp, Pp, pstride, Dp, amax_p, growth);
  check_launch(ctx);
}

// The guarded matrices of a uniform sweep: all nw of them.
static void guard_uniform(GuardSet& gs, double* eps, int n, int ldn, size_t stride, int nw, int* status) {
  gs.nall = nw;
  gs.mats.resize(nw);
  for (int w = 0; w < nw; ++w) {
    GuardMat& g = gs.mats[w];
    g = GuardMat{};
    g.M = eps + (size_t)w * stride;
    g.n = n;
    g.ldn = ldn;
    g.idx = w;
    g.status = status + w;
  }
}

static void sweep_update(qx_ctx* ctx, cudaStream_t st, double* eps, int n, int ldn, size_t stride, int nw, int k0,
                         int kb, const double* Tp, const double* Pp, size_t pstride, int mode, int nk0, int nkb) {
  const int tiles = ceil_div(n, SweepTile::BM);
  dim3 ug(tiles * (tiles + 1) / 2, nw);
  k_sweep_update<<<ug, SweepTile::THREADS, SweepTile::SMEM, st>>>(eps, n, ldn, stride, k0, kb, Tp, Pp, pstride, mode,
                                                                  nk0, nkb);
  check_launch(ctx);
}

void launch_invert_wc(qx_ctx* ctx, double* eps, int n, int ldn, size_t stride, int nw, int guard, int half_lower,
                      int split_update) {
  QX_REQUIRE(nw >= 1 && nw <= 65535, QX_ERR_INVALID_INPUT, "%d matrices in one sweep (1 to 65535)", nw);
  // The split trailing update's error bound needs eps >= I: guarded matrices
  // are swept with FP64 updates.
  if (guard) split_update = 0;
  const size_t pstride = (size_t)n * SWEEP_NB;
  const size_t dsz = (size_t)nw * SWEEP_NB * SWEEP_NB;
  DevBuf& pan = ctx->ws[WS_PANEL];
  // T[2], P[2] (pstride per matrix), D[2]
  pan.reserve((4 * pstride * nw + 2 * dsz) * sizeof(double) + 256);
  double* T0 = pan.as<double>();
  double* T1 = T0 + pstride * nw;
  double* P0 = T1 + pstride * nw;
  double* P1 = P0 + pstride * nw;
  double* D0 = P1 + pstride * nw;
  double* D1 = D0 + dsz;
  double* Tb[2] = {T0, T1};
  double* Pb[2] = {P0, P1};
  double* Db[2] = {D0, D1};
  int* status = status_words(ctx, nw);
  QX_CUDA(cudaMemsetAsync(status, 0, nw * sizeof(int), ctx->stream));
  sweep_attributes_once(ctx->device);
  GuardSet gs;
  if (guard) {
    guard_uniform(gs, eps, n, ldn, stride, nw, status);
    DevBuf& gb = ctx->ws[WS_GUARD];
    gb.reserve(guard_bytes(n, ldn, nw));
    guard_layout(gs, gb.ptr, gb.bytes);
    guard_begin(ctx, gs);
  }
  const GuardSet* gp = guard ? &gs : nullptr;
  const int nsteps = ceil_div(n, SWEEP_NB);
  // Split form: panel splits (two steps in flight) and one tcgen05 error word
  // per update launch, zeroed here on the context stream.
  const bool tc = split_update && nsteps > 1;
  void* split_base = nullptr;
  int* tc_err = nullptr;
  if (tc) {
    DevBuf& sb = ctx->ws[WS_SWEEP_SPLIT];
    sb.reserve((size_t)2 * 4 * nw * n * SWEEP_NB * 2);
    split_base = sb.ptr;
    tc_err = status_words(ctx, 2 * nsteps);
    QX_CUDA(cudaMemsetAsync(tc_err, 0, 2 * nsteps * sizeof(int), ctx->stream));
  }
  if (nsteps == 1) {
    sweep_front(ctx, ctx->stream, eps, n, ldn, stride, nw, 0, n, T0, D0, P0, pstride, status, nullptr, nullptr, gp);
  } else {
    // Look-ahead: critical chain (D, T, write, next-block update) on a
    // high-priority stream, the remaining trailing update on a low-priority one.
    if (!ctx->sweep_hi) {
      int lo = 0, hi = 0;
      QX_CUDA(cudaDeviceGetStreamPriorityRange(&lo, &hi));
      if (ctx->worker) lo = hi = 0;
      QX_CUDA(cudaStreamCreateWithPriority(&ctx->sweep_hi, cudaStreamNonBlocking, hi));
      QX_CUDA(cudaStreamCreateWithPriority(&ctx->sweep_lo, cudaStreamNonBlocking, lo));
      for (auto& e : ctx->sweep_ev) QX_CUDA(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
    }
    cudaStream_t s0 = ctx->sweep_hi, s1 = ctx->sweep_lo;
    cudaEvent_t ev_start = ctx->sweep_ev[0], ev_front = ctx->sweep_ev[1], ev_rest = ctx->sweep_ev[2],
                ev_done = ctx->sweep_ev[3];
    QX_CUDA(cudaEventRecord(ev_start, ctx->stream));
    QX_CUDA(cudaStreamWaitEvent(s0, ev_start, 0));
    QX_CUDA(cudaStreamWaitEvent(s1, ev_start, 0));
    for (int step = 0; step < nsteps; ++step) {
      const int k0 = step * SWEEP_NB, kb = min(SWEEP_NB, n - k0);
      const int b = step & 1;
      sweep_front(ctx, s0, eps, n, ldn, stride, nw, k0, kb, Tb[b], Db[b], Pb[b], pstride, status,
                  tc ? split_amax_words(ctx, 3 + 2 * b) : nullptr, tc ? split_amax_words(ctx, 4 + 2 * b) : nullptr,
                  gp);
      SweepSplit sp{};
      if (tc) sp = launch_sweep_split(ctx, s0, Tb[b], Pb[b], n, kb, nw, b, split_base);
      // The previous step's trailing update must be done before this step's
      // updates touch the same tiles.
      if (step > 0) QX_CUDA(cudaStreamWaitEvent(s0, ev_rest, 0));
      if (step + 1 < nsteps) {
        const int nk0 = k0 + SWEEP_NB, nkb = min(SWEEP_NB, n - nk0);
        QX_CUDA(cudaEventRecord(ev_front, s0));
        if (tc)
          launch_sweep_update_tc(ctx, s0, eps, n, ldn, stride, nw, step, sp, 1, step + 1, tc_err + 2 * step);
        else
          sweep_update(ctx, s0, eps, n, ldn, stride, nw, k0, kb, Tb[b], Pb[b], pstride, 1, nk0, nkb);
        QX_CUDA(cudaStreamWaitEvent(s1, ev_front, 0));
        if (tc)
          launch_sweep_update_tc(ctx, s1, eps, n, ldn, stride, nw, step, sp, 2, step + 1, tc_err + 2 * step + 1);
        else
          sweep_update(ctx, s1, eps, n, ldn, stride, nw, k0, kb, Tb[b], Pb[b], pstride, 2, nk0, nkb);
        QX_CUDA(cudaEventRecord(ev_rest, s1));
      } else if (tc) {
        launch_sweep_update_tc(ctx, s0, eps, n, ldn, stride, nw, step, sp, 0, -1, tc_err + 2 * step);
      } else {
        sweep_update(ctx, s0, eps, n, ldn, stride, nw, k0, kb, Tb[b], Pb[b], pstride, 0, 0, 0);
      }
    }
    QX_CUDA(cudaEventRecord(ev_done, s0));
    QX_CUDA(cudaStreamWaitEvent(ctx->stream, ev_done, 0));
  }
  // Guarded: the flagged matrices are inverted again with pivoting.
  if (guard) guard_end(ctx, gs);
  dim3 fg(ceil_div(n, kFinishRows), nw);
  k_finish_wc<<<fg, 256, 0, ctx->stream>>>(eps, n, ldn, stride, status, half_lower);
  check_launch(ctx);
  ctx->pending.push_back({status, nw, 1});
  if (tc) ctx->pending.push_back({tc_err, 2 * nsteps, 0});
}

void launch_invert_wc_panels(qx_ctx* ctx, double* eps, int n, int ldn, size_t stride, int nw, double* Tp,
                             double* Dp, double* Pp, int* status, void* guard_mem, size_t guard_mem_bytes) {
  const size_t pstride = (size_t)n * SWEEP_NB;
  GuardSet gs;
  if (guard_mem) {
    guard_uniform(gs, eps, n, ldn, stride, nw, status);
    guard_layout(gs, guard_mem, guard_mem_bytes);
    guard_begin(ctx, gs);
  }
  const GuardSet* gp = guard_mem ? &gs : nullptr;
  for (int k0 = 0; k0 < n; k0 += SWEEP_NB) {
    const int kb = min(SWEEP_NB, n - k0);
    sweep_front(ctx, ctx->stream, eps, n, ldn, stride, nw, k0, kb, Tp, Dp, Pp, pstride, status, nullptr, nullptr, gp);
    sweep_update(ctx, ctx->stream, eps, n, ldn, stride, nw, k0, kb, Tp, Pp, pstride, 0, 0, 0);
  }
  if (guard_mem) guard_end(ctx, gs);
  dim3 fg(ceil_div(n, kFinishRows), nw);
  k_finish_wc<<<fg, 256, 0, ctx->stream>>>(eps, n, ldn, stride, status, 0);
  check_launch(ctx);
}

// ---------------------------------------------------------------------------
// Grouped block sweep: the kernels above over a table of matrices of
// different orders.  A CTA finds its matrix by binary search in a prefix
// table of per-matrix CTA counts (matrices sorted by order, largest first, so
// those still active at a step are a prefix).
// ---------------------------------------------------------------------------
__device__ __forceinline__ int group_of(const int* __restrict__ pre, int count, int b) {
  int lo = 0, hi = count - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (__ldg(pre + mid) <= b)
      lo = mid;
    else
      hi = mid - 1;
  }
  return lo;
}

template <bool GUARD>
__global__ void __launch_bounds__(512) k_gsweep_diag(const GMat* __restrict__ mats, int k0, double* __restrict__ Dp,
                                                     int* __restrict__ status,
                                                     const unsigned long long* __restrict__ gamax,
                                                     unsigned long long* __restrict__ growth) {
  const int g = blockIdx.x;
  const GMat m = mats[g];
  const bool guarded = GUARD && m.guard;
  sweep_diag_body<GUARD>(m.M + (size_t)k0 * m.ldn + k0, m.ldn, min(SWEEP_NB, m.n - k0),
                         Dp + (size_t)g * SWEEP_NB * SWEEP_NB, status + g, guarded ? guard_tol(gamax, g) : 0.0,
                         guarded ? growth + g : nullptr);
}

// Two 64-column tiles per 64 rows: all 128 panel columns are written (zero past kb).
__global__ void __launch_bounds__(PanelTile::THREADS) k_gsweep_tpanel(const GMat* __restrict__ mats,
                                                                      const int* __restrict__ pre, int count, int k0,
                                                                      const double* __restrict__ Dp,
                                                                      double* __restrict__ Tcat,
                                                                      unsigned long long* amax) {
  const int g = group_of(pre, count, blockIdx.x);
  const int t = blockIdx.x - pre[g];
  const GMat m = mats[g];
  sweep_tpanel_body(m.M, m.n, m.ldn, k0, min(SWEEP_NB, m.n - k0), Dp + (size_t)g * SWEEP_NB * SWEEP_NB,
                    Tcat + (size_t)m.prow * SWEEP_NB, (t >> 1) * PanelTile::BM, (t & 1) * PanelTile::BN, amax);
}

__global__ void __launch_bounds__(256) k_gsweep_write(const GMat* __restrict__ mats, const int* __restrict__ pre,
                                                      int count, int k0, const double* __restrict__ Tcat,
                                                      double* __restrict__ Pcat, const double* __restrict__ Dp,
                                                      unsigned long long* amax, unsigned long long* growth) {
  const int g = group_of(pre, count, blockIdx.x);
  const GMat m = mats[g];
  sweep_write_tile(m.M, m.n, m.ldn, k0, min(SWEEP_NB, m.n - k0), Tcat + (size_t)m.prow * SWEEP_NB,
                   Pcat + (size_t)m.prow * SWEEP_NB, Dp + (size_t)g * SWEEP_NB * SWEEP_NB,
                   (blockIdx.x - pre[g]) * kWriteRows, amax, (growth && m.guard) ? growth + g : nullptr);
}

__global__ void __launch_bounds__(SweepTile::THREADS) k_gsweep_update(const GMat* __restrict__ mats,
                                                                      const int* __restrict__ pre, int count, int k0,
                                                                      const double* __restrict__ Tcat,
                                                                      const double* __restrict__ Pcat) {
  const int g = group_of(pre, count, blockIdx.x);
  const GMat m = mats[g];
  int tm, tn;
  lower_tile(blockIdx.x - pre[g], tm, tn);
  sweep_update_body(m.M, m.n, m.ldn, k0, min(SWEEP_NB, m.n - k0), Tcat + (size_t)m.prow * SWEEP_NB,
                    Pcat + (size_t)m.prow * SWEEP_NB, tm, tn, 0, 0, 0);
}

__global__ void __launch_bounds__(32 * kFinishRows) k_gfinish_wc(const GMat* __restrict__ mats,
                                                                 const int* __restrict__ pre, int count,
                                                                 const int* __restrict__ status, int half_lower) {
  const int g = group_of(pre, count, blockIdx.x);
  const GMat m = mats[g];
  finish_wc_rows(m.M, m.n, m.ldn, status[g] != 0, half_lower, blockIdx.x - pre[g]);
}

// Zero the padding rows [n, n rounded up to 128) of each matrix's panels
// (read by the tcgen05 tiles and the splits, written by no sweep kernel).
__global__ void k_gzero_pad(const GMat* __restrict__ mats, double* __restrict__ Tcat, double* __restrict__ Pcat) {
  const GMat m = mats[blockIdx.x];
  const int rows = (m.n + SWEEP_NB - 1) / SWEEP_NB * SWEEP_NB - m.n;
  for (int idx = threadIdx.x; idx < rows * SWEEP_NB; idx += blockDim.x) {
    const size_t at = (size_t)(m.prow + m.n) * SWEEP_NB + idx;
    Tcat[at] = 0.0;
    Pcat[at] = 0.0;
  }
}

void launch_invert_wc_group(qx_ctx* ctx, const GMat* mats_in, int G, int half_lower, int split_update) {
  QX_REQUIRE(mats_in && G > 0, QX_ERR_INVALID_INPUT, "empty matrix group");
  std::vector<int> ord(G);
  for (int i = 0; i < G; ++i) ord[i] = i;
  std::stable_sort(ord.begin(), ord.end(), [&](int a, int b) { return mats_in[a].n > mats_in[b].n; });
  std::vector<GMat> m(G);
  int prow = 0;
  for (int i = 0; i < G; ++i) {
    m[i] = mats_in[ord[i]];
    QX_REQUIRE(m[i].M && m[i].n > 0 && m[i].n <= 32768 && m[i].ldn >= m[i].n, QX_ERR_INVALID_INPUT,
               "grouped sweep: matrix %d has n=%d ldn=%d", ord[i], m[i].n, m[i].ldn);
    m[i].prow = prow;
    QX_REQUIRE((size_t)prow + round_up(m[i].n, SWEEP_NB) < (1u << 30), QX_ERR_INVALID_INPUT,
               "grouped sweep: too many panel rows");
    prow += round_up(m[i].n, SWEEP_NB);
  }
  const int R = prow;
  const int nsteps = ceil_div(m[0].n, SWEEP_NB);
  bool any_guard = false;
  for (int i = 0; i < G; ++i) any_guard = any_guard || m[i].guard;
  const bool tc = split_update != 0 && !any_guard;
  // Prefix tables: per step the tpanel, write and update CTA counts of the
  // active matrices, then the finish counts of all.
  std::vector<int> tab;
  auto add_table = [&](int count, auto tiles) {
    const size_t off = tab.size();
    long long acc = 0;
    for (int g = 0; g < count; ++g) {
      tab.push_back((int)acc);
      acc += tiles(m[g]);
    }
    QX_REQUIRE(acc < (1ll << 31), QX_ERR_INVALID_INPUT, "grouped sweep: too many CTAs");
    tab.push_back((int)acc);
    return off;
  };
  std::vector<int> act(nsteps), rows_act(nsteps);
  std::vector<size_t> off_tp(nsteps), off_wr(nsteps), off_up(nsteps);
  for (int s = 0; s < nsteps; ++s) {
    const int k0 = s * SWEEP_NB;
    int a = 0;
    while (a < G && m[a].n > k0) ++a;
    act[s] = a;
    rows_act[s] = m[a - 1].prow + round_up(m[a - 1].n, SWEEP_NB);
    off_tp[s] = add_table(a, [](const GMat& x) { return (long long)ceil_div(x.n, PanelTile::BM) * 2; });
    off_wr[s] = add_table(a, [](const GMat& x) { return (long long)ceil_div(x.n, kWriteRows); });
    if (tc)
      off_up[s] = add_table(a, [](const GMat& x) {
        const long long t = ceil_div(x.n, SWEEP_NB);
        return t * (t + 1) / 2;
      });
    else
      off_up[s] = add_table(a, [](const GMat& x) {
        const long long t = ceil_div(x.n, SweepTile::BM);
        return t * (t + 1) / 2;
      });
  }
  const size_t off_fin = add_table(G, [](const GMat& x) { return (long long)ceil_div(x.n, kFinishRows); });
  // Workspace: T, P [R][128] FP64, D [G][128][128], the matrix and prefix tables.
  const size_t pan = (size_t)R * SWEEP_NB;
  const size_t dsz = (size_t)G * SWEEP_NB * SWEEP_NB;
  DevBuf& wb = ctx->ws[WS_PANEL];
  wb.reserve((2 * pan + dsz) * sizeof(double) + G * sizeof(GMat) + tab.size() * sizeof(int) + 512);
  double* Tcat = wb.as<double>();
  double* Pcat = Tcat + pan;
  double* Dp = Pcat + pan;
  GMat* d_mats = reinterpret_cast<GMat*>(Dp + dsz);
  int* d_tab = reinterpret_cast<int*>(d_mats + G);
  QX_CUDA(cudaMemcpyAsync(d_mats, m.data(), G * sizeof(GMat), cudaMemcpyHostToDevice, ctx->stream));
  QX_CUDA(cudaMemcpyAsync(d_tab, tab.data(), tab.size() * sizeof(int), cudaMemcpyHostToDevice, ctx->stream));
  int* status = status_words(ctx, G);
  QX_CUDA(cudaMemsetAsync(status, 0, G * sizeof(int), ctx->stream));
  // Guarded matrices (those the caller cannot show to be >= I).
  GuardSet gs;
  gs.nall = G;
  for (int g = 0; g < G; ++g)
    if (m[g].guard) {
      GuardMat gm{};
      gm.M = m[g].M;
      gm.n = m[g].n;
      gm.ldn = m[g].ldn;
      gm.idx = g;
      gm.status = status + g;
      gs.mats.push_back(gm);
    }
  const bool guarded = !gs.mats.empty();
  // As launch_invert_wc: no split trailing update once any matrix is guarded.
  if (guarded) split_update = 0;
  if (guarded) {
    size_t bytes = 0;
    for (const GuardMat& gm : gs.mats) bytes += guard_bytes(gm.n, gm.ldn, 1);
    bytes += guard_bytes(0, 0, G);
    DevBuf& gb = ctx->ws[WS_GUARD];
    gb.reserve(bytes);
    guard_layout(gs, gb.ptr, gb.bytes);
    guard_begin(ctx, gs);
  }
  unsigned long long* gamax = guarded ? gs.amax : nullptr;
  unsigned long long* ggrowth = guarded ? gs.growth : nullptr;
  int* tc_err = nullptr;
  void* split_base = nullptr;
  if (tc) {
    tc_err = status_words(ctx, nsteps);
    QX_CUDA(cudaMemsetAsync(tc_err, 0, nsteps * sizeof(int), ctx->stream));
    DevBuf& sb = ctx->ws[WS_SWEEP_SPLIT];
    sb.reserve(pan * 2 * 4 + 256);
    split_base = sb.ptr;
  }
  sweep_attributes_once(ctx->device);
  k_gzero_pad<<<G, 256, 0, ctx->stream>>>(d_mats, Tcat, Pcat);
  check_launch(ctx);
  const int diag_smem = (SWEEP_NB * SWEEP_NB + SWEEP_NB * 33) * sizeof(double);
  for (int s = 0; s < nsteps; ++s) {
    const int k0 = s * SWEEP_NB, a = act[s];
    if (guarded)
      k_gsweep_diag<true><<<a, 512, diag_smem, ctx->stream>>>(d_mats, k0, Dp, status, gamax, ggrowth);
    else
      k_gsweep_diag<false><<<a, 512, diag_smem, ctx->stream>>>(d_mats, k0, Dp, status, nullptr, nullptr);
    check_launch(ctx);
    // Split form: the panel and write kernels accumulate max|T|, max|P| over
    // all matrices (one scale each) for the splits.
    unsigned long long* amax_t = tc ? split_amax_words(ctx, 3) : nullptr;
    unsigned long long* amax_p = tc ? split_amax_words(ctx, 4) : nullptr;
    if (tc) {
      QX_CUDA(cudaMemsetAsync(amax_t, 0, sizeof(unsigned long long), ctx->stream));
      QX_CUDA(cudaMemsetAsync(amax_p, 0, sizeof(unsigned long long), ctx->stream));
    }
    k_gsweep_tpanel<<<tab[off_tp[s] + a], PanelTile::THREADS, PanelTile::SMEM, ctx->stream>>>(
        d_mats, d_tab + off_tp[s], a, k0, Dp, Tcat, amax_t);
    check_launch(ctx);
    k_gsweep_write<<<tab[off_wr[s] + a], 256, 0, ctx->stream>>>(d_mats, d_tab + off_wr[s], a, k0, Tcat, Pcat, Dp,
                                                                amax_p, ggrowth);
    check_launch(ctx);
    if (tc) {
      uint8_t* b = static_cast<uint8_t*>(split_base);
      TcOperand T{b, b + pan * 2, nullptr}, P{b + pan * 4, b + pan * 6, nullptr};
      const int rows = rows_act[s];
      launch_split(ctx, Tcat, rows, SWEEP_NB, SWEEP_NB, T.hi, T.lo, SWEEP_NB, 0, 0, 1, 1, 3, &T.scale, amax_t);
      launch_split(ctx, Pcat, rows, SWEEP_NB, SWEEP_NB, P.hi, P.lo, SWEEP_NB, 0, 0, 1, 1, 4, &P.scale, amax_p);
      launch_gsweep_update_tc(ctx, d_mats, d_tab + off_up[s], a, tab[off_up[s] + a], s, T, P, rows, tc_err + s);
    } else {
      k_gsweep_update<<<tab[off_up[s] + a], SweepTile::THREADS, SweepTile::SMEM, ctx->stream>>>(
          d_mats, d_tab + off_up[s], a, k0, Tcat, Pcat);
      check_launch(ctx);
    }
  }
  if (guarded) guard_end(ctx, gs);
  k_gfinish_wc<<<tab[off_fin + G], 256, 0, ctx->stream>>>(d_mats, d_tab + off_fin, G, status, half_lower);
  check_launch(ctx);
  ctx->pending.push_back({status, G, 1});
  if (tc) ctx->pending.push_back({tc_err, nsteps, 0});
}

// ---------------------------------------------------------------------------
// Gathers.
// bpt[p][P] = lpq[P][pairs[p].x][pairs[p].y]   (tiled transpose through smem)
// ---------------------------------------------------------------------------
// Tiles of 32 pairs x 32 aux rows, pair block fastest; a block walks the tiles
// blockIdx.x, blockIdx.x + gridDim.x, ... (one tile each on a full grid; a
// grid of one block per SM when lpq is host memory read over the host link,
// which leaves room on every SM for the kernels that run beside it).
__global__ void k_gather_pairs(const double* __restrict__ lpq, int naux, int nmo, const int2* __restrict__ pairs,
                               int npair, double* __restrict__ bpt, int ldk) {
  __shared__ double tile[32][33];
  __shared__ int off[32];
  const int npb = (npair + 31) / 32, ntiles = npb * ((ldk + 31) / 32);
  for (int t = blockIdx.x; t < ntiles; t += gridDim.x) {
    const int Pb = t / npb;
    const int p0 = (t - Pb * npb) * 32, P0 = Pb * 32;
    if (threadIdx.y == 0) {
      int p = p0 + threadIdx.x;
      off[threadIdx.x] = (p < npair) ? pairs[p].x * nmo + pairs[p].y : 0;
    }
    __syncthreads();
    for (int r = threadIdx.y; r < 32; r += blockDim.y) {
      int P = P0 + r, p = p0 + threadIdx.x;
      tile[r][threadIdx.x] = (P < naux && p < npair) ? lpq[(size_t)P * nmo * nmo + off[threadIdx.x]] : 0.0;
    }
    __syncthreads();
    for (int r = threadIdx.y; r < 32; r += blockDim.y) {
      int p = p0 + r, P = P0 + threadIdx.x;
      if (p < npair && P < ldk) bpt[(size_t)p * ldk + P] = (P < naux) ? tile[threadIdx.x][r] : 0.0;
    }
    __syncthreads();
  }
}

void launch_gather_pairs(qx_ctx* ctx, cudaStream_t st, const double* lpq, int naux, int nmo, const int2* pairs,
                         int npair, double* bpt, int ldk, int max_blocks) {
  if (npair <= 0) return;
  const int ntiles = ceil_div(npair, 32) * ceil_div(ldk, 32);
  const int grid = max_blocks > 0 ? std::min(ntiles, max_blocks) : ntiles;
  k_gather_pairs<<<grid, dim3(32, 8), 0, st>>>(lpq, naux, nmo, pairs, npair, bpt, ldk);
  check_launch(ctx);
}

// bov[P][i*nvir + a] = lpq[P][i][nocc + a]
// bov[P][i nvir + a] = lpq[P][i][nocc + a], zero in the padding columns
// [nocc nvir, ldov): block (i, P) copies one contiguous run of nvir values
// (block i = nocc writes the padding), so no index is divided.
__global__ void k_gather_ov(const double* __restrict__ lpq, int naux, int nmo, int nocc, double* __restrict__ bov,
                            int ldov) {
  const int i = blockIdx.x, P = blockIdx.y;
  const int nvir = nmo - nocc;
  double* dst = bov + (size_t)P * ldov;
  if (i == nocc) {
    for (int k = nocc * nvir + threadIdx.x; k < ldov; k += blockDim.x) dst[k] = 0.0;
    return;
  }
  const double* src = lpq + (size_t)P * nmo * nmo + (size_t)i * nmo + nocc;
  for (int a = threadIdx.x; a < nvir; a += blockDim.x) dst[(size_t)i * nvir + a] = src[a];
}

void launch_gather_ov(qx_ctx* ctx, const double* lpq, int naux, int nmo, int nocc, double* bov, int ldov) {
  dim3 grid(nocc + 1, naux);
  k_gather_ov<<<grid, 128, 0, ctx->stream>>>(lpq, naux, nmo, nocc, bov, ldov);
  check_launch(ctx);
}

// bov[P][i nvir + a] = bpt[pair(i, nocc + a)][P], zero in the padding columns
// [nocc nvir, ldov), when every orbital is a target (row i of the pair index
// table pidx lists the pairs of orbital i).  The occupied-virtual block is
// then transposed out of the gathered pair tensor instead of being read from
// lpq a second time (lpq may be host memory read in place).  Tiled transpose
// through shared memory: 32 columns x 32 aux rows per block.
__global__ void k_ov_from_pairs(const double* __restrict__ bpt, int ldk, const int* __restrict__ pidx, int naux,
                                int nmo, int nocc, double* __restrict__ bov, int ldov) {
  __shared__ double tile[32][33];
  __shared__ int row[32];
  const int c0 = blockIdx.x * 32, P0 = blockIdx.y * 32;
  const int nvir = nmo - nocc, nov = nocc * nvir;
  if (threadIdx.y == 0) {
    const int c = c0 + threadIdx.x;
    int r = -1;
    if (c < nov) {
      const int i = c / nvir;
      r = pidx[(size_t)i * nmo + nocc + (c - i * nvir)];
    }
    row[threadIdx.x] = r;
  }
  __syncthreads();
  for (int cc = threadIdx.y; cc < 32; cc += blockDim.y) {
    const int r = row[cc], P = P0 + threadIdx.x;
    tile[cc][threadIdx.x] = (r >= 0 && P < naux) ? bpt[(size_t)r * ldk + P] : 0.0;
  }
  __syncthreads();
  for (int pp = threadIdx.y; pp < 32; pp += blockDim.y) {
    const int P = P0 + pp, c = c0 + threadIdx.x;
    if (P < naux && c < ldov) bov[(size_t)P * ldov + c] = tile[threadIdx.x][pp];
  }
}

void launch_ov_from_pairs(qx_ctx* ctx, const double* bpt, int ldk, const int* pidx, int naux, int nmo, int nocc,
                          double* bov, int ldov) {
  dim3 grid(ceil_div(ldov, 32), ceil_div(naux, 32));
  k_ov_from_pairs<<<grid, dim3(32, 8), 0, ctx->stream>>>(bpt, ldk, pidx, naux, nmo, nocc, bov, ldov);
  check_launch(ctx);
}

// sx[t] = -sum_{i < nocc} sum_R bpt[pair(t, i)][R]^2 for the targets t (row
// t of pidx): the exchange diagonal of qp/evgw.rs:1167-1193 read from the
// gathered pair tensor, whose rows are contiguous in R, instead of from
// lpq's scattered lpq[R][t][i].  One block per target, a fixed summation
// order (per thread over i and R, then a tree over the block).
__global__ void __launch_bounds__(256) k_exchange_pairs(const double* __restrict__ bpt, int ldk,
                                                        const int* __restrict__ pidx, int naux, int nmo, int nocc,
                                                        double* __restrict__ sx) {
  const int t = blockIdx.x;
  double s0 = 0.0, s1 = 0.0;
  for (int i = 0; i < nocc; ++i) {
    const double* row = bpt + (size_t)__ldg(pidx + (size_t)t * nmo + i) * ldk;
    int R = threadIdx.x;
    for (; R + 256 < naux; R += 512) {
      const double u = __ldg(row + R), v = __ldg(row + R + 256);
      s0 += u * u;
      s1 += v * v;
    }
    if (R < naux) {
      const double u = __ldg(row + R);
      s0 += u * u;
    }
  }
  __shared__ double red[256];
  red[threadIdx.x] = s0 + s1;
  __syncthreads();
  for (int o = 128; o > 0; o >>= 1) {
    if (threadIdx.x < o) red[threadIdx.x] += red[threadIdx.x + o];
    __syncthreads();
  }
  if (threadIdx.x == 0) sx[t] = -red[0];
}

void launch_exchange_pairs(qx_ctx* ctx, const double* bpt, int ldk, const int* pidx, int naux, int nmo, int nocc,
                           int norbs, double* sx) {
  k_exchange_pairs<<<norbs, 256, 0, ctx->stream>>>(bpt, ldk, pidx, naux, nmo, nocc, sx);
  check_launch(ctx);
}

// sx[p] = -sum_{R,i} lpq[R][p][i]^2   (qp/evgw.rs:1167-1193).  One block of
// 1024 threads per orbital; each thread keeps four loads in flight (the
// elements are scattered over naux rows, so latency, not bandwidth, bounds a
// block), and the sum has a fixed order.
__global__ void __launch_bounds__(1024) k_exchange_diag(const double* __restrict__ lpq, int naux, int nmo, int nocc,
                                                        const int* __restrict__ orbs, double* __restrict__ sx) {
  const int p = orbs ? orbs[blockIdx.x] : blockIdx.x;
  const int total = naux * nocc;
  double s[4] = {0.0, 0.0, 0.0, 0.0};
  for (int idx = threadIdx.x; idx < total; idx += 4 * blockDim.x) {
#pragma unroll
    for (int u = 0; u < 4; ++u) {
      const int k = idx + u * blockDim.x;
      if (k < total) {
        const int R = k / nocc, i = k % nocc;
        const double v = __ldg(lpq + (size_t)R * nmo * nmo + (size_t)p * nmo + i);
        s[u] += v * v;
      }
    }
  }
  __shared__ double red[1024];
  red[threadIdx.x] = (s[0] + s[1]) + (s[2] + s[3]);
  __syncthreads();
  for (int o = 512; o > 0; o >>= 1) {
    if (threadIdx.x < o) red[threadIdx.x] += red[threadIdx.x + o];
    __syncthreads();
  }
  if (threadIdx.x == 0) sx[p] = -red[0];
}

void launch_exchange_diag(qx_ctx* ctx, const double* lpq, int naux, int nmo, int nocc, double* sx,
                          const int* orbs, int norbs) {
  k_exchange_diag<<<orbs ? norbs : nmo, 1024, 0, ctx->stream>>>(lpq, naux, nmo, nocc, orbs, sx);
  check_launch(ctx);
}

// ---------------------------------------------------------------------------
// Pair contraction: v[w][p] = 2 sum_Q Bpt[p][Q] sum_{P <= Q} W'[w][Q][P] Bpt[p][P]
// with W' the half-lower form of Wc (k_finish_wc), i.e. Bpt[p]^T Wc[w] Bpt[p].
// One CTA per (128-pair block, frequency); it walks every Q tile, so the
// per-pair sums stay in shared memory and are written once (deterministic).
// ---------------------------------------------------------------------------
using PairTile = F64Tile<128, 64, 4, 2, 3>;

__global__ void __launch_bounds__(PairTile::THREADS) k_pair_contract_f64(const double* __restrict__ bpt, int ldk,
                                                                         int npair, int naux,
                                                                         const double* __restrict__ wc, int ldn,
                                                                         size_t wc_stride,
                                                                         double* __restrict__ v, int ldv) {
  using T = PairTile;
  extern __shared__ double smem[];
  __shared__ double part[T::WARPS_N][T::BM];
  __shared__ double rowacc[T::BM];
  const int w = blockIdx.y;
  const int m0 = blockIdx.x * T::BM;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int wn = warp % T::WARPS_N;
  for (int i = threadIdx.x; i < T::BM; i += T::THREADS) rowacc[i] = 0.0;
  const double* Wc = wc + (size_t)w * wc_stride;
  const double* Arow = bpt + (size_t)m0 * ldk;
  for (int n0 = 0; n0 < naux; n0 += T::BN) {
    double acc[T::MI][T::NJ][2];
#pragma unroll
    for (int i = 0; i < T::MI; ++i)
#pragma unroll
      for (int j = 0; j < T::NJ; ++j) acc[i][j][0] = acc[i][j][1] = 0.0;
    // W' is lower triangular: rows Q of this tile need P <= Q < n0 + BN only.
    f64_mainloop<T>(acc, smem, Arow, ldk, npair - m0, Wc + (size_t)n0 * ldn, ldn, naux - n0, nullptr,
                    min(naux, n0 + T::BN));
    // Row partials: sum_n acc[m][n] * Bpt[m0+m][n0+n].
#pragma unroll
    for (int i = 0; i < T::MI; ++i) {
      const int m = f64_row<T>(i);
      double s = 0.0;
      if (m0 + m < npair) {
        const double* brow = bpt + (size_t)(m0 + m) * ldk + n0;
#pragma unroll
        for (int j = 0; j < T::NJ; ++j) {
          const int c = f64_col<T>(j, 0);
          if (n0 + c + 1 < naux) {
            double2 bb = *reinterpret_cast<const double2*>(brow + c);
            s += acc[i][j][0] * bb.x + acc[i][j][1] * bb.y;
          } else if (n0 + c < naux) {
            s += acc[i][j][0] * brow[c];
          }
        }
      }
      s += __shfl_xor_sync(0xffffffffu, s, 1);
      s += __shfl_xor_sync(0xffffffffu, s, 2);
      if ((lane & 3) == 0) part[wn][m] = s;
    }
    __syncthreads();
    for (int r = threadIdx.x; r < T::BM; r += T::THREADS) {
      double s = rowacc[r];
#pragma unroll
      for (int q = 0; q < T::WARPS_N; ++q) s += part[q][r];
      rowacc[r] = s;
    }
    __syncthreads();
  }
  for (int r = threadIdx.x; r < T::BM; r += T::THREADS)
    if (m0 + r < npair) v[(size_t)w * ldv + m0 + r] = 2.0 * rowacc[r];
}

void launch_pair_contract_fp64(qx_ctx* ctx, const double* bpt, int ldk, int npair, int naux, const double* wc,
                               int ldn, size_t wc_stride, int nw, double* v, int ldv) {
  using T = PairTile;
  static PerDeviceOnce attr_once;
  attr_once(ctx->device, [&] {
    QX_CUDA(cudaFuncSetAttribute(k_pair_contract_f64, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)T::SMEM));
  });
  dim3 grid(ceil_div(npair, T::BM), nw);
  k_pair_contract_f64<<<grid, T::THREADS, T::SMEM, ctx->stream>>>(bpt, ldk, npair, naux, wc, ldn, wc_stride, v, ldv);
  check_launch(ctx);
}

// ---------------------------------------------------------------------------
// Sigma_c(iw_k) = -(1/pi) sum_w sum_m v[w][pair(t,m)] wts_w emo/(emo^2 + f_w^2),
// emo = s i iw_k + ef - e_m, s = -1 for occupied targets, +1 for virtual
// (correlation_ac.rs:286-314, 404-438).  The Green's-function factors depend
// only on (s, k, w, m), so they are tabulated once per call as
// G[(s, k, re/im)][(w, m)] and the sum becomes one DGEMM
//   C[t][(s, k, c)] = sum_{(w,m)} V[t][(w,m)] G[(s, k, c)][(w,m)],
// with V[t][(w,m)] = v[w][pair(t,m)] gathered first.
// ---------------------------------------------------------------------------
__global__ void k_sigma_gtab(const double* __restrict__ en, double ef, const double* __restrict__ freqs,
                             const double* __restrict__ wts, const double* __restrict__ iw, int nw, int nmo, int nws,
                             double* __restrict__ G, int ldg) {
  const int row = blockIdx.y;  // (s, k, c): s in {occ, vir}
  const int c = row & 1, k = (row >> 1) % nws, sidx = (row >> 1) / nws;
  const double b = (sidx == 0 ? -1.0 : 1.0) * iw[k];
  for (int idx = blockIdx.x * blockDim.x + threadIdx.x; idx < ldg; idx += gridDim.x * blockDim.x) {
    double val = 0.0;
    if (idx < nw * nmo) {
      const int w = idx / nmo, m = idx % nmo;
      const double a = ef - en[m], f2 = freqs[w] * freqs[w], wt = wts[w];
      // emo = a + ib ; den = emo^2 + f^2 = (a^2 - b^2 + f^2) + i 2ab
      const double dr = a * a - b * b + f2, di = 2.0 * a * b;
      const double dd = dr * dr + di * di;
      val = (c == 0) ? wt * (a * dr + b * di) / dd : wt * (b * dr - a * di) / dd;
    }
    G[(size_t)row * ldg + idx] = val;
  }
}

__global__ void k_sigma_gather(const double* __restrict__ v, int ldv, int nw, const int* __restrict__ pidx, int nmo,
                               double* __restrict__ V, int ldg) {
  const int t = blockIdx.y;
  for (int idx = blockIdx.x * blockDim.x + threadIdx.x; idx < ldg; idx += gridDim.x * blockDim.x) {
    double val = 0.0;
    if (idx < nw * nmo) {
      const int w = idx / nmo, m = idx % nmo;
      val = v[(size_t)w * ldv + pidx[(size_t)t * nmo + m]];
    }
    V[(size_t)t * ldg + idx] = val;
  }
}

__global__ void k_sigma_pick(const double* __restrict__ C, int ldc, const int* __restrict__ orbs, int nocc, int norbs,
                             int nws, double* __restrict__ sigma) {
  for (int idx = blockIdx.x * blockDim.x + threadIdx.x; idx < norbs * nws; idx += gridDim.x * blockDim.x) {
    const int t = idx / nws, k = idx % nws;
    const int sidx = orbs[t] < nocc ? 0 : 1;
    const double* c = C + (size_t)t * ldc + 2 * (sidx * nws + k);
    sigma[2 * (size_t)idx] = -c[0] / M_PI;
    sigma[2 * (size_t)idx + 1] = -c[1] / M_PI;
  }
}

size_t sigma_workspace_doubles(int norbs, int nws, int nw, int nmo) {
  const size_t ldg = round_up(nw * nmo, 8), ng = 4 * (size_t)nws;
  return round_up(norbs * nws * 2, 8) + ng * ldg + (size_t)norbs * ldg + (size_t)norbs * ng + 16;
}

void launch_sigma_assemble(qx_ctx* ctx, const double* v, int ldv, int nw, const int* pair_index, int norbs,
                           int nmo, const int* orbs, int nocc, const double* energies, double ef,
                           const double* freqs, const double* wts, const double* iw, int nws,
                           double* sigma) {
  const int K = nw * nmo, ldg = round_up(K, 8), ng = 4 * nws;
  DevBuf& sb = ctx->ws[WS_SIGMA];
  const size_t out = (size_t)norbs * nws * 2;
  QX_REQUIRE(sigma == sb.as<double>() && sb.bytes >= sigma_workspace_doubles(norbs, nws, nw, nmo) * sizeof(double),
             QX_ERR_INVALID_INPUT, "sigma must live in the sized sigma workspace");
  double* G = sb.as<double>() + round_up((int)out, 8);
  double* V = G + (size_t)ng * ldg;
  double* C = V + (size_t)norbs * ldg;
  k_sigma_gtab<<<dim3(std::min(ceil_div(ldg, 256), 1024), ng), 256, 0, ctx->stream>>>(energies, ef, freqs, wts, iw,
                                                                                      nw, nmo, nws, G, ldg);
  check_launch(ctx);
  k_sigma_gather<<<dim3(std::min(ceil_div(ldg, 256), 1024), norbs), 256, 0, ctx->stream>>>(v, ldv, nw, pair_index,
                                                                                         nmo, V, ldg);
  check_launch(ctx);
  GemmNT g{};
  g.M = norbs;
  g.N = ng;
  g.K = ldg;
  g.A = V;
  g.lda = ldg;
  g.B = G;
  g.ldb = ldg;
  g.C = C;
  g.ldc = ng;
  g.batch = 1;
  g.alpha = 1.0;
  g.splitk = 0;
  gemm_nt_f64(ctx, g);
  k_sigma_pick<<<ceil_div(norbs * nws, 256), 256, 0, ctx->stream>>>(C, ng, orbs, nocc, norbs, nws, sigma);
  check_launch(ctx);
}

}  // namespace qx
