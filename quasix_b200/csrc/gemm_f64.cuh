// FP64 tensor-core (DMMA, mma.sync m8n8k4) "NT" GEMM mainloop:
//   acc[m][n] += sum_k A[m][k] * s[k] * B[n][k]
// A and B are row-major with K contiguous (leading dimensions even, base
// 16-byte aligned).  Operand tiles are staged global -> shared with a 3-stage
// cp.async pipeline; rows beyond M/N and columns beyond K are zero-filled.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

namespace qx {

template <int BM_, int BN_, int WARPS_M_, int WARPS_N_, int STAGES_ = 3>
struct F64Tile {
  static constexpr int BM = BM_, BN = BN_, BK = 16, PAD = 4, LDS = BK + PAD;
  static constexpr int WARPS_M = WARPS_M_, WARPS_N = WARPS_N_;
  static constexpr int THREADS = WARPS_M * WARPS_N * 32;
  static constexpr int WM = BM / WARPS_M, WN = BN / WARPS_N;
  static constexpr int MI = WM / 8, NJ = WN / 8;
  static constexpr int STAGES = STAGES_;
  static constexpr int A_ELEMS = BM * LDS, B_ELEMS = BN * LDS;
  static constexpr int STAGE_ELEMS = A_ELEMS + B_ELEMS + BK;  // + scale tile
  static constexpr size_t SMEM = size_t(STAGES) * STAGE_ELEMS * sizeof(double);
  static_assert(WM % 8 == 0 && WN % 8 == 0, "warp tile");
};

__device__ __forceinline__ void dmma_8x8x4(double (&c)[2], double a, double b) {
  asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};\n"
               : "+d"(c[0]), "+d"(c[1])
               : "d"(a), "d"(b));
}

__device__ __forceinline__ void cp_async16(void* smem, const void* gmem, int src_bytes) {
  unsigned s = static_cast<unsigned>(__cvta_generic_to_shared(smem));
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(s), "l"(gmem), "r"(src_bytes));
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::); }
template <int N>
__device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_group %0;\n" ::"n"(N)); }

// Load one BK-wide k-tile of A (rows [0,M)), B (rows [0,N)) and the scale.
template <class T>
__device__ __forceinline__ void f64_load_tile(double* st, const double* A, int lda, int M, const double* B,
                                              int ldb, int N, const double* scale, int K, int k0) {
  double* As = st;
  double* Bs = st + T::A_ELEMS;
  double* Ss = st + T::A_ELEMS + T::B_ELEMS;
  constexpr int CH = T::BK / 2;  // 16-byte chunks per row
  for (int c = threadIdx.x; c < T::BM * CH; c += T::THREADS) {
    int r = c / CH, kc = (c % CH) * 2;
    int kg = k0 + kc;
    int bytes = (r < M) ? max(0, min(2, K - kg)) * 8 : 0;
    const double* src = bytes ? A + (size_t)r * lda + kg : A;
    cp_async16(As + r * T::LDS + kc, src, bytes);
  }
  for (int c = threadIdx.x; c < T::BN * CH; c += T::THREADS) {
    int r = c / CH, kc = (c % CH) * 2;
    int kg = k0 + kc;
    int bytes = (r < N) ? max(0, min(2, K - kg)) * 8 : 0;
    const double* src = bytes ? B + (size_t)r * ldb + kg : B;
    cp_async16(Bs + r * T::LDS + kc, src, bytes);
  }
  if (scale != nullptr) {
    for (int c = threadIdx.x; c < CH; c += T::THREADS) {
      int kg = k0 + c * 2;
      int bytes = max(0, min(2, K - kg)) * 8;
      cp_async16(Ss + c * 2, bytes ? scale + kg : scale, bytes);
    }
  }
}

// Mainloop.  acc must be zeroed by the caller.  smem holds STAGES stages.
template <class T>
__device__ __forceinline__ void f64_mainloop(double (&acc)[T::MI][T::NJ][2], double* smem, const double* A,
                                             int lda, int M, const double* B, int ldb, int N,
                                             const double* scale, int K) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int wm = warp / T::WARPS_N, wn = warp % T::WARPS_N;
  const int ktiles = (K + T::BK - 1) / T::BK;
#pragma unroll
  for (int s = 0; s < T::STAGES - 1; ++s) {
    if (s < ktiles) f64_load_tile<T>(smem + s * T::STAGE_ELEMS, A, lda, M, B, ldb, N, scale, K, s * T::BK);
    cp_async_commit();
  }
  for (int kt = 0; kt < ktiles; ++kt) {
    cp_async_wait<T::STAGES - 2>();
    __syncthreads();
    {
      int nk = kt + T::STAGES - 1;
      if (nk < ktiles)
        f64_load_tile<T>(smem + (nk % T::STAGES) * T::STAGE_ELEMS, A, lda, M, B, ldb, N, scale, K, nk * T::BK);
      cp_async_commit();
    }
    const double* As = smem + (kt % T::STAGES) * T::STAGE_ELEMS;
    const double* Bs = As + T::A_ELEMS;
    const double* Ss = Bs + T::B_ELEMS;
#pragma unroll
    for (int kk = 0; kk < T::BK / 4; ++kk) {
      const int kcol = kk * 4 + (lane & 3);
      double a[T::MI], b[T::NJ];
      double sc = scale ? Ss[kcol] : 1.0;
#pragma unroll
      for (int i = 0; i < T::MI; ++i) a[i] = As[(wm * T::WM + i * 8 + (lane >> 2)) * T::LDS + kcol] * sc;
#pragma unroll
      for (int j = 0; j < T::NJ; ++j) b[j] = Bs[(wn * T::WN + j * 8 + (lane >> 2)) * T::LDS + kcol];
#pragma unroll
      for (int i = 0; i < T::MI; ++i)
#pragma unroll
        for (int j = 0; j < T::NJ; ++j) dmma_8x8x4(acc[i][j], a[i], b[j]);
    }
  }
  cp_async_wait<0>();
  __syncthreads();
}

// Coordinates of accumulator element (i, j, e) of this thread within the CTA tile.
template <class T>
__device__ __forceinline__ int f64_row(int i) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  return (warp / T::WARPS_N) * T::WM + i * 8 + (lane >> 2);
}
template <class T>
__device__ __forceinline__ int f64_col(int j, int e) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  return (warp % T::WARPS_N) * T::WN + j * 8 + (lane & 3) * 2 + e;
}

}  // namespace qx
