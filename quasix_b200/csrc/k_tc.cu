// tcgen05 (5th-generation tensor core) kernels for the split-operand forms.
//
// Each FP64 operand X is split into hi = r(s X) and lo = r(s X - hi), with r()
// rounding to bf16 (BF16X3, s = 1) or to fp16 (FP16X3, s a power of two per
// matrix and frequency that puts max|s X| in [2^14, 2^15)).  A product is
// formed as hi*hi' + hi*lo' + lo*hi' with FP32 accumulation in TMEM and the
// scales divided out in the epilogue.  Relative error per product: ~2^-17
// (bf16 pairs) or ~2^-22 (fp16 pairs), vs 2^-9 / 2^-12 for one product.
//
// One warp-specialised "NT" GEMM serves both contractions of the GW chain:
//   C[m][n] = sum_k A[m][k] B[w][n][k]     (A, B K-major, bf16 hi/lo pairs)
//   EPI_ROWDOT : out[w][m] = sum_n C[m][n] X[m][n]          (Sigma_c pair contraction)
//   EPI_STORE  : out[w][m][n] = C[m][n] + delta_mn (FP64)   (eps = I + B chi B^T)
// Warp 0 issues TMA loads (128B-swizzled K-major tiles), warp 1 allocates TMEM
// and issues tcgen05.mma (M=128, N=BN, K=16), warps 2..5 drain the
// double-buffered TMEM accumulator with tcgen05.ld.  Every wait is bounded:
// on timeout the CTA records an error code and unwinds.
#include <cuda.h>
#include <cuda_bf16.h>
#include <cuda_fp16.h>

#include <array>
#include <map>
#include <cstring>
#include <mutex>
#include <vector>

#include "qx_internal.cuh"
#include "split_round.cuh"

namespace qx {

// ---------------------------------------------------------------------------
// PTX helpers
// ---------------------------------------------------------------------------
__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}
__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;\n" ::"r"(smem_u32(bar)), "r"(count));
}
__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n" ::"r"(smem_u32(bar)), "r"(bytes)
               : "memory");
}
__device__ __forceinline__ void mbar_arrive(uint64_t* bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];\n" ::"r"(smem_u32(bar)) : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
      : "=r"(ok)
      : "r"(smem_u32(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}

// Bounded wait (about one second of SM clock).  Returns false on timeout or
// when another thread of the CTA has already aborted.
constexpr long long WAIT_CYCLES = 2000000000LL;
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity, volatile int* abort_flag,
                                          int* err, int code) {
  if (mbar_try_wait(bar, parity)) return true;
  const long long t0 = clock64();
  while (true) {
    if (mbar_try_wait(bar, parity)) return true;
    if (*abort_flag) return false;
    if (clock64() - t0 > WAIT_CYCLES) {
      *abort_flag = 1;
      atomicCAS(err, 0, code);
      return false;
    }
  }
}

__device__ __forceinline__ void tma_load_2d(void* dst, const CUtensorMap* map, uint64_t* bar, int c0, int c1) {
  asm volatile(
      "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%3, %4}], [%2];\n" ::"r"(
          smem_u32(dst)),
      "l"(map), "r"(smem_u32(bar)), "r"(c0), "r"(c1)
      : "memory");
}
__device__ __forceinline__ void tma_load_3d(void* dst, const CUtensorMap* map, uint64_t* bar, int c0, int c1,
                                            int c2) {
  asm volatile(
      "cp.async.bulk.tensor.3d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%3, %4, %5}], "
      "[%2];\n" ::"r"(smem_u32(dst)),
      "l"(map), "r"(smem_u32(bar)), "r"(c0), "r"(c1), "r"(c2)
      : "memory");
}

__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory"); }

// SM100 shared-memory matrix descriptor (version 1) for a K-major operand tile of BK 16-bit elements per row: BK = 64 uses the 128-byte
// swizzle (layout 2, 8-row groups 1024 bytes apart), BK = 32 the 64-byte swizzle
// (layout 4, 512 bytes apart).
template <int BK>
__device__ __forceinline__ uint64_t umma_desc(uint32_t saddr) {
  static_assert(BK == 32 || BK == 64, "K block of 32 or 64 elements");
  uint64_t d = 0;
  d |= (uint64_t)((saddr & 0x3FFFF) >> 4);          // start address
  d |= (uint64_t)1 << 16;                           // leading byte offset (unused for swizzled K-major)
  d |= (uint64_t)((8 * BK * 2) >> 4) << 32;         // stride byte offset: 8 rows
  d |= (uint64_t)1 << 46;                           // descriptor version (sm_100)
  d |= (uint64_t)(BK == 64 ? 2 : 4) << 61;          // SWIZZLE_128B / SWIZZLE_64B
  return d;
}


// Instruction descriptor: kind::f16 with bf16 (fmt 1) or fp16 (fmt 0) A and B of
// the same type, f32 accumulator, K-major A and B.
__host__ __device__ constexpr uint32_t umma_idesc_f16(int M, int N, int fp16) {
  return (1u << 4) | ((fp16 ? 0u : 1u) << 7) | ((fp16 ? 0u : 1u) << 10) | ((uint32_t)(N >> 3) << 17) |
         ((uint32_t)(M >> 4) << 24);
}

__device__ __forceinline__ void umma_f16(uint32_t tmem_d, uint64_t adesc, uint64_t bdesc, uint32_t idesc,
                                          uint32_t accumulate) {
  asm volatile(
      "{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n}\n" ::"r"(
          tmem_d),
      "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate));
}
__device__ __forceinline__ void umma_commit(uint64_t* bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];\n" ::"r"(smem_u32(bar))
               : "memory");
}
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float (&v)[16]) {
  uint32_t r[16];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];\n"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]), "=r"(r[8]),
        "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
      : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;\n" ::: "memory");
#pragma unroll
  for (int i = 0; i < 16; ++i) v[i] = __uint_as_float(r[i]);
}

// CTA-pair (cluster of two) helpers.
__device__ __forceinline__ uint32_t cluster_ctarank() {
  uint32_t r;
  asm volatile("mov.u32 %0, %%cluster_ctarank;\n" : "=r"(r));
  return r;
}
__device__ __forceinline__ uint32_t cluster_nctarank() {
  uint32_t r;
  asm volatile("mov.u32 %0, %%cluster_nctarank;\n" : "=r"(r));
  return r;
}
__device__ __forceinline__ uint32_t cluster_id_x() {
  uint32_t r;
  asm volatile("mov.u32 %0, %%clusterid.x;\n" : "=r"(r));
  return r;
}
__device__ __forceinline__ uint32_t cluster_count_x() {
  uint32_t r;
  asm volatile("mov.u32 %0, %%nclusterid.x;\n" : "=r"(r));
  return r;
}
// The shared::cluster address of the same shared-memory offset in CTA rank.
__device__ __forceinline__ uint32_t mapa_rank(uint32_t saddr, uint32_t rank) {
  uint32_t r;
  asm volatile("mapa.shared::cluster.u32 %0, %1, %2;\n" : "=r"(r) : "r"(saddr), "r"(rank));
  return r;
}
__device__ __forceinline__ void cluster_sync_all() {
  asm volatile("barrier.cluster.arrive.release.aligned;\n" ::: "memory");
  asm volatile("barrier.cluster.wait.acquire.aligned;\n" ::: "memory");
}
// TMA loads into this CTA's shared memory whose completion is counted on an
// mbarrier of either CTA of the pair (shared::cluster address).
__device__ __forceinline__ void tma_load_2d_pair(uint32_t dst, const CUtensorMap* map, uint32_t bar, int c0, int c1) {
  asm volatile(
      "cp.async.bulk.tensor.2d.cta_group::2.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%3, "
      "%4}], [%2];\n" ::"r"(dst),
      "l"(map), "r"(bar), "r"(c0), "r"(c1)
      : "memory");
}
__device__ __forceinline__ void tma_load_3d_pair(uint32_t dst, const CUtensorMap* map, uint32_t bar, int c0, int c1,
                                                 int c2) {
  asm volatile(
      "cp.async.bulk.tensor.3d.cta_group::2.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%3, "
      "%4, %5}], [%2];\n" ::"r"(dst),
      "l"(map), "r"(bar), "r"(c0), "r"(c1), "r"(c2)
      : "memory");
}
__device__ __forceinline__ void umma_f16_pair(uint32_t tmem_d, uint64_t adesc, uint64_t bdesc, uint32_t idesc,
                                              uint32_t accumulate) {
  asm volatile(
      "{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n tcgen05.mma.cta_group::2.kind::f16 [%0], %1, %2, %3, p;\n}\n" ::"r"(
          tmem_d),
      "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate));
}
// Arrive on the mbarrier at this offset in both CTAs once the MMAs issued so far complete.
__device__ __forceinline__ void umma_commit_pair_both(uint64_t* bar) {
  asm volatile(
      "tcgen05.commit.cta_group::2.mbarrier::arrive::one.shared::cluster.multicast::cluster.b64 [%0], %1;\n" ::"r"(
          smem_u32(bar)),
      "h"((unsigned short)3)
      : "memory");
}
__device__ __forceinline__ void umma_commit_pair_own(uint64_t* bar) {
  asm volatile("tcgen05.commit.cta_group::2.mbarrier::arrive::one.shared::cluster.b64 [%0];\n" ::"r"(smem_u32(bar))
               : "memory");
}
__device__ __forceinline__ void mbar_arrive_rank(uint64_t* bar, uint32_t rank) {
  asm volatile("mbarrier.arrive.release.cluster.shared::cluster.b64 _, [%0];\n" ::"r"(mapa_rank(smem_u32(bar), rank))
               : "memory");
}
// mbar_wait with cluster-scope acquire (arrivals from the other CTA).
__device__ __forceinline__ bool mbar_wait_cluster(uint64_t* bar, uint32_t parity, volatile int* abort_flag, int* err,
                                                  int code) {
  const long long t0 = clock64();
  while (true) {
    uint32_t ok;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.acquire.cluster.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, "
        "0, p;\n}\n"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    if (ok) return true;
    if (*abort_flag) return false;
    if (clock64() - t0 > WAIT_CYCLES) {
      *abort_flag = 1;
      atomicCAS(err, 0, code);
      return false;
    }
  }
}

// ---------------------------------------------------------------------------
// The GEMM kernel.
// ---------------------------------------------------------------------------
// EPI_UPDATE is the STORE epilogue in its subtract form (the sweep's trailing
// update), instantiated apart so that profiles tell it from P0.
// EPI_GUPDATE is the grouped form of the update (one persistent CTA per SM
// over the tiles of many matrices): two groups of four epilogue warps take
// alternate tiles, each with its own TMEM buffer, staging area and named
// barrier, so that one group's drain and barriers overlap the other's
// read-modify-write.
enum { EPI_ROWDOT = 0, EPI_STORE = 1, EPI_UPDATE = 2, EPI_GUPDATE = 3 };

constexpr int TC_BM = 128;
// Pipeline shape per epilogue: 64-wide K blocks, in 2 stages except where
// noted below.  32-wide blocks in 4 stages (the same shared memory, more TMA
// requests in flight) measured slower for the pair contraction (7.8 vs 6.1 ms
// at nmo 300 / naux 1000 / nw 32).  STORE runs 3 stages: with P0's drain made
// cheaper (units drained in pairs), the MMA thread's waits for the loads
// showed, and the third stage took P0 from 1.73 to 1.70 ms per iteration.
template <int EPI>
struct TcPipe {
  static constexpr int BK = 64;
  // The grouped update holds two staging tiles instead of a second stage
  // (its K of 128 is two blocks, loaded and multiplied one after the other).
  // (STORE with the converter's FP32 ring keeps two: TcStages.)
  static constexpr int STAGES = EPI == EPI_GUPDATE ? 1 : EPI == EPI_STORE ? 3 : 2;
  // TMEM accumulators of BN columns (STORE: four, so that P0 can drain its
  // accumulation units in pairs while the MMAs fill the other two).
  static constexpr int NBUF = EPI == EPI_STORE ? 4 : 2;
};
template <int EPI, bool CONVB>
struct TcStages {
  static constexpr int VALUE = CONVB ? 2 : TcPipe<EPI>::STAGES;
};

// STORE (the FP64-output GEMMs: P0, the sweep update, the BSE direct term):
// the accumulator restarts every TcArgs::unit k-blocks and the epilogue sums
// the units in FP64.  The FP32 -> FP64 conversions of one drain cost about as
// much as the MMAs of one 64-wide k-block, so a drain per block left P0
// drain-bound: at nmo 300 / naux 1000 / nw 32, P0 took 2.29 ms per evGW
// iteration with unit 1, 1.93 ms with unit 2 and 1.72 ms with unit 4, at QP
// errors against FP64 of 0.024, 0.036 and 0.068 meV.  Once the chi-scaled
// operand was split in one pass for all frequencies, unit 4 no longer beat
// unit 2 (1.86 vs 1.89 ms) and doubled the error, so P0 uses unit 2; the
// sweep's update uses unit 2 too (one unit covers its K of 128); the BSE
// direct term keeps unit 1, since with unit 2 the Davidson residuals of the
// 26 400-dimensional problem stalled above 1e-8.  P0 (TcArgs::pair_units)
// then drains its units two at a time, adding their FP32 partials in FP32
// before the one conversion (1.73 -> 1.62 ms; the BSE term's Davidson took 177
// instead of 167 iterations with the same pairing, so it drains one unit).
// Largest chi-scaled P0 operand (hi + lo of B_ov chi'_w s_w for every
// frequency) that is materialised; larger problems use the converter form.
constexpr size_t kP0SplitBudget = (size_t)6 << 30;
constexpr int kP0Unit = 128 / TcPipe<EPI_STORE>::BK;
constexpr int kBseUnit = 64 / TcPipe<EPI_STORE>::BK;
constexpr int kUpdateUnit = 2;
// Epilogue warps: 8, two per TMEM lane quarter (ROWDOT: half an N tile each;
// STORE: 64 columns each).  For STORE, 16 warps of 32 columns (FP64 or
// Kahan-compensated FP32 drain) measured no faster for P0 and slower for the
// BSE direct term.
template <int EPI>
struct TcWarps {
  static constexpr int NEPI = 8;
  static constexpr int THREADS = 64 + 32 * NEPI;
};
// Converter warps of the STORE form whose B operand is built in shared memory
// (CONVB): the FP32 source times a per-batch column scale, split into hi/lo
// and written in the 128-byte-swizzled layout that TMA would have written.
constexpr int kConvWarps = 2;
template <int EPI, bool CONVB>
struct TcThreads {
  static constexpr int VALUE = TcWarps<EPI>::THREADS + (CONVB ? 32 * kConvWarps : 0);
};

template <int BN, int EPI, bool CONVB = false>
struct TcSmem {
  static constexpr int A_BYTES = TC_BM * TcPipe<EPI>::BK * 2;
  static constexpr int B_BYTES = BN * TcPipe<EPI>::BK * 2;
  static constexpr int STAGE_BYTES = 2 * A_BYTES + 2 * B_BYTES;
  // CONVB: a ring of F32_STAGES slots for the FP32 B tile as TMA lands it
  // (two 32-column boxes with the 128-byte swizzle), read by the converter
  // warps; it runs F32_STAGES k-blocks ahead of the converters.
  static constexpr int F32_STAGES = 3;
  static constexpr int F32_BYTES = CONVB ? BN * TcPipe<EPI>::BK * 4 : 0;
  static constexpr int F32_OFF = TcStages<EPI, CONVB>::VALUE * STAGE_BYTES;
  static constexpr int BAR_OFF = F32_OFF + (CONVB ? F32_STAGES * F32_BYTES : 0);
  static constexpr int RED_OFF = BAR_OFF + 256;  // ROWDOT: partial row sums [2][128] doubles + 2 flags
  // ROWDOT: two buffers of [2][128] doubles + 2 flags (8 doubles), alternating per item.
  static constexpr int CS_OFF = RED_OFF + (EPI == EPI_ROWDOT ? 2 * (2 * TC_BM + 8) * 8 : 0);
  // UPDATE: the FP32 tile C, staged for the coalesced row passes of the
  // read-modify-write (row stride CS_LD floats against bank conflicts).
  static constexpr int CS_LD = BN + 1;
  static constexpr int CS_BYTES = EPI == EPI_UPDATE ? TC_BM * CS_LD * 4 : EPI == EPI_GUPDATE ? 2 * TC_BM * CS_LD * 4 : 0;
  // UPDATE, grouped: a shared-memory copy of the prefix table of CTA counts
  // (up to GP_CAP matrices), so that finding a tile's matrix costs no
  // dependent global loads.
  static constexpr int GP_CAP = 2048;
  static constexpr int GP_OFF = CS_OFF + CS_BYTES;
  static constexpr int GP_BYTES = (EPI == EPI_UPDATE || EPI == EPI_GUPDATE) ? GP_CAP * 4 : 0;
  static constexpr int TOTAL = GP_OFF + GP_BYTES + 1024;  // + slack for the 1024-byte alignment
};

struct TcArgs {
  int M, N, K;          // rows of A, rows of B (per batch), reduction length
  int nbatch;           // frequencies
  int m_blocks;         // ceil(M / 128)
  int wgroup;           // frequencies grouped per pair block in the CTA order
  // EPI_ROWDOT
  const float* X;       // [M][ldx]
  int ldx;
  double* out;          // ROWDOT: [nbatch][ldo]; STORE: [nbatch][M][ldo]
  int ldo;
  size_t out_stride;
  int lower_tiles;      // STORE: enumerate lower-triangular (m, n) tile pairs and mirror
  int add_identity;     // STORE: add delta_mn
  int fp16;             // operand type: 0 bf16, 1 fp16
  int tri;              // ROWDOT with lower-triangular B: N tile n0 needs K < n0 + BN, result x2
  const float* scaleA;  // [1] (or [nbatch] with a_batched) scale applied to A before the split
  const float* scaleB;  // [nbatch] scale applied to B[w] before the split
  int* err;
  // STORE, trailing update of the block sweep (subtract = 1, with
  // lower_tiles): out = out - C; the tiles whose row or column index is
  // skip_tile are left alone; filter_mode 1 keeps only the tiles whose row or
  // column index is filter_tile, 2 only the others (0: no filter).
  // a_batched: A has a batch index (3D map) and a scale per batch.
  int a_batched;
  int subtract;
  int skip_tile;
  int filter_mode;
  int filter_tile;
  // Grouped trailing update (with subtract): a CTA's matrix is found in the
  // prefix table gpre over gcount matrices gmats; A and B rows are offset by
  // the matrix's panel row, out / M / N / ldo come from the matrix.
  const GMat* gmats;
  const int* gpre;
  int gcount;
  int items;  // tiles of the grouped table (the item count with gmats)
  int unit;  // STORE: k-blocks per FP32 accumulation unit (0 counts as 1)
  int pair_units;  // STORE: drain the accumulation units two at a time (P0)
  // CONVB: B[w][n][k] = convB[n][k] * convC[w][k] (FP32, zero past K): the
  // FP32 tile of convB arrives by TMA (map in the mapBh slot), and the
  // converter warps scale and split it into the hi/lo tile the MMA reads.
  const float* convC;
  int ldcc;
};

// Byte offset of the 16-bit element (row r, column c) in a 64-wide K-major
// tile with the 128-byte swizzle (the layout TMA's SWIZZLE_128B writes into a
// 1024-byte-aligned buffer, umma_desc<64>): rows of 128 bytes, whose 16-byte
// chunks are permuted by chunk ^ (r % 8).
__device__ __forceinline__ uint32_t sw128_offset(int r, int c) {
  return (uint32_t)r * 128u + ((uint32_t)((c >> 3) ^ (r & 7)) << 4) + (uint32_t)(c & 7) * 2u;
}

// x[q] = xr[q] for the columns col0 + q < N of a valid row, 0 otherwise
// (vector loads for a full chunk; indices are compile-time, x stays in registers).
__device__ __forceinline__ void load_x16(const float* xr, int col0, int N, bool row_ok, float (&x)[16]) {
  if (row_ok && col0 + 16 <= N) {
#pragma unroll
    for (int q = 0; q < 16; q += 4) {
      const float4 v = *reinterpret_cast<const float4*>(xr + q);
      x[q] = v.x;
      x[q + 1] = v.y;
      x[q + 2] = v.z;
      x[q + 3] = v.w;
    }
  } else {
#pragma unroll
    for (int q = 0; q < 16; ++q) x[q] = (row_ok && col0 + q < N) ? xr[q] : 0.0f;
  }
}

// sum_q v[q] x[q] over a 16-value chunk: two FP32 FMA chains, one conversion
// to FP64 per chunk.  Converting both factors of every product to FP64 (two
// conversions and an FP64 FMA per value) bounded the ROWDOT epilogue; the
// chunk sums err by ~1e-6 relative, below the FP32 accumulation of the
// accumulator itself over K.
__device__ __forceinline__ double chunk_dot16(const float (&v)[16], const float (&x)[16]) {
  float s0 = 0.0f, s1 = 0.0f;
#pragma unroll
  for (int q = 0; q < 16; q += 2) {
    s0 = fmaf(v[q], x[q], s0);
    s1 = fmaf(v[q + 1], x[q + 1], s1);
  }
  return (double)s0 + (double)s1;
}

__device__ __forceinline__ double unscale_rowdot(const TcArgs& a, int w) {
  return 1.0 / ((double)a.scaleA[0] * (double)a.scaleB[w]);
}

// A STORE / UPDATE output tile: 128-row block mb and BN-column tile nt of
// the matrix out (leading dimension ld, outM x outN; out already points at
// frequency w), whose operand rows start at row_off (grouped panels).
struct StoreTile {
  int mb, nt, w, row_off, outM, outN, ld;
  double* out;
};

template <int BN, int EPI, bool CONVB = false>
__global__ void __launch_bounds__(TcThreads<EPI, CONVB>::VALUE, 1)
    k_tc_gemm(const __grid_constant__ CUtensorMap mapAh, const __grid_constant__ CUtensorMap mapAl,
              const __grid_constant__ CUtensorMap mapBh, const __grid_constant__ CUtensorMap mapBl, TcArgs args) {
  static_assert(!CONVB || (EPI == EPI_STORE && BN == 128), "the converted B operand serves P0's STORE tiles");
  using L = TcSmem<BN, EPI, CONVB>;
  constexpr int TC_BK = TcPipe<EPI>::BK;
  constexpr int TC_STAGES = TcStages<EPI, CONVB>::VALUE;
  extern __shared__ __align__(1024) uint8_t smem_raw[];
  uint8_t* smem = reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
  uint64_t* full = reinterpret_cast<uint64_t*>(smem + L::BAR_OFF);
  uint64_t* empty = full + TC_STAGES;
  constexpr int NBUF = TcPipe<EPI>::NBUF;
  uint64_t* acc_full = empty + TC_STAGES;   // [NBUF]
  uint64_t* acc_empty = acc_full + NBUF;    // [NBUF]
  uint64_t* drain = acc_empty + NBUF;       // all issued MMAs complete
  uint64_t* conv = drain + 1;               // CONVB: [TC_STAGES] converted B tile ready
  uint64_t* f32_full = conv + TC_STAGES;    // CONVB: [F32_STAGES] FP32 tile landed
  uint64_t* f32_empty = f32_full + L::F32_STAGES;  // CONVB: [F32_STAGES] FP32 slot read by every converter warp
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(f32_empty + L::F32_STAGES);
  volatile int* abort_flag = reinterpret_cast<volatile int*>(tmem_slot + 1);

  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;

  const int n_tiles = (args.N + BN - 1) / BN;
  const int k_blocks = (args.K + TC_BK - 1) / TC_BK;
  // Items.  ROWDOT: (pair block, frequency), ordered so that the frequencies
  // of a group of wgroup share each pair block while it is in L2.  STORE and
  // UPDATE: (frequency, output tile), or a tile of the grouped table.  CTA b
  // of a grid of G CTAs takes the items b, b + G, ...: a persistent grid (one
  // CTA per SM) runs many, a grid of one CTA per item runs one.  TMEM
  // buffers, stages and barrier phases run on across items, so the epilogue
  // of one item overlaps the loads and MMAs of the next.
  const int tiles_pb = args.lower_tiles ? args.m_blocks * (args.m_blocks + 1) / 2 : args.m_blocks * n_tiles;
  const int n_items = (EPI == EPI_ROWDOT)
                          ? (args.nbatch + args.wgroup - 1) / args.wgroup * args.m_blocks * args.wgroup
                          : (args.gmats ? args.items : tiles_pb * args.nbatch);
  const int item0 = (int)(blockIdx.x + blockIdx.y * gridDim.x);
  const int item_step = (int)(gridDim.x * gridDim.y);
  auto rowdot_item = [&](int b, int& mb_, int& w_) {
    const int g = args.wgroup;
    const int per_group = args.m_blocks * g;
    const int grp = b / per_group, r = b % per_group;
    mb_ = r / g;
    w_ = grp * g + r % g;
  };
  // STORE / UPDATE item -> output tile; false when the tile is left alone
  // (the sweep update's pivot row and column, and the look-ahead filter).
  const bool gp_shared = (EPI == EPI_UPDATE || EPI == EPI_GUPDATE) && args.gmats && args.gcount <= L::GP_CAP;
  const int* gpre = args.gpre;
  if (gp_shared) {
    int* gs = reinterpret_cast<int*>(smem + L::GP_OFF);
    for (int i = threadIdx.x; i < args.gcount; i += blockDim.x) gs[i] = __ldg(args.gpre + i);
    gpre = gs;
    __syncthreads();
  }
  auto tile_item = [&](int it, StoreTile& t) -> bool {
    int r = it, tm, tn;
    t.w = 0;
    if (args.gmats) {
      int lo = 0, hi = args.gcount - 1;
      while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (gpre[mid] <= it)
          lo = mid;
        else
          hi = mid - 1;
      }
      const GMat gm = args.gmats[lo];
      r = it - gpre[lo];
      t.row_off = gm.prow;
      t.outM = t.outN = gm.n;
      t.ld = gm.ldn;
      t.out = gm.M;
    } else {
      t.w = it / tiles_pb;
      r = it - t.w * tiles_pb;
      t.row_off = 0;
      t.outM = args.M;
      t.outN = args.N;
      t.ld = args.ldo;
      t.out = args.out + (size_t)t.w * args.out_stride;
    }
    if (args.gmats || args.lower_tiles) {
      // Single precision is exact for 8 r + 1 < 2^24; the loops below fix
      // any off-by-one of the rounded root.
      tm = (int)((sqrtf(8.0f * (float)r + 1.0f) - 1.0f) * 0.5f);
      while ((tm + 1) * (tm + 2) / 2 <= r) ++tm;
      while (tm * (tm + 1) / 2 > r) --tm;
      tn = r - tm * (tm + 1) / 2;
    } else {
      tm = r / n_tiles;
      tn = r - tm * n_tiles;
    }
    t.mb = tm;
    t.nt = tn;
    if (args.subtract) {
      if (tm == args.skip_tile || tn == args.skip_tile) return false;
      if (args.filter_mode) {
        const bool touches = (tm == args.filter_tile || tn == args.filter_tile);
        if (touches != (args.filter_mode == 1)) return false;
      }
    }
    return true;
  };
  // The first item of this CTA with work (CONVB runs exactly one item per
  // CTA and takes its frequency and tile from it); a CTA without any exits
  // before any barrier or TMEM allocation.
  StoreTile t0{};
  if (EPI != EPI_ROWDOT) {
    int it = item0;
    while (it < n_items && !tile_item(it, t0)) it += item_step;
    if (it >= n_items) return;
  }

  if (threadIdx.x == 0) {
    for (int s = 0; s < TC_STAGES; ++s) {
      mbar_init(&full[s], 1);
      mbar_init(&empty[s], 1);
      // CONVB: one arrival per converter warp once the hi/lo B tile is written.
      if (CONVB) mbar_init(&conv[s], kConvWarps);
    }
    for (int s = 0; s < (CONVB ? L::F32_STAGES : 0); ++s) {
      mbar_init(&f32_full[s], 1);
      mbar_init(&f32_empty[s], kConvWarps);
    }
    for (int b = 0; b < NBUF; ++b) {
      mbar_init(&acc_full[b], 1);
      // One arrival per epilogue warp (GUPDATE: per warp of the group that
      // owns the buffer).
      mbar_init(&acc_empty[b], EPI == EPI_GUPDATE ? TcWarps<EPI>::NEPI / 2 : TcWarps<EPI>::NEPI);
    }
    mbar_init(drain, 1);
    *abort_flag = 0;
    asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
  }
  if (warp == 1) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;\n" ::"r"(smem_u32(tmem_slot)),
                 "r"(NBUF * BN));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;\n" ::);
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem_base = *tmem_slot;

  {
    if (warp == 0) {
      // ---------------- TMA producer ----------------
      if (lane == 0) {
        int g = 0;
        int issued = 0;
        for (int it = item0; it < n_items; it += item_step) {
        int mi, wi, ntb, nte, row_off = 0;
        if (EPI == EPI_ROWDOT) {
          rowdot_item(it, mi, wi);
          if (wi >= args.nbatch) continue;
          ntb = 0;
          nte = n_tiles;
        } else {
          StoreTile ti;
          if (!tile_item(it, ti)) continue;
          mi = ti.mb;
          wi = ti.w;
          ntb = ti.nt;
          nte = ti.nt + 1;
          row_off = ti.row_off;
        }
        const int mi0 = mi * TC_BM;
        for (int nt = ntb; nt < nte; ++nt) {
          const int n0 = nt * BN;
          const int kbe = args.tri ? min(k_blocks, (n0 + BN + TC_BK - 1) / TC_BK) : k_blocks;
          for (int kb = 0; kb < kbe; ++kb, ++g) {
            const int s = g % TC_STAGES;
            if (g >= TC_STAGES) {
              if (!mbar_wait(&empty[s], ((g / TC_STAGES) - 1) & 1, abort_flag, args.err, 1)) goto producer_done;
            }
            uint8_t* st = smem + s * L::STAGE_BYTES;
            mbar_expect_tx(&full[s], CONVB ? 2 * L::A_BYTES : L::STAGE_BYTES);
            const int k0 = kb * TC_BK;
            if (args.a_batched) {
              tma_load_3d(st, &mapAh, &full[s], k0, mi0, wi);
              tma_load_3d(st + L::A_BYTES, &mapAl, &full[s], k0, mi0, wi);
            } else {
              tma_load_2d(st, &mapAh, &full[s], k0, row_off + mi0);
              tma_load_2d(st + L::A_BYTES, &mapAl, &full[s], k0, row_off + mi0);
            }
            if (!CONVB) {
              tma_load_3d(st + 2 * L::A_BYTES, &mapBh, &full[s], k0, row_off + n0, wi);
              tma_load_3d(st + 2 * L::A_BYTES + L::B_BYTES, &mapBl, &full[s], k0, row_off + n0, wi);
            }
            issued = g + 1;
          }
        }
        }
      producer_done:
        if (*abort_flag) {
          // Let the copies still in flight land before the CTA exits.
          for (int q = (issued > TC_STAGES ? issued - TC_STAGES : 0); q < issued; ++q) {
            volatile int no_abort = 0;
            mbar_wait(&full[q % TC_STAGES], (q / TC_STAGES) & 1, &no_abort, args.err, 5);
          }
        }
      }
    } else if (warp == 1) {
      // ---------------- MMA issuer ----------------
      // Accumulation units: ROWDOT accumulates a whole N tile in one TMEM
      // buffer; STORE restarts the accumulator every UNIT k-blocks and the
      // epilogue sums the units in FP64, because the FP32 accumulation of the
      // tensor pipe carries a small same-signed error per step that grows
      // linearly over long positive sums (the diagonal of Pi over K = nov).
      if (lane == 0) {
        const uint32_t idesc = umma_idesc_f16(TC_BM, BN, args.fp16);
        int g = 0, u = 0;
        bool ok = true;
        for (int it = item0; it < n_items && ok; it += item_step) {
        int ntb, nte;
        if (EPI == EPI_ROWDOT) {
          int mi, wi;
          rowdot_item(it, mi, wi);
          if (wi >= args.nbatch) continue;
          ntb = 0;
          nte = n_tiles;
        } else {
          StoreTile ti;
          if (!tile_item(it, ti)) continue;
          ntb = ti.nt;
          nte = ti.nt + 1;
        }
        for (int nt = ntb; nt < nte && ok; ++nt) {
          const int kbe = args.tri ? min(k_blocks, (nt * BN + BN + TC_BK - 1) / TC_BK) : k_blocks;
          for (int kb = 0; kb < kbe; ++kb, ++g) {
            const int unit = args.unit > 0 ? args.unit : 1;
            const bool unit_start = (EPI != EPI_ROWDOT) ? (kb % unit == 0) : kb == 0;
            const bool unit_end = (EPI != EPI_ROWDOT) ? (kb % unit == unit - 1 || kb == kbe - 1) : kb == kbe - 1;
            const int buf = u % NBUF;
            if (unit_start && u >= NBUF) {
              if (!mbar_wait(&acc_empty[buf], ((u / NBUF) - 1) & 1, abort_flag, args.err, 2)) {
                ok = false;
                break;
              }
            }
            const int s = g % TC_STAGES;
            if (!mbar_wait(&full[s], (g / TC_STAGES) & 1, abort_flag, args.err, 3) ||
                (CONVB && !mbar_wait(&conv[s], (g / TC_STAGES) & 1, abort_flag, args.err, 8))) {
              ok = false;
              break;
            }
            tc_fence_after();
            const uint32_t dacc = tmem_base + buf * BN;
            uint8_t* st = smem + s * L::STAGE_BYTES;
            const uint32_t ah = smem_u32(st), al = ah + L::A_BYTES;
            const uint32_t bh = ah + 2 * L::A_BYTES, bl = bh + L::B_BYTES;
#pragma unroll
            for (int kk = 0; kk < TC_BK / 16; ++kk) {
              const uint32_t off = kk * 32;
              const uint32_t acc0 = (!unit_start || kk > 0) ? 1u : 0u;
              umma_f16(dacc, umma_desc<TC_BK>(ah + off), umma_desc<TC_BK>(bh + off), idesc, acc0);
              umma_f16(dacc, umma_desc<TC_BK>(ah + off), umma_desc<TC_BK>(bl + off), idesc, 1u);
              umma_f16(dacc, umma_desc<TC_BK>(al + off), umma_desc<TC_BK>(bh + off), idesc, 1u);
            }
            umma_commit(&empty[s]);
            if (unit_end) {
              umma_commit(&acc_full[buf]);
              ++u;
            }
          }
        }
        }
        // Wait until every MMA this thread issued has completed (TMEM and the
        // stages are released only after that).
        umma_commit(drain);
        volatile int no_abort = 0;
        mbar_wait(drain, 0, &no_abort, args.err, 6);
      }
    } else if (CONVB && warp >= 2 + TcWarps<EPI>::NEPI) {
      // ---------------- B operand converters (CONVB) ----------------
      // Thread t owns the 8-column chunk cc = t % 8 of rows t / 8 + 8 i of
      // the 128-row tile.  Per k block it reads the FP32 tile that TMA
      // landed (two 32-column boxes, 128-byte swizzle: the chunk of 4 floats
      // q of row r sits at r * 128 + ((q ^ r % 8) << 4)), forms x = b * c in
      // FP32, hi = rn16(x), lo = rn16(x - hi) (split_round's rounding) and
      // stores both 16-byte chunks into the swizzled hi/lo tile.  A warp's
      // stores cover four whole rows and its loads two 128-byte row halves
      // per box, so neither has bank conflicts beyond the 4 wavefronts of a
      // 512-byte access.  The generic-proxy stores are made visible to the
      // tensor core's async proxy before the warp arrives on conv[s].
      const int ct = threadIdx.x - 32 * (2 + TcWarps<EPI>::NEPI);
      const int cc = ct & 7, rg = ct >> 3;
      constexpr int ROWS_PER_PASS = 4 * kConvWarps;  // row groups of 8 chunk threads
      const float* cw_scale = args.convC + (size_t)t0.w * args.ldcc + 8 * cc;
      // Column scales of the next k block, loaded one block ahead.
      float4 cn0 = make_float4(0.f, 0.f, 0.f, 0.f), cn1 = cn0;
      if (8 * cc < args.K) {
        cn0 = __ldg(reinterpret_cast<const float4*>(cw_scale));
        cn1 = __ldg(reinterpret_cast<const float4*>(cw_scale + 4));
      }
      const int h = cc >> 2, q0 = 2 * (cc & 3);
      const int n0 = t0.nt * BN;
      constexpr int FS = L::F32_STAGES;
      // Converter thread 0 keeps the FP32 ring FS blocks ahead.
      auto issue_f32 = [&](int kb) {
        const int f = kb % FS;
        uint8_t* dst = smem + L::F32_OFF + f * L::F32_BYTES;
        mbar_expect_tx(&f32_full[f], L::F32_BYTES);
        tma_load_2d(dst, &mapBh, &f32_full[f], kb * TC_BK, n0);
        tma_load_2d(dst + L::F32_BYTES / 2, &mapBh, &f32_full[f], kb * TC_BK + TC_BK / 2, n0);
      };
      // issued: FP32 blocks requested so far (kept identically by the lanes
      // of converter warp 0; lane 0 issues).  Every exit from the loop below
      // is warp-uniform.
      const bool feeder = ct < 32;
      int issued = 0;
      for (; issued < FS && issued < k_blocks; ++issued)
        if (ct == 0) issue_f32(issued);
      int kb = 0;
      for (; kb < k_blocks; ++kb) {
        const float4 c0 = cn0, c1 = cn1;
        const int kn = (kb + 1) * TC_BK + 8 * cc;
        if (kb + 1 < k_blocks && kn < args.K) {
          cn0 = __ldg(reinterpret_cast<const float4*>(cw_scale + (size_t)(kb + 1) * TC_BK));
          cn1 = __ldg(reinterpret_cast<const float4*>(cw_scale + (size_t)(kb + 1) * TC_BK + 4));
        } else {
          cn0 = cn1 = make_float4(0.f, 0.f, 0.f, 0.f);
        }
        const int s = kb % TC_STAGES, f = kb % FS;
        // The hi/lo stage must be released by the MMAs of its previous use,
        // and the FP32 tile of this block must have landed.
        bool ok = kb < TC_STAGES || mbar_wait(&empty[s], ((kb / TC_STAGES) - 1) & 1, abort_flag, args.err, 7);
        ok = ok && mbar_wait(&f32_full[f], (kb / FS) & 1, abort_flag, args.err, 9);
        if (__any_sync(0xffffffffu, !ok)) break;
        uint8_t* st = smem + s * L::STAGE_BYTES;
        const uint32_t bh = smem_u32(st + 2 * L::A_BYTES), bl = bh + L::B_BYTES;
        const uint32_t f32 = smem_u32(smem + L::F32_OFF + f * L::F32_BYTES) + h * (L::F32_BYTES / 2);
#pragma unroll 4
        for (int i = 0; i < BN / ROWS_PER_PASS; ++i) {
          const int r = rg + ROWS_PER_PASS * i;
          const uint32_t rb = f32 + r * 128;
          // The eight threads of a 128-byte load phase (one row, cc = 0..7)
          // must hit eight different 16-byte bank groups: the two box halves
          // map to the same banks, so threads cc >= 4 load their second chunk
          // first.
          float4 u0, u1;
          const int qa = q0 + h, qb = q0 + 1 - h;
          asm volatile("ld.shared.v4.f32 {%0, %1, %2, %3}, [%4];\n"
                       : "=f"(u0.x), "=f"(u0.y), "=f"(u0.z), "=f"(u0.w)
                       : "r"(rb + ((qa ^ (r & 7)) << 4)));
          asm volatile("ld.shared.v4.f32 {%0, %1, %2, %3}, [%4];\n"
                       : "=f"(u1.x), "=f"(u1.y), "=f"(u1.z), "=f"(u1.w)
                       : "r"(rb + ((qb ^ (r & 7)) << 4)));
          const float4 v0 = h ? u1 : u0, v1 = h ? u0 : u1;
          const float x[8] = {v0.x * c0.x, v0.y * c0.y, v0.z * c0.z, v0.w * c0.w,
                              v1.x * c1.x, v1.y * c1.y, v1.z * c1.z, v1.w * c1.w};
          uint32_t hw[4], lw[4];
#pragma unroll
          for (int p = 0; p < 4; ++p) {
            if (args.fp16) {
              const __half2 hh = __floats2half2_rn(x[2 * p], x[2 * p + 1]);
              const float2 hf = __half22float2(hh);
              const __half2 ll = __floats2half2_rn(x[2 * p] - hf.x, x[2 * p + 1] - hf.y);
              hw[p] = *reinterpret_cast<const uint32_t*>(&hh);
              lw[p] = *reinterpret_cast<const uint32_t*>(&ll);
            } else {
              const __nv_bfloat162 hh = __floats2bfloat162_rn(x[2 * p], x[2 * p + 1]);
              const float2 hf = __bfloat1622float2(hh);
              const __nv_bfloat162 ll = __floats2bfloat162_rn(x[2 * p] - hf.x, x[2 * p + 1] - hf.y);
              hw[p] = *reinterpret_cast<const uint32_t*>(&hh);
              lw[p] = *reinterpret_cast<const uint32_t*>(&ll);
            }
          }
          const uint32_t off = sw128_offset(r, 8 * cc);
          asm volatile("st.shared.v4.b32 [%0], {%1, %2, %3, %4};\n" ::"r"(bh + off), "r"(hw[0]), "r"(hw[1]),
                       "r"(hw[2]), "r"(hw[3])
                       : "memory");
          asm volatile("st.shared.v4.b32 [%0], {%1, %2, %3, %4};\n" ::"r"(bl + off), "r"(lw[0]), "r"(lw[1]),
                       "r"(lw[2]), "r"(lw[3])
                       : "memory");
        }
        asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
        __syncwarp();
        if (lane == 0) {
          mbar_arrive(&conv[s]);
          mbar_arrive(&f32_empty[f]);
        }
        // Refill slot f once every converter warp has read it.
        if (feeder && issued < k_blocks) {
          bool rok = true;
          if (ct == 0) {
            rok = mbar_wait(&f32_empty[f], (kb / FS) & 1, abort_flag, args.err, 11);
            if (rok) issue_f32(issued);
          }
          if (__any_sync(0xffffffffu, !rok)) break;
          ++issued;
        }
      }
      if (kb < k_blocks && ct == 0) {
        // Aborted: let the FP32 copies still in flight land before the CTA exits.
        for (int q = kb; q < issued; ++q) {
          volatile int no_abort = 0;
          mbar_wait(&f32_full[q % FS], (q / FS) & 1, &no_abort, args.err, 10);
        }
      }
    } else if (EPI == EPI_ROWDOT) {
      // ---------------- epilogue (warps 2..9): row dot products ----------------
      // Two warps per TMEM lane quarter, each over half of the N tile.
      const int quarter = warp & 3;  // TMEM lane quarter this warp may access
      const int half = (warp - 2) >> 2;
      const int row = quarter * 32 + lane;
      constexpr int HB = BN / 2;
      int t = 0, done_items = 0;
      bool ok = true;
      for (int it = item0; it < n_items && ok; it += item_step) {
        int mi, wi;
        rowdot_item(it, mi, wi);
        if (wi >= args.nbatch) continue;
        const int m = mi * TC_BM + row;
        double rowsum = 0.0;
        int tiles_done = 0;
        for (int nt = 0; nt < n_tiles; ++nt, ++t) {
          const int buf = t % NBUF;
          if (!mbar_wait(&acc_full[buf], (t / NBUF) & 1, abort_flag, args.err, 4)) {
            ok = false;
            break;
          }
          tc_fence_after();
          const int n0 = nt * BN + half * HB;
          const uint32_t taddr = tmem_base + ((uint32_t)(quarter * 32) << 16) + buf * BN + half * HB;
          // The pair-row values of the next 16 columns are loaded before the
          // TMEM load of the current ones, so the two latencies overlap.
          const float* xrow = args.X + (size_t)(m < args.M ? m : 0) * args.ldx + n0;
          float xn[16];
          load_x16(xrow, n0, args.N, m < args.M, xn);
#pragma unroll 1
          for (int c = 0; c < HB; c += 16) {
            float xc[16];
#pragma unroll
            for (int q = 0; q < 16; ++q) xc[q] = xn[q];
            if (c + 16 < HB) load_x16(xrow + c + 16, n0 + c + 16, args.N, m < args.M, xn);
            float v[16];
            tmem_ld16(taddr + c, v);
            rowsum += chunk_dot16(v, xc);
          }
          tc_fence_before();
          __syncwarp();
          if (lane == 0) mbar_arrive(&acc_empty[buf]);
          ++tiles_done;
        }
        // Combine the two halves (named barrier of the 8 epilogue warps; every
        // one of them reaches it, also after an abort).  The buffer alternates
        // between items: item i + 2 rewrites it only after the barrier of item
        // i + 1, which every reader of item i has passed.
        double* red = reinterpret_cast<double*>(smem + L::RED_OFF) + (done_items & 1) * (2 * TC_BM + 8);
        int* done = reinterpret_cast<int*>(red + 2 * TC_BM);  // two flags after the sums
        const bool full_item = tiles_done == n_tiles;
        red[half * TC_BM + row] = full_item ? rowsum : 0.0;
        if (lane == 0 && quarter == 0) done[half] = full_item ? 1 : 0;
        asm volatile("bar.sync 1, 256;\n" ::: "memory");
        if (half == 0 && m < args.M && done[0] && done[1])
          args.out[(size_t)wi * args.ldo + m] =
              (red[row] + red[TC_BM + row]) * unscale_rowdot(args, wi) * (args.tri ? 2.0 : 1.0);
        ++done_items;
        // Both halves leave the item loop together (the flags are shared).
        ok = done[0] && done[1];
      }
    } else if (EPI == EPI_GUPDATE) {
      // ---------------- epilogue (warps 2..9): grouped update, two groups ----------------
      // Group gi (warps 2..5 or 6..9, one per TMEM lane quarter) takes the
      // CTA's runnable tiles j = gi, gi + 2, ...; tile j is accumulation unit
      // j (one unit covers K), so it sits in TMEM buffer gi, and the group
      // stages it in its own FP32 area, passes its own named barrier and
      // updates the lower tile and its mirror, 32 rows of each per warp in
      // pipelined batches of RB = 4.
      const int quarter = warp & 3;
      const int gi = (warp - 2) >> 2;
      const int e = (warp - 2) & 3;  // this warp's rank in its group
      constexpr int CLD = L::CS_LD;
      float* Cs = reinterpret_cast<float*>(smem + L::CS_OFF) + gi * (TC_BM * CLD);
      const int rl = quarter * 32 + lane;
      const uint32_t bar_id = 1 + gi;
      bool ok = true;
      int unscale_w = -1;
      double unscale = 1.0;
      int j = 0;  // runnable tiles of this CTA seen so far
      for (int it = item0; it < n_items; it += item_step) {
        StoreTile ti;
        if (!tile_item(it, ti)) continue;
        const int jj = j++;
        if ((jj & 1) != gi) continue;
        const int buf = gi;
        if (ti.w != unscale_w) {
          unscale = 1.0 / ((double)args.scaleA[args.a_batched ? ti.w : 0] * (double)args.scaleB[ti.w]);
          unscale_w = ti.w;
        }
        const bool got = ok && mbar_wait(&acc_full[buf], (jj >> 1) & 1, abort_flag, args.err, 4);
        ok = got;
        if (got) {
          tc_fence_after();
          const uint32_t taddr = tmem_base + ((uint32_t)(quarter * 32) << 16) + buf * BN;
#pragma unroll
          for (int c = 0; c < BN; c += 16) {
            float v[16];
            tmem_ld16(taddr + c, v);
            float* cr = Cs + rl * CLD + c;
#pragma unroll
            for (int q = 0; q < 16; ++q) cr[q] = v[q];
          }
          tc_fence_before();
          __syncwarp();
          if (lane == 0) mbar_arrive(&acc_empty[buf]);
        }
        asm volatile("bar.sync %0, 128;\n" ::"r"(bar_id) : "memory");
        if (ok && !*abort_flag) {
          constexpr int RB = 4, NBT = 16;  // 8 batches of the lower tile, 8 of the mirror
          const int m0 = ti.mb * TC_BM, nb = ti.nt * BN;
          const int outM = ti.outM, outN = ti.outN, out_ld = ti.ld;
          double* outw = ti.out;
          static_assert(EPI != EPI_GUPDATE || (TC_BM == 128 && BN == 128), "row passes assume 128 x 128 tiles");
          auto elem = [&](int b, int k, int q, bool& v) -> double* {
            if (b < NBT / 2) {
              const int mm = m0 + e + 16 * b + 4 * k, n = nb + lane + 32 * q;
              v = mm < outM && n < outN && n <= mm;
              return outw + (size_t)mm * out_ld + n;
            }
            const int n = nb + e + 16 * (b - NBT / 2) + 4 * k, mm = m0 + lane + 32 * q;
            v = mm < outM && n < outN && n < mm;
            return outw + (size_t)n * out_ld + mm;
          };
          auto cval = [&](int b, int k, int q) -> double {
            return (double)(b < NBT / 2 ? Cs[(e + 16 * b + 4 * k) * CLD + lane + 32 * q]
                                        : Cs[(lane + 32 * q) * CLD + e + 16 * (b - NBT / 2) + 4 * k]);
          };
          double x[RB][4], y[RB][4];
#pragma unroll
          for (int k = 0; k < RB; ++k)
#pragma unroll
            for (int q = 0; q < 4; ++q) {
              bool v;
              const double* ptr = elem(0, k, q, v);
              x[k][q] = v ? *ptr : 0.0;
            }
#pragma unroll 2
          for (int b = 0; b < NBT; ++b) {
            if (b + 1 < NBT) {
#pragma unroll
              for (int k = 0; k < RB; ++k)
#pragma unroll
                for (int q = 0; q < 4; ++q) {
                  bool v;
                  const double* ptr = elem(b + 1, k, q, v);
                  y[k][q] = v ? *ptr : 0.0;
                }
            }
#pragma unroll
            for (int k = 0; k < RB; ++k)
#pragma unroll
              for (int q = 0; q < 4; ++q) {
                bool v;
                double* ptr = elem(b, k, q, v);
                if (v) *ptr = x[k][q] - cval(b, k, q) * unscale;
              }
#pragma unroll
            for (int k = 0; k < RB; ++k)
#pragma unroll
              for (int q = 0; q < 4; ++q) x[k][q] = y[k][q];
          }
        }
        // The group's next tile rewrites its staging area only after every
        // warp of the group has read this one.
        asm volatile("bar.sync %0, 128;\n" ::"r"(bar_id) : "memory");
      }
    } else {
      // ---------------- epilogue (warps 2..9): FP64 sum of k-block partials ----------------
      constexpr int CPW = BN * 4 / TcWarps<EPI>::NEPI;  // columns per epilogue warp
      const int quarter = warp & 3;
      const int part = (warp - 2) >> 2;  // columns [CPW part, CPW part + CPW) of the tile
      const int unit = args.unit > 0 ? args.unit : 1;
      const int n_units = (k_blocks + unit - 1) / unit;
      // After a failed wait a warp waits no more but still passes the named
      // barriers of every later item, as the other epilogue warps do.
      bool ok = true;
      int u = 0;
      int it = item0;
      int unscale_w = -1;
      double unscale = 1.0;
      StoreTile ti;
      while (it < n_items && !tile_item(it, ti)) it += item_step;
      while (it < n_items) {
        // UPDATE: the next item of this CTA is decoded now, so that its table
        // loads are in flight during this item's work (STORE, with its FP64
        // accumulators live, decodes it after the item).
        int nit = it + item_step;
        StoreTile tnext;
        if (EPI == EPI_UPDATE)
          while (nit < n_items && !tile_item(nit, tnext)) nit += item_step;
        const int m0 = ti.mb * TC_BM;
        const int m = m0 + quarter * 32 + lane;
        // The scales change with the frequency only (once per launch in the
        // grouped update).
        if (ti.w != unscale_w) {
          unscale = 1.0 / ((double)args.scaleA[args.a_batched ? ti.w : 0] * (double)args.scaleB[ti.w]);
          unscale_w = ti.w;
        }
        constexpr int CLD = L::CS_LD;
        float* Cs = reinterpret_cast<float*>(smem + L::CS_OFF);
        const int rl = quarter * 32 + lane;
        double acc[CPW];
#pragma unroll
        for (int c = 0; c < CPW; ++c) acc[c] = 0.0;
        for (int uu = 0; uu < n_units;) {
          // P0 (pair_units) drains two accumulation units at once: their FP32
          // partials are added in FP32 (one rounding to nearest) before the
          // conversion to FP64, so the drain converts half as many values.
          const int nu = (EPI == EPI_STORE && args.pair_units && uu + 1 < n_units) ? 2 : 1;
          const int buf = u % NBUF, buf2 = (u + 1) % NBUF;
          const bool got = ok && mbar_wait(&acc_full[buf], (u / NBUF) & 1, abort_flag, args.err, 4) &&
                           (nu == 1 || mbar_wait(&acc_full[buf2], ((u + 1) / NBUF) & 1, abort_flag, args.err, 4));
          if (!got) {
            ok = false;
            uu += nu;
            u += nu;
            continue;
          }
          tc_fence_after();
          const uint32_t lrow = (uint32_t)(quarter * 32) << 16;
          const uint32_t taddr = tmem_base + lrow + buf * BN + CPW * part;
          const uint32_t taddr2 = tmem_base + lrow + buf2 * BN + CPW * part;
#pragma unroll
          for (int j = 0; j < CPW / 16; ++j) {
            // Columns past N (a narrow GEMM, e.g. a few vectors) are not
            // drained; the condition is warp-uniform.
            if (ti.nt * BN + CPW * part + 16 * j >= ti.outN) continue;
            float v[16];
            tmem_ld16(taddr + 16 * j, v);
            if (EPI == EPI_UPDATE) {
              // UPDATE stages the FP32 tile as it is drained (one
              // accumulation unit covers K; further units would add).
              float* cr = Cs + rl * CLD + CPW * part + 16 * j;
#pragma unroll
              for (int q = 0; q < 16; ++q) cr[q] = uu == 0 ? v[q] : cr[q] + v[q];
            } else {
              if (nu == 2) {
                float v2[16];
                tmem_ld16(taddr2 + 16 * j, v2);
#pragma unroll
                for (int q = 0; q < 16; ++q) v[q] += v2[q];
              }
#pragma unroll
              for (int q = 0; q < 16; ++q) acc[16 * j + q] += (double)v[q];
            }
          }
          tc_fence_before();
          __syncwarp();
          if (lane == 0) {
            mbar_arrive(&acc_empty[buf]);
            if (nu == 2) mbar_arrive(&acc_empty[buf2]);
          }
          uu += nu;
          u += nu;
        }
        if (EPI == EPI_UPDATE) {
          // The tile C (exactly FP32: one accumulation unit covers K, the
          // launchers ask for it) was staged in its own shared-memory area
          // while drained (the stages already hold the next item's operands);
          // the lower tile and its mirror are now updated in row-wise passes
          // that are coalesced along the rows of M; the mirror reads its old
          // value from the upper element itself, M being stored exactly
          // symmetric.  After an abort nothing more is written.
          asm volatile("bar.sync 1, 256;\n" ::: "memory");
          if (ok && !*abort_flag) {
            // Warp e updates eight batches of RB = 4 rows: rows e + 32 b + 8 k
            // of the lower tile (b < 4), then rows nb + e + 32 (b - 4) + 8 k of
            // the mirror in the upper tile (b >= 4), each row 128 coalesced
            // doubles.  The loads of batch b + 1 are issued before the stores
            // of batch b: with all warps passing the tile's barriers together,
            // loads followed by stores in lockstep kept only half of HBM busy
            // (3.4 against 6.1 TB/s pipelined, measured on this access pattern
            // alone; two batches of 4 rows fit the 168 registers of the
            // 320-thread CTA).  The lower and mirror elements are disjoint, so
            // no store of a batch aliases a later load.
            constexpr int RB = 4, NBT = 8;
            const int e = warp - 2;
            const int nb = ti.nt * BN;
            const int outM = ti.outM, outN = ti.outN, out_ld = ti.ld;
            double* outw = ti.out;
            static_assert(EPI != EPI_UPDATE || (TC_BM == 128 && BN == 128), "row passes assume 128 x 128 tiles");
            auto elem = [&](int b, int k, int q, bool& v) -> double* {
              if (b < NBT / 2) {
                const int mm = m0 + e + 32 * b + 8 * k, n = nb + lane + 32 * q;
                v = mm < outM && n < outN && n <= mm;
                return outw + (size_t)mm * out_ld + n;
              }
              const int n = nb + e + 32 * (b - NBT / 2) + 8 * k, mm = m0 + lane + 32 * q;
              v = mm < outM && n < outN && n < mm;
              return outw + (size_t)n * out_ld + mm;
            };
            auto cval = [&](int b, int k, int q) -> double {
              return (double)(b < NBT / 2 ? Cs[(e + 32 * b + 8 * k) * CLD + lane + 32 * q]
                                          : Cs[(lane + 32 * q) * CLD + e + 32 * (b - NBT / 2) + 8 * k]);
            };
            double x[RB][4], y[RB][4];
#pragma unroll
            for (int k = 0; k < RB; ++k)
#pragma unroll
              for (int q = 0; q < 4; ++q) {
                bool v;
                const double* ptr = elem(0, k, q, v);
                x[k][q] = v ? *ptr : 0.0;
              }
#pragma unroll
            for (int b = 0; b < NBT; ++b) {
              if (b + 1 < NBT) {
#pragma unroll
                for (int k = 0; k < RB; ++k)
#pragma unroll
                  for (int q = 0; q < 4; ++q) {
                    bool v;
                    const double* ptr = elem(b + 1, k, q, v);
                    y[k][q] = v ? *ptr : 0.0;
                  }
              }
#pragma unroll
              for (int k = 0; k < RB; ++k)
#pragma unroll
                for (int q = 0; q < 4; ++q) {
                  bool v;
                  double* ptr = elem(b, k, q, v);
                  if (v) *ptr = x[k][q] - cval(b, k, q) * unscale;
                }
              if (b + 1 < NBT) {
#pragma unroll
                for (int k = 0; k < RB; ++k)
#pragma unroll
                  for (int q = 0; q < 4; ++q) x[k][q] = y[k][q];
              }
            }
          }
          // The next item rewrites Cs only after every warp has read this one.
          asm volatile("bar.sync 1, 256;\n" ::: "memory");
        } else if (ok && m < ti.outM) {
          const int n0 = ti.nt * BN + CPW * part;
          double* orow = ti.out + (size_t)m * ti.ld;
#pragma unroll
          for (int c = 0; c < CPW; ++c) {
            const int n = n0 + c;
            // Lower-triangular mode writes the lower triangle and mirrors it,
            // so the stored matrix is exactly symmetric.
            if (n < ti.outN && !(args.lower_tiles && n > m)) {
              const double val = args.subtract ? orow[n] - acc[c] * unscale
                                               : acc[c] * unscale + ((args.add_identity && m == n) ? 1.0 : 0.0);
              orow[n] = val;
              if (args.lower_tiles && n != m) ti.out[(size_t)n * ti.ld + m] = val;
            }
          }
        }
        if (EPI != EPI_UPDATE)
          while (nit < n_items && !tile_item(nit, tnext)) nit += item_step;
        ti = tnext;
        it = nit;
      }
    }
  }
  // Teardown: every warp reaches this point (all waits are bounded).
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  if (warp == 1) {
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;\n" ::"r"(tmem_base), "r"(NBUF * BN));
  }
}

// ---------------------------------------------------------------------------
// Host side: tensor maps and launchers.
// ---------------------------------------------------------------------------
typedef CUresult (*EncodeTiledFn)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                                  const cuuint64_t*, const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave,
                                  CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

static EncodeTiledFn encode_fn() {
  static std::once_flag once;
  static EncodeTiledFn fn = nullptr;
  std::call_once(once, [] {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q;
    QX_CUDA(cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q));
    QX_REQUIRE(p != nullptr && q == cudaDriverEntryPointSuccess, QX_ERR_CUDA, "cuTensorMapEncodeTiled unavailable");
    fn = reinterpret_cast<EncodeTiledFn>(p);
  });
  return fn;
}

// bf16 matrix [batch][rows][ld] (K contiguous, K valid = cols) with box {64, box_rows, 1}.
static CUtensorMap make_map(const void* base, int cols, int rows, int ld, int batch, int box_rows, int rank,
                            int fp16, int bk) {
  QX_REQUIRE((reinterpret_cast<uintptr_t>(base) & 15) == 0 && (ld * 2) % 16 == 0, QX_ERR_INVALID_INPUT,
             "tensor map base/stride not 16-byte aligned");
  CUtensorMap m;
  cuuint64_t dims[3] = {(cuuint64_t)cols, (cuuint64_t)rows, (cuuint64_t)batch};
  cuuint64_t strides[2] = {(cuuint64_t)ld * 2, (cuuint64_t)ld * 2 * rows};
  cuuint32_t box[3] = {(cuuint32_t)bk, (cuuint32_t)box_rows, 1};
  cuuint32_t estr[3] = {1, 1, 1};
  CUresult r = encode_fn()(&m, fp16 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT16 : CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, rank, const_cast<void*>(base), dims, strides, box,
                           estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
                           bk == 64 ? CU_TENSOR_MAP_SWIZZLE_128B : CU_TENSOR_MAP_SWIZZLE_64B,
                           CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  QX_REQUIRE(r == CUDA_SUCCESS, QX_ERR_CUDA, "cuTensorMapEncodeTiled failed (%d)", (int)r);
  return m;
}

// 2D FP32 map over a [rows][ld] array (cols valid), box 32 columns x box_rows
// with the 128-byte swizzle (32 floats = one 128-byte row of the atom).
static CUtensorMap make_map_f32(const float* base, int cols, int rows, int ld, int box_rows) {
  QX_REQUIRE((reinterpret_cast<uintptr_t>(base) & 15) == 0 && (ld * 4) % 16 == 0, QX_ERR_INVALID_INPUT,
             "tensor map base/stride not 16-byte aligned");
  CUtensorMap m;
  cuuint64_t dims[2] = {(cuuint64_t)cols, (cuuint64_t)rows};
  cuuint64_t strides[1] = {(cuuint64_t)ld * 4};
  cuuint32_t box[2] = {32, (cuuint32_t)box_rows};
  cuuint32_t estr[2] = {1, 1};
  CUresult r = encode_fn()(&m, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 2, const_cast<float*>(base), dims, strides, box, estr,
                           CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B,
                           CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  QX_REQUIRE(r == CUDA_SUCCESS, QX_ERR_CUDA, "cuTensorMapEncodeTiled failed (%d)", (int)r);
  return m;
}

// (cudaDeviceGetAttribute: a full property query costs milliseconds per call.)
bool tc_supported(qx_ctx* ctx) {
  int major = 0;
  if (cudaDeviceGetAttribute(&major, cudaDevAttrComputeCapabilityMajor, ctx->device) != cudaSuccess) return false;
  return major == 10;
}

// max|x| per batch (x >= 0 compares as its bit pattern).  Index type I: 32-bit
// when rows * cols < 2^31 (the division per element is then cheap).  Four
// independent loads per thread and step keep enough bytes in flight for HBM.
template <typename I>
__global__ void k_amax(const double* __restrict__ src, int rows, int cols, int ld, size_t stride,
                       unsigned long long* __restrict__ out) {
  const int b = blockIdx.y;
  const double* S = src + (size_t)b * stride;
  double m = 0.0;
  const I total = (I)rows * (I)cols, ucols = (I)cols;
  const I step = (I)gridDim.x * blockDim.x;
  for (I i = (I)blockIdx.x * blockDim.x + threadIdx.x; i < total; i += 4 * step) {
    double v[4];
#pragma unroll
    for (int u = 0; u < 4; ++u) {
      const I j = i + (I)u * step;
      v[u] = 0.0;
      if (j < total) {
        const I r = j / ucols, c = j - r * ucols;
        v[u] = fabs(S[(size_t)r * ld + c]);
      }
    }
    m = fmax(m, fmax(fmax(v[0], v[1]), fmax(v[2], v[3])));
  }
  // One atomic per block: same-address atomics serialise in L2, so a per-warp
  // atomic over thousands of blocks costs more than the pass itself.
  __shared__ double wmax[32];
  for (int o = 16; o > 0; o >>= 1) m = fmax(m, __shfl_xor_sync(0xffffffffu, m, o));
  if ((threadIdx.x & 31) == 0) wmax[threadIdx.x >> 5] = m;
  __syncthreads();
  if (threadIdx.x < 32) {
    m = threadIdx.x < (blockDim.x >> 5) ? wmax[threadIdx.x] : 0.0;
    for (int o = 16; o > 0; o >>= 1) m = fmax(m, __shfl_xor_sync(0xffffffffu, m, o));
    if (threadIdx.x == 0) atomicMax(out + b, __double_as_longlong(m));
  }
}

// Power-of-two scale s for batch b: the largest 2^k with 2^k * bound <= 32768,
// bound = amax_src * amax_col (fp16 only; 1 for bf16 or an empty bound).
__device__ __forceinline__ float split_scale(int fp16, int b, size_t src_stride,
                                             const unsigned long long* __restrict__ amax_src,
                                             const unsigned long long* __restrict__ amax_col) {
  float s = 1.0f;
  if (fp16) {
    double bound = __longlong_as_double(amax_src[src_stride ? b : 0]);
    if (amax_col) bound *= __longlong_as_double(amax_col[b]);
    if (bound > 0.0 && isfinite(bound)) s = exp2f(floorf(log2f((float)(32768.0 / bound))));
  }
  return s;
}

// Split s*x*c into hi/lo (bf16 or fp16).  c = colscale[b][col] (or 1); s is a
// power of two from the bound amax_src * amax_col (fp16 only, else 1) and is
// written to scale_out[b].
__global__ void k_split(const double* __restrict__ src, int rows, int cols, int ld_src, size_t src_stride,
                        const double* __restrict__ colscale, int ld_cs, void* __restrict__ hi_, void* __restrict__ lo_,
                        int ld_dst, size_t dst_stride, int fp16, const unsigned long long* __restrict__ amax_src,
                        const unsigned long long* __restrict__ amax_col, float* __restrict__ scale_out) {
  const int b = blockIdx.y;
  const float s = split_scale(fp16, b, src_stride, amax_src, amax_col);
  if (blockIdx.x == 0 && threadIdx.x == 0 && scale_out) scale_out[b] = s;
  const size_t total = (size_t)rows * ld_dst;
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < total; i += (size_t)gridDim.x * blockDim.x) {
    const int r = (int)(i / ld_dst), c = (int)(i % ld_dst);
    double x = 0.0;
    if (c < cols) {
      x = src[(size_t)b * src_stride + (size_t)r * ld_src + c];
      if (colscale) x *= colscale[(size_t)b * ld_cs + c];
    }
    x *= (double)s;
    uint16_t h, l;
    if (fp16)
      split_round<true>(x, h, l);
    else
      split_round<false>(x, h, l);
    reinterpret_cast<uint16_t*>(hi_)[(size_t)b * dst_stride + i] = h;
    reinterpret_cast<uint16_t*>(lo_)[(size_t)b * dst_stride + i] = l;
  }
}

// Eight source values of row `row` from column c0 (zero past cols), times the
// column scales cs[c0..] when cs is given.  16-byte loads for a full group.
__device__ __forceinline__ void load8(const double* __restrict__ row, const double* __restrict__ cs, int c0,
                                      int cols, double (&x)[8]) {
  if (c0 + 8 <= cols) {
#pragma unroll
    for (int j = 0; j < 8; j += 2) {
      const double2 v = *reinterpret_cast<const double2*>(row + c0 + j);
      x[j] = v.x;
      x[j + 1] = v.y;
    }
    if (cs) {
#pragma unroll
      for (int j = 0; j < 8; j += 2) {
        const double2 v = *reinterpret_cast<const double2*>(cs + c0 + j);
        x[j] *= v.x;
        x[j + 1] *= v.y;
      }
    }
  } else {
#pragma unroll
    for (int j = 0; j < 8; ++j) {
      x[j] = 0.0;
      if (c0 + j < cols) {
        x[j] = row[c0 + j];
        if (cs) x[j] *= cs[c0 + j];
      }
    }
  }
}

// hi/lo of s*x[0..8) packed into one 16-byte word each (split_round, as k_split).
template <bool FP16>
__device__ __forceinline__ void split8_store(const double (&x)[8], float s, uint4* __restrict__ H,
                                             uint4* __restrict__ L) {
  uint32_t hw[4], lw[4];
  const double sd = (double)s;
#pragma unroll
  for (int j = 0; j < 8; j += 2) split_round2<FP16>(x[j] * sd, x[j + 1] * sd, hw[j >> 1], lw[j >> 1]);
  *H = make_uint4(hw[0], hw[1], hw[2], hw[3]);
  *L = make_uint4(lw[0], lw[1], lw[2], lw[3]);
}

// k_split with eight destination columns per thread: double2 loads and one
// 16-byte store each of hi and lo.  Same rounding as k_split, element for
// element.  Requires ld_dst % 8 == 0 (a group never straddles rows), 16-byte
// aligned hi/lo with dst_stride % 8 == 0, 16-byte aligned src (and colscale)
// with even ld_src, src_stride (and ld_cs), and rows * ld_dst / 8 < 2^31.
template <bool FP16>
__global__ void k_split8(const double* __restrict__ src, int rows, int cols, int ld_src, size_t src_stride,
                         const double* __restrict__ colscale, int ld_cs, void* __restrict__ hi_,
                         void* __restrict__ lo_, int ld_dst, size_t dst_stride,
                         const unsigned long long* __restrict__ amax_src,
                         const unsigned long long* __restrict__ amax_col, float* __restrict__ scale_out) {
  const int b = blockIdx.y;
  const float s = split_scale(FP16, b, src_stride, amax_src, amax_col);
  if (blockIdx.x == 0 && threadIdx.x == 0 && scale_out) scale_out[b] = s;
  const unsigned gpr = (unsigned)ld_dst >> 3;
  const unsigned total = (unsigned)rows * gpr;
  const double* S = src + (size_t)b * src_stride;
  const double* CS = colscale ? colscale + (size_t)b * ld_cs : nullptr;
  uint4* H = reinterpret_cast<uint4*>(reinterpret_cast<uint16_t*>(hi_) + (size_t)b * dst_stride);
  uint4* L = reinterpret_cast<uint4*>(reinterpret_cast<uint16_t*>(lo_) + (size_t)b * dst_stride);
  for (unsigned g = blockIdx.x * blockDim.x + threadIdx.x; g < total; g += gridDim.x * blockDim.x) {
    const unsigned r = g / gpr;
    const int c0 = (int)(g - r * gpr) << 3;
    double x[8];
    load8(S + (size_t)r * ld_src, CS, c0, cols, x);
    split8_store<FP16>(x, s, H + g, L + g);
  }
}

// k_split8 for one source shared by every batch (src_stride == 0) with a
// column scale per batch (the chi-scaled operand of P0): each thread reads the
// eight source values of RB rows once and writes the hi/lo groups of all
// batches, so the FP64 source crosses memory once instead of once per batch,
// and each batch's eight column scales are loaded once for the RB rows (with
// RB = 1 the scale loads are twice the hi/lo bytes stored and the kernel is
// bound by L1 traffic).  The per-batch scales sit in shared memory ([batch]
// floats, batch <= 1024).
template <bool FP16, int RB>
__global__ void __launch_bounds__(256, 2)
    k_split8_bcast(const double* __restrict__ src, int rows, int cols, int ld_src,
                   const double* __restrict__ colscale, int ld_cs, void* __restrict__ hi_, void* __restrict__ lo_,
                   int ld_dst, size_t dst_stride, int batch, const unsigned long long* __restrict__ amax_src,
                   const unsigned long long* __restrict__ amax_col, float* __restrict__ scale_out) {
  __shared__ float s_scale[1024];
  for (int b = threadIdx.x; b < batch; b += blockDim.x) {
    s_scale[b] = split_scale(FP16, b, 0, amax_src, amax_col);
    if (blockIdx.x == 0 && scale_out) scale_out[b] = s_scale[b];
  }
  __syncthreads();
  const unsigned gpr = (unsigned)ld_dst >> 3;
  const unsigned total = ((unsigned)rows + RB - 1) / RB * gpr;
  uint4* H = reinterpret_cast<uint4*>(hi_);
  uint4* L = reinterpret_cast<uint4*>(lo_);
  const size_t bstride = dst_stride >> 3;  // in 16-byte groups
  for (unsigned g = blockIdx.x * blockDim.x + threadIdx.x; g < total; g += gridDim.x * blockDim.x) {
    const unsigned rb = g / gpr;
    const unsigned cg = g - rb * gpr;
    const int c0 = (int)cg << 3;
    const int r0 = (int)rb * RB;
    const int nr = min(RB, rows - r0);
    double x0[RB][8];
#pragma unroll
    for (int i = 0; i < RB; ++i) {
      if (i < nr) {
        load8(src + (size_t)(r0 + i) * ld_src, nullptr, c0, cols, x0[i]);
      } else {
#pragma unroll
        for (int j = 0; j < 8; ++j) x0[i][j] = 0.0;
      }
    }
    const bool full = c0 + 8 <= cols;
    const size_t g0 = (size_t)r0 * gpr + cg;  // group of (r0, c0) in one batch
    for (int b = 0; b < batch; ++b) {
      const double* cs = colscale + (size_t)b * ld_cs;
      double c[8];
      if (full) {
#pragma unroll
        for (int j = 0; j < 8; j += 2) {
          const double2 v = *reinterpret_cast<const double2*>(cs + c0 + j);
          c[j] = v.x;
          c[j + 1] = v.y;
        }
      } else {
#pragma unroll
        for (int j = 0; j < 8; ++j) c[j] = (c0 + j < cols) ? cs[c0 + j] : 0.0;
      }
      const float sb = s_scale[b];
      const size_t gb = (size_t)b * bstride + g0;
#pragma unroll
      for (int i = 0; i < RB; ++i) {
        if (i < nr) {
          double x[8];
#pragma unroll
          for (int j = 0; j < 8; ++j) x[j] = x0[i][j] * c[j];
          split8_store<FP16>(x, sb, H + gb + (size_t)i * gpr, L + gb + (size_t)i * gpr);
        }
      }
    }
  }
}

// Scratch for the amax words and scales: [0, 1024) amax of sources, [1024, 2048)
// amax of column scales, then float scales.
struct SplitScratch {
  unsigned long long* amax_src;
  unsigned long long* amax_col;
  float* scale;
};
static SplitScratch split_scratch(qx_ctx* ctx, int slot_offset) {
  DevBuf& b = ctx->ws[WS_TCERR];
  b.reserve(256 + 8 * 20480);
  uint8_t* p = b.as<uint8_t>() + 256 + slot_offset * 20480;
  SplitScratch s;
  s.amax_src = reinterpret_cast<unsigned long long*>(p);
  s.amax_col = s.amax_src + 1024;
  s.scale = reinterpret_cast<float*>(s.amax_col + 1024);
  return s;
}

static void split(qx_ctx* ctx, const double* src, int rows, int cols, int ld_src, size_t src_stride, void* hi,
                  void* lo, int ld_dst, size_t dst_stride, int batch, const double* colscale, int ld_cs, int fp16,
                  int slot, float** scale_out, const unsigned long long* given_amax = nullptr,
                  cudaStream_t stream = nullptr) {
  QX_REQUIRE(batch <= 1024, QX_ERR_INVALID_INPUT, "at most 1024 frequencies per split");
  SplitScratch sc = split_scratch(ctx, slot);
  cudaStream_t st = stream ? stream : ctx->stream;
  if (fp16) {
    const int nsrc = src_stride ? batch : 1;
    if (given_amax) {
      // The source's bound is already on the device (the same source split
      // before, or accumulated by the kernel that wrote it).
      sc.amax_src = const_cast<unsigned long long*>(given_amax);
      if (colscale) QX_CUDA(cudaMemsetAsync(sc.amax_col, 0, 1024 * sizeof(unsigned long long), st));
    } else {
      QX_CUDA(cudaMemsetAsync(sc.amax_src, 0, 2048 * sizeof(unsigned long long), st));
      // About eight blocks per SM over all batches, each thread four
      // elements per step at least.
      const size_t tot = (size_t)rows * cols;
      const size_t per_batch = std::max<size_t>(1, 1184 / nsrc);
      dim3 g1((unsigned)std::min<size_t>((tot + 1023) / 1024, per_batch), nsrc);
      if (tot < (1u << 31))
        k_amax<unsigned><<<g1, 256, 0, st>>>(src, rows, cols, ld_src, src_stride, sc.amax_src);
      else
        k_amax<size_t><<<g1, 256, 0, st>>>(src, rows, cols, ld_src, src_stride, sc.amax_src);
      check_launch(ctx);
    }
    if (colscale) {
      dim3 g2(ceil_div(cols, 1024), batch);
      k_amax<unsigned><<<g2, 256, 0, st>>>(colscale, 1, cols, ld_cs, ld_cs, sc.amax_col);
      check_launch(ctx);
    }
  }
  auto a16 = [](const void* p) { return (reinterpret_cast<uintptr_t>(p) & 15) == 0; };
  const bool vec = ld_dst % 8 == 0 && dst_stride % 8 == 0 && a16(hi) && a16(lo) && ld_src % 2 == 0 &&
                   src_stride % 2 == 0 && a16(src) && (!colscale || (a16(colscale) && ld_cs % 2 == 0));
  const unsigned long long* acol = colscale ? sc.amax_col : nullptr;
  const size_t groups = (size_t)rows * (ld_dst / 8);
  if (vec && groups < (1u << 31) && src_stride == 0 && colscale && batch > 1) {
    // Four rows per thread when that still gives every SM two full blocks
    // (the kernel's residency), else one; a grid-stride loop over at most
    // those resident blocks.
    const size_t resident = 2 * (size_t)std::max(ctx->sm_count, 1);
    const bool rb4 = (groups + 3) / 4 >= resident * 256;
    const size_t items = rb4 ? ((size_t)(rows + 3) / 4) * (ld_dst / 8) : groups;
    dim3 grid((unsigned)std::min<size_t>((items + 255) / 256, rb4 ? resident : 4096));
    if (fp16 && rb4)
      k_split8_bcast<true, 4><<<grid, 256, 0, st>>>(src, rows, cols, ld_src, colscale, ld_cs, hi, lo, ld_dst,
                                                    dst_stride, batch, sc.amax_src, acol, sc.scale);
    else if (fp16)
      k_split8_bcast<true, 1><<<grid, 256, 0, st>>>(src, rows, cols, ld_src, colscale, ld_cs, hi, lo, ld_dst,
                                                    dst_stride, batch, sc.amax_src, acol, sc.scale);
    else if (rb4)
      k_split8_bcast<false, 4><<<grid, 256, 0, st>>>(src, rows, cols, ld_src, colscale, ld_cs, hi, lo, ld_dst,
                                                     dst_stride, batch, sc.amax_src, acol, sc.scale);
    else
      k_split8_bcast<false, 1><<<grid, 256, 0, st>>>(src, rows, cols, ld_src, colscale, ld_cs, hi, lo, ld_dst,
                                                     dst_stride, batch, sc.amax_src, acol, sc.scale);
  } else if (vec && groups < (1u << 31)) {
    dim3 grid((unsigned)std::min<size_t>((groups + 255) / 256, 4096), batch);
    if (fp16)
      k_split8<true><<<grid, 256, 0, st>>>(src, rows, cols, ld_src, src_stride, colscale, ld_cs, hi, lo,
                                                    ld_dst, dst_stride, sc.amax_src, acol, sc.scale);
    else
      k_split8<false><<<grid, 256, 0, st>>>(src, rows, cols, ld_src, src_stride, colscale, ld_cs, hi, lo,
                                                     ld_dst, dst_stride, sc.amax_src, acol, sc.scale);
  } else {
    const size_t total = (size_t)rows * ld_dst;
    dim3 grid((unsigned)std::min<size_t>((total + 255) / 256, 4096), batch);
    k_split<<<grid, 256, 0, st>>>(src, rows, cols, ld_src, src_stride, colscale, ld_cs, hi, lo, ld_dst,
                                           dst_stride, fp16, sc.amax_src, acol, sc.scale);
  }
  check_launch(ctx);
  if (scale_out) *scale_out = sc.scale;
}

void launch_split(qx_ctx* ctx, const double* src, int rows, int cols, int ld_src, void* hi, void* lo, int ld_dst,
                  size_t src_stride, size_t dst_stride, int batch, int fp16, int slot, float** scale_out,
                  const unsigned long long* given_amax) {
  split(ctx, src, rows, cols, ld_src, src_stride, hi, lo, ld_dst, dst_stride, batch, nullptr, 0, fp16, slot,
        scale_out, given_amax);
}

unsigned long long* split_amax_words(qx_ctx* ctx, int slot) { return split_scratch(ctx, slot).amax_src; }

__global__ void k_fill_u64(unsigned long long* __restrict__ w, int n, unsigned long long v) {
  for (int i = threadIdx.x; i < n; i += blockDim.x) w[i] = v;
}

unsigned long long* split_bound_words(qx_ctx* ctx, int slot, int n, double bound) {
  QX_REQUIRE(n > 0 && n <= 1024, QX_ERR_INVALID_INPUT, "at most 1024 bounds per split");
  unsigned long long* w = split_scratch(ctx, slot).amax_src;
  unsigned long long bits;
  std::memcpy(&bits, &bound, sizeof bits);
  k_fill_u64<<<1, 256, 0, ctx->stream>>>(w, n, bits);
  check_launch(ctx);
  return w;
}

// One error word per launch, from the context's status arena.
static int* tc_err_slot(qx_ctx* ctx) { return status_words(ctx, 1); }

static void check_tc_err(qx_ctx* ctx, int* d_err) { ctx->pending.push_back({d_err, 1, 0}); }

template <int BN, int EPI, bool CONVB = false>
static void launch_tc(qx_ctx* ctx, const CUtensorMap& ah, const CUtensorMap& al, const CUtensorMap& bh,
                      const CUtensorMap& bl, const TcArgs& a, dim3 grid, cudaStream_t stream = nullptr) {
  using L = TcSmem<BN, EPI, CONVB>;
  static PerDeviceOnce attr_once;
  attr_once(ctx->device, [&] {
    QX_CUDA(cudaFuncSetAttribute(k_tc_gemm<BN, EPI, CONVB>, cudaFuncAttributeMaxDynamicSharedMemorySize, L::TOTAL));
  });
  k_tc_gemm<BN, EPI, CONVB><<<grid, TcThreads<EPI, CONVB>::VALUE, L::TOTAL, stream ? stream : ctx->stream>>>(
      ah, al, bh, bl, a);
  check_launch(ctx);
}

// Autotuned frequency-group size of the pair contraction, per (npair, naux,
// nw, device): candidates 4, 8, 16, 32 (<= nw) are timed with CUDA events on
// the first call of a shape; later calls reuse the fastest.
template <class F>
static int tuned_wgroup(qx_ctx* ctx, int npair, int naux, int nw, F&& launch_with) {
  static std::mutex mu;
  static std::map<std::array<int, 4>, int> table;
  const std::array<int, 4> key{npair, naux, nw, ctx->device};
  {
    std::lock_guard<std::mutex> lock(mu);
    auto it = table.find(key);
    if (it != table.end()) return it->second;
  }
  std::vector<int> cand;
  for (int g : {4, 8, 16, 32})
    if (g <= nw) cand.push_back(g);
  if (cand.empty()) cand.push_back(nw);
  cudaEvent_t e0, e1;
  QX_CUDA(cudaEventCreate(&e0));
  QX_CUDA(cudaEventCreate(&e1));
  int best = cand[0];
  float best_ms = 1e30f;
  for (int g : cand) {
    QX_CUDA(cudaEventRecord(e0, ctx->stream));
    launch_with(g);
    QX_CUDA(cudaEventRecord(e1, ctx->stream));
    QX_CUDA(cudaEventSynchronize(e1));
    float ms = 0.f;
    QX_CUDA(cudaEventElapsedTime(&ms, e0, e1));
    if (ms < best_ms) {
      best_ms = ms;
      best = g;
    }
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  std::lock_guard<std::mutex> lock(mu);
  table[key] = best;
  return best;
}

// v[w][p] = 2 sum_Q X[p][Q] sum_{P <= Q} (Bh+Bl)[p][P] (W'h+W'l)[w][Q][P] / (sA sB[w]),
// W' the half-lower form of Wc (three products per term)
// ---------------------------------------------------------------------------
// The pair contraction on CTA pairs (tcgen05 cta_group::2, M = 256, N = 256).
// ---------------------------------------------------------------------------
// The two CTAs of a cluster take the items (pair-block pair, frequency) in the
// order of the single-CTA form; CTA r of the pair holds pair block 2 i + r
// (a copy of 2 i, not stored, past the last block) and, of each 256-wide N
// tile of W', the rows [n0 + 128 r, n0 + 128 r + 128).  The even CTA's MMAs
// read both CTAs' operands and leave each CTA's 128 x 256 accumulator in its
// own TMEM, which its ROWDOT epilogue contracts with its own pair rows.  Per
// k block an SM loads 64 KB (its A rows and half of the W' tile) instead of
// 96 KB: in the single-CTA form the MMA thread waited ~40 % of each k block
// for the TMA loads.  Barrier protocol as in k_p0_pair.
namespace pairrd {
constexpr int STAGES = 3;
constexpr int BK = 64;
constexpr int BN = 256;                              // N of the MMA (both CTAs)
constexpr int A_BYTES = TC_BM * BK * 2;              // 16 KB: this CTA's 128 pair rows
constexpr int B_BYTES = (BN / 2) * BK * 2;           // 16 KB: half of the W' tile
constexpr int STAGE_BYTES = 2 * A_BYTES + 2 * B_BYTES;  // 64 KB
constexpr int BAR_OFF = STAGES * STAGE_BYTES;
constexpr int RED_OFF = BAR_OFF + 256;
constexpr int TOTAL = RED_OFF + 2 * (2 * TC_BM + 8) * 8 + 1024;
constexpr int NEPI = 8;
constexpr int THREADS = 64 + 32 * NEPI;
}  // namespace pairrd

__global__ void __launch_bounds__(pairrd::THREADS, 1)
    k_rowdot_pair(const __grid_constant__ CUtensorMap mapAh, const __grid_constant__ CUtensorMap mapAl,
                  const __grid_constant__ CUtensorMap mapBh, const __grid_constant__ CUtensorMap mapBl, TcArgs args) {
  namespace P = pairrd;
  if (cluster_nctarank() != 2) {
    if (threadIdx.x == 0) atomicCAS(args.err, 0, 30);
    return;
  }
  extern __shared__ __align__(1024) uint8_t smem_raw[];
  uint8_t* smem = reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
  uint64_t* full = reinterpret_cast<uint64_t*>(smem + P::BAR_OFF);
  uint64_t* empty = full + P::STAGES;
  uint64_t* acc_full = empty + P::STAGES;  // [2]
  uint64_t* acc_empty = acc_full + 2;      // [2]
  uint64_t* drain = acc_empty + 2;
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(drain + 1);
  volatile int* abort_flag = reinterpret_cast<volatile int*>(tmem_slot + 1);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const uint32_t rank = cluster_ctarank();
  const bool leader = rank == 0;
  const int n_tiles = (args.N + P::BN - 1) / P::BN;
  const int k_blocks = (args.K + P::BK - 1) / P::BK;
  const int mpairs = (args.m_blocks + 1) / 2;
  const int g = args.wgroup;
  const int n_items = (args.nbatch + g - 1) / g * mpairs * g;
  const int item0 = (int)cluster_id_x(), item_step = (int)cluster_count_x();
  // Item -> frequency, this CTA's pair block and whether its rows are stored.
  auto item_of = [&](int b, int& mb, int& w, bool& store) {
    const int per_group = mpairs * g;
    const int grp = b / per_group, r = b % per_group;
    const int mp = r / g;
    w = grp * g + r % g;
    mb = 2 * mp + (int)rank;
    store = mb < args.m_blocks;
    if (!store) mb = 2 * mp;
  };
  // K range of N tile nt: W' is half-lower, zero past column n0 + BN.
  auto kbe_of = [&](int nt) { return min(k_blocks, (nt * P::BN + P::BN + P::BK - 1) / P::BK); };

  if (threadIdx.x == 0) {
    for (int s = 0; s < P::STAGES; ++s) {
      mbar_init(&full[s], 1);
      mbar_init(&empty[s], 1);
    }
    for (int b = 0; b < 2; ++b) {
      mbar_init(&acc_full[b], 1);
      mbar_init(&acc_empty[b], 2 * P::NEPI);  // every epilogue warp of both CTAs
    }
    mbar_init(drain, 1);
    *abort_flag = 0;
    asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
  }
  if (warp == 1) {
    asm volatile("tcgen05.alloc.cta_group::2.sync.aligned.shared::cta.b32 [%0], %1;\n" ::"r"(smem_u32(tmem_slot)),
                 "r"(2 * P::BN));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::2.sync.aligned;\n" ::);
  }
  tc_fence_before();
  __syncthreads();
  cluster_sync_all();
  tc_fence_after();
  const uint32_t tmem_base = *tmem_slot;

  if (warp == 0) {
    // ---------------- TMA producer (both CTAs) ----------------
    if (lane == 0) {
      const uint32_t full_leader = mapa_rank(smem_u32(full), 0);
      int gk = 0;
      bool ok = true;
      for (int it = item0; it < n_items && ok; it += item_step) {
        int mb, w;
        bool st;
        item_of(it, mb, w, st);
        if (w >= args.nbatch) continue;
        for (int nt = 0; nt < n_tiles && ok; ++nt) {
          const int kbe = kbe_of(nt);
          for (int kb = 0; kb < kbe; ++kb, ++gk) {
            const int s = gk % P::STAGES;
            if (gk >= P::STAGES && !mbar_wait(&empty[s], ((gk / P::STAGES) - 1) & 1, abort_flag, args.err, 31)) {
              ok = false;
              break;
            }
            if (leader) mbar_expect_tx(&full[s], 2 * P::STAGE_BYTES);
            const uint32_t dst = smem_u32(smem + s * P::STAGE_BYTES);
            const uint32_t fb = full_leader + s * 8;
            const int k0 = kb * P::BK;
            const int brow = nt * P::BN + (P::BN / 2) * (int)rank;
            tma_load_2d_pair(dst, &mapAh, fb, k0, mb * TC_BM);
            tma_load_2d_pair(dst + P::A_BYTES, &mapAl, fb, k0, mb * TC_BM);
            tma_load_3d_pair(dst + 2 * P::A_BYTES, &mapBh, fb, k0, brow, w);
            tma_load_3d_pair(dst + 2 * P::A_BYTES + P::B_BYTES, &mapBl, fb, k0, brow, w);
          }
        }
      }
      for (int q = (gk > P::STAGES ? gk - P::STAGES : 0); q < gk; ++q) {
        volatile int no_abort = 0;
        mbar_wait(&empty[q % P::STAGES], (q / P::STAGES) & 1, &no_abort, args.err, 32);
      }
    }
  } else if (warp == 1) {
    // ---------------- MMA issuer (even CTA) ----------------
    if (leader && lane == 0) {
      const uint32_t idesc = umma_idesc_f16(2 * TC_BM, P::BN, args.fp16);
      int gk = 0, t = 0;
      bool ok = true;
      for (int it = item0; it < n_items && ok; it += item_step) {
        int mb, w;
        bool st;
        item_of(it, mb, w, st);
        if (w >= args.nbatch) continue;
        for (int nt = 0; nt < n_tiles && ok; ++nt, ++t) {
          const int kbe = kbe_of(nt);
          const int buf = t & 1;
          if (t >= 2 && !mbar_wait_cluster(&acc_empty[buf], ((t / 2) - 1) & 1, abort_flag, args.err, 33)) {
            ok = false;
            break;
          }
          const uint32_t dacc = tmem_base + buf * P::BN;
          for (int kb = 0; kb < kbe; ++kb, ++gk) {
            const int s = gk % P::STAGES;
            if (!mbar_wait(&full[s], (gk / P::STAGES) & 1, abort_flag, args.err, 34)) {
              ok = false;
              break;
            }
            tc_fence_after();
            const uint32_t ah = smem_u32(smem + s * P::STAGE_BYTES), al = ah + P::A_BYTES;
            const uint32_t bh = ah + 2 * P::A_BYTES, bl = bh + P::B_BYTES;
#pragma unroll
            for (int kk = 0; kk < P::BK / 16; ++kk) {
              const uint32_t off = kk * 32;
              const uint32_t acc0 = (kb > 0 || kk > 0) ? 1u : 0u;
              umma_f16_pair(dacc, umma_desc<P::BK>(ah + off), umma_desc<P::BK>(bh + off), idesc, acc0);
              umma_f16_pair(dacc, umma_desc<P::BK>(ah + off), umma_desc<P::BK>(bl + off), idesc, 1u);
              umma_f16_pair(dacc, umma_desc<P::BK>(al + off), umma_desc<P::BK>(bh + off), idesc, 1u);
            }
            umma_commit_pair_both(&empty[s]);
          }
          if (!ok) break;
          umma_commit_pair_both(&acc_full[buf]);
        }
      }
      umma_commit_pair_own(drain);
      volatile int no_abort = 0;
      mbar_wait(drain, 0, &no_abort, args.err, 35);
    }
  } else {
    // ---------------- epilogue (warps 2..9, both CTAs): row dot products ----------------
    const int quarter = warp & 3;
    const int half = (warp - 2) >> 2;
    const int row = quarter * 32 + lane;
    constexpr int HB = P::BN / 2;
    int t = 0, done_items = 0;
    bool ok = true;
    for (int it = item0; it < n_items && ok; it += item_step) {
      int mb, w;
      bool st;
      item_of(it, mb, w, st);
      if (w >= args.nbatch) continue;
      const int m = mb * TC_BM + row;
      double rowsum = 0.0;
      int tiles_done = 0;
      for (int nt = 0; nt < n_tiles; ++nt, ++t) {
        const int buf = t & 1;
        if (!mbar_wait(&acc_full[buf], (t / 2) & 1, abort_flag, args.err, 36)) {
          ok = false;
          break;
        }
        tc_fence_after();
        const int n0 = nt * P::BN + half * HB;
        const uint32_t taddr = tmem_base + ((uint32_t)(quarter * 32) << 16) + buf * P::BN + half * HB;
        const float* xrow = args.X + (size_t)(m < args.M ? m : 0) * args.ldx + n0;
        float xn[16];
        load_x16(xrow, n0, args.N, m < args.M, xn);
#pragma unroll 1
        for (int c = 0; c < HB; c += 16) {
          float xc[16];
#pragma unroll
          for (int q = 0; q < 16; ++q) xc[q] = xn[q];
          if (c + 16 < HB) load_x16(xrow + c + 16, n0 + c + 16, args.N, m < args.M, xn);
          float v[16];
          tmem_ld16(taddr + c, v);
          rowsum += chunk_dot16(v, xc);
        }
        tc_fence_before();
        __syncwarp();
        if (lane == 0) {
          if (leader)
            mbar_arrive(&acc_empty[buf]);
          else
            mbar_arrive_rank(&acc_empty[buf], 0);
        }
        ++tiles_done;
      }
      // Combine the two halves (named barrier of the 8 epilogue warps, reached
      // by every one of them, also after an abort); the buffer alternates
      // between items.
      double* red = reinterpret_cast<double*>(smem + P::RED_OFF) + (done_items & 1) * (2 * TC_BM + 8);
      int* done = reinterpret_cast<int*>(red + 2 * TC_BM);
      const bool full_item = tiles_done == n_tiles;
      red[half * TC_BM + row] = full_item ? rowsum : 0.0;
      if (lane == 0 && quarter == 0) done[half] = full_item ? 1 : 0;
      asm volatile("bar.sync 1, 256;\n" ::: "memory");
      if (half == 0 && st && m < args.M && done[0] && done[1])
        args.out[(size_t)w * args.ldo + m] = (red[row] + red[TC_BM + row]) * unscale_rowdot(args, w) * 2.0;
      ++done_items;
      ok = done[0] && done[1];
    }
  }
  tc_fence_before();
  __syncthreads();
  cluster_sync_all();
  tc_fence_after();
  if (warp == 1) {
    asm volatile("tcgen05.dealloc.cta_group::2.sync.aligned.b32 %0, %1;\n" ::"r"(tmem_base), "r"(2 * P::BN));
  }
}

static void launch_rowdot_pair(qx_ctx* ctx, const CUtensorMap& ah, const CUtensorMap& al, const CUtensorMap& bh,
                               const CUtensorMap& bl, const TcArgs& a) {
  static PerDeviceOnce attr_once;
  static int max_clusters[PerDeviceOnce::kMaxDevices] = {};
  cudaLaunchConfig_t cfg = {};
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeClusterDimension;
  attr[0].val.clusterDim.x = 2;
  attr[0].val.clusterDim.y = 1;
  attr[0].val.clusterDim.z = 1;
  cfg.blockDim = dim3(pairrd::THREADS);
  cfg.dynamicSmemBytes = pairrd::TOTAL;
  cfg.stream = ctx->stream;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  attr_once(ctx->device, [&] {
    QX_CUDA(cudaFuncSetAttribute(k_rowdot_pair, cudaFuncAttributeMaxDynamicSharedMemorySize, pairrd::TOTAL));
    cfg.gridDim = dim3(2 * ctx->sm_count);
    int n = 0;
    QX_CUDA(cudaOccupancyMaxActiveClusters(&n, k_rowdot_pair, &cfg));
    max_clusters[ctx->device] = std::max(n, 1);
  });
  const int items = ceil_div(a.nbatch, a.wgroup) * ceil_div(a.m_blocks, 2) * a.wgroup;
  cfg.gridDim = dim3(2 * std::min(items, max_clusters[ctx->device]));
  QX_CUDA(cudaLaunchKernelEx(&cfg, k_rowdot_pair, ah, al, bh, bl, a));
  check_launch(ctx);
}

void launch_pair_contract_tc(qx_ctx* ctx, const TcOperand& A, const float* bpt_f32, int ldk, int npair, int naux,
                             const TcOperand& W, int ldw, size_t wc_stride, int nw, double* v, int ldv, int fp16) {
  constexpr int BN = 256;
  QX_REQUIRE(wc_stride == (size_t)naux * ldw, QX_ERR_INVALID_INPUT, "Wc stride must be naux*ldw");
  constexpr int BK = TcPipe<EPI_ROWDOT>::BK;
  CUtensorMap ah = make_map(A.hi, naux, npair, ldk, 1, TC_BM, 2, fp16, BK);
  CUtensorMap al = make_map(A.lo, naux, npair, ldk, 1, TC_BM, 2, fp16, BK);
  // CTA pairs stage half of each W' tile per CTA.
  const bool pair = ctx->contraction_form != QX_CONTRACT_SINGLE;
  CUtensorMap bh = make_map(W.hi, naux, naux, ldw, nw, pair ? BN / 2 : BN, 3, fp16, BK);
  CUtensorMap bl = make_map(W.lo, naux, naux, ldw, nw, pair ? BN / 2 : BN, 3, fp16, BK);
  int* d_err = tc_err_slot(ctx);
  QX_CUDA(cudaMemsetAsync(d_err, 0, sizeof(int), ctx->stream));
  TcArgs a{};
  a.M = npair;
  a.N = naux;
  a.K = naux;
  a.nbatch = nw;
  a.m_blocks = ceil_div(npair, TC_BM);
  a.wgroup = std::min(nw, 8);
  a.X = bpt_f32;
  a.ldx = ldk;
  a.out = v;
  a.ldo = ldv;
  a.fp16 = fp16;
  a.tri = 1;
  a.scaleA = A.scale;
  a.scaleB = W.scale;
  a.err = d_err;
  // CTA order: frequency groups of wgroup, pair blocks inside a group, the
  // group's frequencies innermost.  The group size trades L2 residency of W
  // (wgroup matrices) against re-reads of the pair tensor (nw / wgroup
  // passes); every (frequency, pair block) is still one CTA with the same
  // arithmetic, so the choice does not change the result.  It is tuned once
  // per shape by timing the candidates on the call's own data.
  auto launch_with = [&](int g) {
    a.wgroup = g;
    if (pair) {
      launch_rowdot_pair(ctx, ah, al, bh, bl, a);
    } else {
      // Persistent: one CTA per SM (192 KB of stages each) over all items.
      const int items = ceil_div(nw, g) * a.m_blocks * g;
      launch_tc<BN, EPI_ROWDOT>(ctx, ah, al, bh, bl, a, dim3(std::min(items, ctx->sm_count)));
    }
  };
  a.wgroup = tuned_wgroup(ctx, npair, naux, nw, launch_with);
  launch_with(a.wgroup);
  check_tc_err(ctx, d_err);
}

// eps[w] = I + Bov diag(chi[w]) Bov^T with A = split(Bov), B = split(Bov * chi[w]).
// bf[r][c] = (float)b[r][c] for c < cols, 0 in the padding columns [cols, ld).
__global__ void k_f32_rows(const double* __restrict__ b, int rows, int cols, int ld, float* __restrict__ bf) {
  for (size_t e = (size_t)blockIdx.x * blockDim.x + threadIdx.x; e < (size_t)rows * ld;
       e += (size_t)gridDim.x * blockDim.x) {
    const int c = (int)(e % ld);
    bf[e] = c < cols ? (float)b[e] : 0.0f;
  }
}

// Per frequency w (one block each): s_w, the power of two of the fp16 split
// of B diag(chi'_w) (largest 2^k with 2^k amax(B) max|chi'_w| <= 32768; 1 for
// bf16), and the FP32 column scales cs[w][k] = chi'_w[k] s_w (0 past nov).
__global__ void k_chi_cols(const double* __restrict__ chi, int nov, int ldov, const unsigned long long* amax_b,
                           int fp16, float* __restrict__ cs, float* __restrict__ scale) {
  const int w = blockIdx.x;
  const double* cw = chi + (size_t)w * ldov;
  double m = 0.0;
  for (int k = threadIdx.x; k < nov; k += blockDim.x) m = fmax(m, fabs(cw[k]));
  __shared__ double red[32];
  for (int o = 16; o > 0; o >>= 1) m = fmax(m, __shfl_xor_sync(0xffffffffu, m, o));
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = m;
  __syncthreads();
  if (threadIdx.x < 32) {
    m = threadIdx.x < (blockDim.x >> 5) ? red[threadIdx.x] : 0.0;
    for (int o = 16; o > 0; o >>= 1) m = fmax(m, __shfl_xor_sync(0xffffffffu, m, o));
    if (threadIdx.x == 0) red[0] = m;
  }
  __syncthreads();
  const double bound = __longlong_as_double((long long)*amax_b) * red[0];
  const double s = (fp16 && bound > 0.0 && isfinite(bound)) ? exp2(floor(log2(32768.0 / bound))) : 1.0;
  if (threadIdx.x == 0) scale[w] = (float)s;
  for (int k = threadIdx.x; k < ldov; k += blockDim.x) cs[(size_t)w * ldov + k] = k < nov ? (float)(cw[k] * s) : 0.f;
}

// ---------------------------------------------------------------------------
// P0 on CTA pairs (tcgen05 cta_group::2, M = 256).
// ---------------------------------------------------------------------------
// The two CTAs of a cluster compute two 128-row tiles (m_a, n) and (m_b, n)
// of one column of lower tiles of eps[w] with MMAs of M = 256, N = 128: each
// CTA stages its own 128 A rows and one half (64 rows) of the B tile, the MMA
// issued by the even CTA reads all four operand tiles, and each CTA's
// 128 x 128 accumulator lands in its own TMEM.  Per MMA an SM then reads 6 KB
// of operands from shared memory instead of 8 KB, and loads 48 KB per k block
// instead of 64 KB: the single-CTA 128 x 128 tile reads 128 bytes per tensor
// cycle, all of shared memory's bandwidth before the TMA writes into it.  A
// column with an odd count of lower tiles pairs its last tile with a copy of
// itself whose result is not stored.  Barriers: the even CTA's full[s] counts
// the bytes of both CTAs' loads (each CTA's TMA signals it); the MMA commits
// arrive on empty[s] and acc_full[b] of both CTAs (multicast); the even CTA's
// acc_empty[b] takes an arrival from each of its epilogue warps and one for
// all of the odd CTA's.  The epilogue sums the accumulation units in
// Kahan-compensated FP32 (below).
// Measured at nmo 300 / naux 1000 / nw 32 (a P0 stage with its split): with
// the FP64 sums of the single-CTA epilogue the pair took 2.35 ms, its MMAs
// waiting on the drain of the accumulators; with the compensated FP32 sums
// 1.74 ms, against 1.69 ms for single-CTA tiles (which drain in FP64: the
// compensated sums measured no faster there).  The single-CTA form stays the
// default; this one is QX_P0_PAIR.
namespace pairp0 {
constexpr int STAGES = 4;
constexpr int BK = 64;
constexpr int A_BYTES = TC_BM * BK * 2;            // 16 KB: this CTA's 128 A rows
constexpr int B_BYTES = (TC_BM / 2) * BK * 2;      // 8 KB: half of the N = 128 B tile
constexpr int STAGE_BYTES = 2 * A_BYTES + 2 * B_BYTES;  // 48 KB
constexpr int BAR_OFF = STAGES * STAGE_BYTES;
constexpr int TOTAL = BAR_OFF + 256 + 1024;  // + slack for the 1024-byte alignment
constexpr int NEPI = 8;
constexpr int THREADS = 64 + 32 * NEPI;
constexpr int CPW = TC_BM * 4 / NEPI;  // accumulator columns per epilogue warp
// TMEM accumulators (128 columns each, all 512 columns): the MMAs may run up
// to NBUF - 1 accumulation units ahead of the slower of the two epilogues,
// whose release of a buffer reaches the even CTA by a remote arrival.
constexpr int NBUF = 4;
}  // namespace pairp0

// Pairs of lower tiles per frequency for T tile rows: column nt holds T - nt tiles.
__host__ __device__ inline int p0_pair_count(int T) {
  int s = 0;
  for (int nt = 0; nt < T; ++nt) s += (T - nt + 1) / 2;
  return s;
}
// Pair r of a frequency -> its column nt and first tile row ma (the second is
// ma + 1, past the last tile row for the odd tile of a column).
__device__ __forceinline__ void p0_pair_tile(int r, int T, int& nt, int& ma) {
  int c = 0;
  for (nt = 0; nt < T - 1; ++nt) {
    const int cnt = (T - nt + 1) / 2;
    if (r < c + cnt) break;
    c += cnt;
  }
  ma = nt + 2 * (r - c);
}

__global__ void __launch_bounds__(pairp0::THREADS, 1)
    k_p0_pair(const __grid_constant__ CUtensorMap mapAh, const __grid_constant__ CUtensorMap mapAl,
              const __grid_constant__ CUtensorMap mapBh, const __grid_constant__ CUtensorMap mapBl, TcArgs args) {
  namespace P = pairp0;
  // Launched only in clusters of two (the launcher sets the attribute); any
  // other shape records an error before touching the tensor cores.
  if (cluster_nctarank() != 2) {
    if (threadIdx.x == 0) atomicCAS(args.err, 0, 20);
    return;
  }
  extern __shared__ __align__(1024) uint8_t smem_raw[];
  uint8_t* smem = reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
  uint64_t* full = reinterpret_cast<uint64_t*>(smem + P::BAR_OFF);
  uint64_t* empty = full + P::STAGES;
  uint64_t* acc_full = empty + P::STAGES;   // [NBUF]
  uint64_t* acc_empty = acc_full + P::NBUF;  // [NBUF]
  uint64_t* drain = acc_empty + P::NBUF;
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(drain + 1);
  volatile int* abort_flag = reinterpret_cast<volatile int*>(tmem_slot + 1);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const uint32_t rank = cluster_ctarank();
  const bool leader = rank == 0;
  const int T = args.m_blocks;
  const int pairs_pb = p0_pair_count(T);
  const int n_items = pairs_pb * args.nbatch;
  const int item0 = (int)cluster_id_x(), item_step = (int)cluster_count_x();
  const int k_blocks = (args.K + P::BK - 1) / P::BK;
  const int unit = args.unit > 0 ? args.unit : 1;
  // Item -> frequency w, column nt, this CTA's tile row m, and whether its
  // tile is stored (the odd tile's copy is not).
  auto item_tile = [&](int it, int& w, int& nt, int& m, bool& store) {
    w = it / pairs_pb;
    int ma;
    p0_pair_tile(it - w * pairs_pb, T, nt, ma);
    store = leader || ma + 1 < T;
    m = (leader || ma + 1 >= T) ? ma : ma + 1;
  };

  if (threadIdx.x == 0) {
    for (int s = 0; s < P::STAGES; ++s) {
      mbar_init(&full[s], 1);
      mbar_init(&empty[s], 1);
    }
    for (int b = 0; b < P::NBUF; ++b) {
      mbar_init(&acc_full[b], 1);
      mbar_init(&acc_empty[b], P::NEPI + 1);  // the even CTA's epilogue warps, one arrival for the odd CTA's
    }
    mbar_init(drain, 1);
    *abort_flag = 0;
    asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
  }
  if (warp == 1) {
    // Both CTAs' MMA warps allocate together; the columns are the same in both.
    asm volatile("tcgen05.alloc.cta_group::2.sync.aligned.shared::cta.b32 [%0], %1;\n" ::"r"(smem_u32(tmem_slot)),
                 "r"(P::NBUF * TC_BM));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::2.sync.aligned;\n" ::);
  }
  tc_fence_before();
  __syncthreads();
  // The other CTA's barriers are initialised before any remote arrival.
  cluster_sync_all();
  tc_fence_after();
  const uint32_t tmem_base = *tmem_slot;

  if (warp == 0) {
    // ---------------- TMA producer (both CTAs) ----------------
    if (lane == 0) {
      const uint32_t full_leader = mapa_rank(smem_u32(full), 0);
      int g = 0;
      bool ok = true;
      for (int it = item0; it < n_items && ok; it += item_step) {
        int w, nt, m;
        bool st;
        item_tile(it, w, nt, m, st);
        for (int kb = 0; kb < k_blocks; ++kb, ++g) {
          const int s = g % P::STAGES;
          if (g >= P::STAGES && !mbar_wait(&empty[s], ((g / P::STAGES) - 1) & 1, abort_flag, args.err, 21)) {
            ok = false;
            break;
          }
          if (leader) mbar_expect_tx(&full[s], 2 * P::STAGE_BYTES);
          const uint32_t dst = smem_u32(smem + s * P::STAGE_BYTES);
          const uint32_t fb = full_leader + s * 8;
          const int k0 = kb * P::BK;
          tma_load_2d_pair(dst, &mapAh, fb, k0, m * TC_BM);
          tma_load_2d_pair(dst + P::A_BYTES, &mapAl, fb, k0, m * TC_BM);
          tma_load_3d_pair(dst + 2 * P::A_BYTES, &mapBh, fb, k0, nt * TC_BM + (TC_BM / 2) * (int)rank, w);
          tma_load_3d_pair(dst + 2 * P::A_BYTES + P::B_BYTES, &mapBl, fb, k0, nt * TC_BM + (TC_BM / 2) * (int)rank,
                           w);
        }
      }
      // The MMA commits of the last stages arrive on this CTA's empty[] too:
      // they have landed before the CTA leaves.
      for (int q = (g > P::STAGES ? g - P::STAGES : 0); q < g; ++q) {
        volatile int no_abort = 0;
        mbar_wait(&empty[q % P::STAGES], (q / P::STAGES) & 1, &no_abort, args.err, 22);
      }
    }
  } else if (warp == 1) {
    // ---------------- MMA issuer (even CTA) ----------------
    if (leader && lane == 0) {
      const uint32_t idesc = umma_idesc_f16(2 * TC_BM, TC_BM, args.fp16);
      int g = 0, u = 0;
      bool ok = true;
      for (int it = item0; it < n_items && ok; it += item_step) {
        for (int kb = 0; kb < k_blocks; ++kb, ++g) {
          const bool unit_start = kb % unit == 0;
          const bool unit_end = kb % unit == unit - 1 || kb == k_blocks - 1;
          const int buf = u % P::NBUF;
          if (unit_start && u >= P::NBUF &&
              !mbar_wait_cluster(&acc_empty[buf], ((u / P::NBUF) - 1) & 1, abort_flag, args.err, 23)) {
            ok = false;
            break;
          }
          const int s = g % P::STAGES;
          if (!mbar_wait(&full[s], (g / P::STAGES) & 1, abort_flag, args.err, 24)) {
            ok = false;
            break;
          }
          tc_fence_after();
          const uint32_t dacc = tmem_base + buf * TC_BM;
          const uint32_t ah = smem_u32(smem + s * P::STAGE_BYTES), al = ah + P::A_BYTES;
          const uint32_t bh = ah + 2 * P::A_BYTES, bl = bh + P::B_BYTES;
#pragma unroll
          for (int kk = 0; kk < P::BK / 16; ++kk) {
            const uint32_t off = kk * 32;
            const uint32_t acc0 = (!unit_start || kk > 0) ? 1u : 0u;
            umma_f16_pair(dacc, umma_desc<P::BK>(ah + off), umma_desc<P::BK>(bh + off), idesc, acc0);
            umma_f16_pair(dacc, umma_desc<P::BK>(ah + off), umma_desc<P::BK>(bl + off), idesc, 1u);
            umma_f16_pair(dacc, umma_desc<P::BK>(al + off), umma_desc<P::BK>(bh + off), idesc, 1u);
          }
          umma_commit_pair_both(&empty[s]);
          if (unit_end) {
            umma_commit_pair_both(&acc_full[buf]);
            ++u;
          }
        }
      }
      umma_commit_pair_own(drain);
      volatile int no_abort = 0;
      mbar_wait(drain, 0, &no_abort, args.err, 25);
    }
  } else {
    // ---------------- epilogue (warps 2..9, both CTAs) ----------------
    const int quarter = warp & 3;
    const int part = (warp - 2) >> 2;
    const int n_units = (k_blocks + unit - 1) / unit;
    bool ok = true;
    int u = 0;
    for (int it = item0; it < n_items; it += item_step) {
      int w, nt, mt;
      bool st;
      item_tile(it, w, nt, mt, st);
      const int m = mt * TC_BM + quarter * 32 + lane;
      const double unscale = 1.0 / ((double)args.scaleA[0] * (double)args.scaleB[w]);
      // Kahan-compensated FP32 sums of the FP32 accumulation units (sum
      // hs, compensation hc): four FP32 additions per value instead of an
      // FP32 -> FP64 conversion and an FP64 addition, whose throughput bounded
      // the drain.  The compensated sum is rounded once to FP32 at the end
      // (2^-24 relative), below the FP32 rounding inside one unit.
      float hs[P::CPW], hc[P::CPW];
#pragma unroll
      for (int c = 0; c < P::CPW; ++c) hs[c] = hc[c] = 0.0f;
      for (int uu = 0; uu < n_units; ++uu, ++u) {
        const int buf = u % P::NBUF;
        // After a failed wait a warp waits no more, but the odd CTA's warps
        // still pass the unit's named barrier together.
        const bool got = ok && mbar_wait(&acc_full[buf], (u / P::NBUF) & 1, abort_flag, args.err, 26);
        ok = got;
        if (got) {
          tc_fence_after();
          const uint32_t taddr = tmem_base + ((uint32_t)(quarter * 32) << 16) + buf * TC_BM + P::CPW * part;
#pragma unroll
          for (int j = 0; j < P::CPW / 16; ++j) {
            if (nt * TC_BM + P::CPW * part + 16 * j >= args.N) continue;  // warp-uniform
            float v[16];
            tmem_ld16(taddr + 16 * j, v);
#pragma unroll
            for (int q = 0; q < 16; ++q) {
              const int c = 16 * j + q;
              const float y = v[q] - hc[c];
              const float t = hs[c] + y;
              hc[c] = (t - hs[c]) - y;
              hs[c] = t;
            }
          }
          tc_fence_before();
        }
        if (leader) {
          __syncwarp();
          if (got && lane == 0) mbar_arrive(&acc_empty[buf]);
        } else {
          // The odd CTA's eight warps meet first, and one remote arrival
          // releases the buffer (a cluster-scope release per warp and unit
          // doubled the odd CTA's drain time).
          asm volatile("bar.sync 1, 256;\n" ::: "memory");
          if (got && warp == 2 && lane == 0) mbar_arrive_rank(&acc_empty[buf], 0);
        }
      }
      if (ok && st && m < args.M) {
        const int n0 = nt * TC_BM + P::CPW * part;
        double* out = args.out + (size_t)w * args.out_stride;
        double* orow = out + (size_t)m * args.ldo;
#pragma unroll
        for (int c = 0; c < P::CPW; ++c) {
          const int n = n0 + c;
          // The lower triangle and its mirror: the stored matrix is exactly symmetric.
          if (n < args.N && n <= m) {
            const double val = (double)(hs[c] - hc[c]) * unscale + ((args.add_identity && m == n) ? 1.0 : 0.0);
            orow[n] = val;
            if (n != m) out[(size_t)n * args.ldo + m] = val;
          }
        }
      }
    }
  }
  // Teardown: every warp of both CTAs reaches this point (all waits are
  // bounded); no remote arrival is still on its way to a CTA that leaves.
  tc_fence_before();
  __syncthreads();
  cluster_sync_all();
  tc_fence_after();
  if (warp == 1) {
    asm volatile("tcgen05.dealloc.cta_group::2.sync.aligned.b32 %0, %1;\n" ::"r"(tmem_base), "r"(P::NBUF * TC_BM));
  }
}

// P0 with the chi-scaled B operand materialised: one pass splits B_ov chi'_w
// s_w for every frequency (k_split8_bcast, 4 nw naux ldov bytes written),
// then the STORE GEMM reads both operands by TMA.
static void launch_p0_pair(qx_ctx* ctx, const CUtensorMap& ah, const CUtensorMap& al, const CUtensorMap& bh,
                           const CUtensorMap& bl, const TcArgs& a) {
  static PerDeviceOnce attr_once;
  static int max_clusters[PerDeviceOnce::kMaxDevices] = {};
  cudaLaunchConfig_t cfg = {};
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeClusterDimension;
  attr[0].val.clusterDim.x = 2;
  attr[0].val.clusterDim.y = 1;
  attr[0].val.clusterDim.z = 1;
  cfg.blockDim = dim3(pairp0::THREADS);
  cfg.dynamicSmemBytes = pairp0::TOTAL;
  cfg.stream = ctx->stream;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  attr_once(ctx->device, [&] {
    QX_CUDA(cudaFuncSetAttribute(k_p0_pair, cudaFuncAttributeMaxDynamicSharedMemorySize, pairp0::TOTAL));
    cfg.gridDim = dim3(2 * ctx->sm_count);
    int n = 0;
    QX_CUDA(cudaOccupancyMaxActiveClusters(&n, k_p0_pair, &cfg));
    max_clusters[ctx->device] = std::max(n, 1);
  });
  // Persistent: as many pairs as fit at once, each walking the pair items.
  const int items = p0_pair_count(a.m_blocks) * a.nbatch;
  cfg.gridDim = dim3(2 * std::min(items, max_clusters[ctx->device]));
  QX_CUDA(cudaLaunchKernelEx(&cfg, k_p0_pair, ah, al, bh, bl, a));
  check_launch(ctx);
}

static void eps_tc_split(qx_ctx* ctx, const double* bov, int ldov, int naux, int nov, const double* chi, int nw,
                         double* eps, int ldn, size_t eps_stride, int fp16, int reuse_a, bool pair) {
  constexpr int BN = 128;
  const size_t a_elems = (size_t)naux * ldov;
  DevBuf& buf = ctx->ws[WS_BOV_HI];
  const size_t need = a_elems * 2 * 2 * (1 + (size_t)nw);
  // The A split (and its scale in split slot 7) survive from the previous
  // call on this context only if the buffer is not reallocated now.
  reuse_a = reuse_a && buf.bytes >= need;
  buf.reserve(need);
  uint8_t* p = buf.as<uint8_t>();
  void* a_hi = p;
  void* a_lo = p + a_elems * 2;
  void* b_hi = p + a_elems * 4;
  void* b_lo = p + a_elems * 4 + a_elems * 2 * nw;
  float *sa = nullptr, *sb = nullptr;
  if (reuse_a)
    sa = split_scratch(ctx, 7).scale;
  else
    split(ctx, bov, naux, nov, ldov, 0, a_hi, a_lo, ldov, 0, 1, nullptr, 0, fp16, 7, &sa);
  split(ctx, bov, naux, nov, ldov, 0, b_hi, b_lo, ldov, a_elems, nw, chi, ldov, fp16, 1, &sb,
        /*the bound of bov*/ split_scratch(ctx, 7).amax_src);
  constexpr int BK = TcPipe<EPI_STORE>::BK;
  CUtensorMap ah = make_map(a_hi, nov, naux, ldov, 1, TC_BM, 2, fp16, BK);
  CUtensorMap al = make_map(a_lo, nov, naux, ldov, 1, TC_BM, 2, fp16, BK);
  // CTA pairs stage half of the B tile each.
  CUtensorMap bh = make_map(b_hi, nov, naux, ldov, nw, pair ? BN / 2 : BN, 3, fp16, BK);
  CUtensorMap bl = make_map(b_lo, nov, naux, ldov, nw, pair ? BN / 2 : BN, 3, fp16, BK);
  int* d_err = tc_err_slot(ctx);
  QX_CUDA(cudaMemsetAsync(d_err, 0, sizeof(int), ctx->stream));
  TcArgs a{};
  a.M = naux;
  a.N = naux;
  a.K = nov;
  a.nbatch = nw;
  a.m_blocks = ceil_div(naux, TC_BM);
  a.out = eps;
  a.ldo = ldn;
  a.out_stride = eps_stride;
  a.lower_tiles = 1;
  a.add_identity = 1;
  a.unit = kP0Unit;
  a.pair_units = 1;
  a.fp16 = fp16;
  a.scaleA = sa;
  a.scaleB = sb;
  a.err = d_err;
  const int tiles = ceil_div(naux, TC_BM);  // BM == BN for the symmetric product
  static_assert(BN == TC_BM, "eps tiles are square");
  if (pair) {
    launch_p0_pair(ctx, ah, al, bh, bl, a);
  } else {
    // Persistent: at most one CTA per SM over the (frequency, tile) items, in
    // tile-fastest order so that neighbouring CTAs share a frequency's operand.
    const int items = tiles * (tiles + 1) / 2 * nw;
    launch_tc<BN, EPI_STORE>(ctx, ah, al, bh, bl, a, dim3(std::min(items, ctx->sm_count)));
  }
  check_tc_err(ctx, d_err);
}

// P0 with chi applied while the B operand is staged (CONVB): no chi-scaled
// operand in memory at all.
static void eps_tc_conv(qx_ctx* ctx, const double* bov, int ldov, int naux, int nov, const double* chi, int nw,
                        double* eps, int ldn, size_t eps_stride, int fp16, int reuse_a) {
  constexpr int BN = 128;
  const size_t a_elems = (size_t)naux * ldov;
  // A: the hi/lo split of B_ov (one scale, slot 7), reusable across calls.
  // B: built in shared memory by the kernel's converter warps from an FP32
  // copy of B_ov and the per-frequency column scales chi' s_w, so that no
  // chi-scaled operand is written to memory.
  DevBuf& buf = ctx->ws[WS_BOV_HI];
  const size_t need = a_elems * 2 * 2 + a_elems * 4 + (size_t)nw * ldov * 4 + (size_t)nw * 4 + 1024;
  reuse_a = reuse_a && buf.bytes >= need;
  buf.reserve(need);
  uint8_t* p = buf.as<uint8_t>();
  void* a_hi = p;
  void* a_lo = p + a_elems * 2;
  float* bf = reinterpret_cast<float*>(p + a_elems * 4);
  float* cs = bf + a_elems;
  float* sb = cs + (size_t)nw * ldov;
  float* sa = nullptr;
  if (reuse_a) {
    sa = split_scratch(ctx, 7).scale;
  } else {
    split(ctx, bov, naux, nov, ldov, 0, a_hi, a_lo, ldov, 0, 1, nullptr, 0, fp16, 7, &sa);
    k_f32_rows<<<(unsigned)std::min<size_t>((a_elems + 255) / 256, 4 * (size_t)ctx->sm_count * 8), 256, 0,
                 ctx->stream>>>(bov, naux, nov, ldov, bf);
    check_launch(ctx);
  }
  k_chi_cols<<<nw, 256, 0, ctx->stream>>>(chi, nov, ldov, split_scratch(ctx, 7).amax_src, fp16, cs, sb);
  check_launch(ctx);
  constexpr int BK = TcPipe<EPI_STORE>::BK;
  CUtensorMap ah = make_map(a_hi, nov, naux, ldov, 1, TC_BM, 2, fp16, BK);
  CUtensorMap al = make_map(a_lo, nov, naux, ldov, 1, TC_BM, 2, fp16, BK);
  QX_REQUIRE(nov % 2 == 0 || ldov > nov, QX_ERR_INVALID_INPUT, "B_ov needs a padding column for odd nov");
  int* d_err = tc_err_slot(ctx);
  QX_CUDA(cudaMemsetAsync(d_err, 0, sizeof(int), ctx->stream));
  TcArgs a{};
  a.M = naux;
  a.N = naux;
  a.K = nov;
  a.nbatch = nw;
  a.m_blocks = ceil_div(naux, TC_BM);
  a.out = eps;
  a.ldo = ldn;
  a.out_stride = eps_stride;
  a.lower_tiles = 1;
  a.add_identity = 1;
  a.unit = kP0Unit;
  a.pair_units = 1;
  a.fp16 = fp16;
  a.scaleA = sa;
  a.scaleB = sb;
  a.err = d_err;
  a.convC = cs;
  a.ldcc = ldov;
  const int tiles = ceil_div(naux, TC_BM);  // BM == BN for the symmetric product
  static_assert(BN == TC_BM, "eps tiles are square");
  // The B slot carries the FP32 map of B_ov; the converters build hi/lo.
  const CUtensorMap bm = make_map_f32(bf, nov, naux, ldov, BN);
  launch_tc<BN, EPI_STORE, true>(ctx, ah, al, bm, bm, a, dim3(tiles * (tiles + 1) / 2, nw));
  check_tc_err(ctx, d_err);
}

void launch_eps_tc(qx_ctx* ctx, const double* bov, int ldov, int naux, int nov, const double* chi, int nw,
                   double* eps, int ldn, size_t eps_stride, int fp16, int reuse_a) {
  // The materialised form is the faster one wherever its chi-scaled operand
  // (4 nw naux ldov bytes) fits the budget; beyond it the converter form
  // keeps P0's memory at the A split and one FP32 copy of B_ov.
  const size_t chi_bytes = (size_t)4 * nw * naux * ldov;
  const bool materialise = ctx->p0_form == QX_P0_MATERIALISED || ctx->p0_form == QX_P0_PAIR ||
                           (ctx->p0_form == QX_P0_AUTO && chi_bytes <= kP0SplitBudget);
  if (materialise)
    eps_tc_split(ctx, bov, ldov, naux, nov, chi, nw, eps, ldn, eps_stride, fp16, reuse_a,
                 ctx->p0_form == QX_P0_PAIR);
  else
    eps_tc_conv(ctx, bov, ldov, naux, nov, chi, nw, eps, ldn, eps_stride, fp16, reuse_a);
}

// out[w][m][n] = sum_k A[m][k] B[w][n][k] in FP64 from split operands:
// A hi/lo [M][lda] (one scale), B hi/lo [nbatch][N][ldb] (a scale per batch).
void launch_gemm_tc(qx_ctx* ctx, const TcOperand& A, int M, int lda, const TcOperand& B, int N, int ldb, int K,
                    int nbatch, double* out, int ldo, size_t out_stride, int fp16) {
  constexpr int BN = 128;
  constexpr int BK = TcPipe<EPI_STORE>::BK;
  CUtensorMap ah = make_map(A.hi, K, M, lda, 1, TC_BM, 2, fp16, BK);
  CUtensorMap al = make_map(A.lo, K, M, lda, 1, TC_BM, 2, fp16, BK);
  CUtensorMap bh = make_map(B.hi, K, N, ldb, nbatch, BN, 3, fp16, BK);
  CUtensorMap bl = make_map(B.lo, K, N, ldb, nbatch, BN, 3, fp16, BK);
  int* d_err = tc_err_slot(ctx);
  QX_CUDA(cudaMemsetAsync(d_err, 0, sizeof(int), ctx->stream));
  TcArgs a{};
  a.M = M;
  a.N = N;
  a.K = K;
  a.nbatch = nbatch;
  a.m_blocks = ceil_div(M, TC_BM);
  a.out = out;
  a.ldo = ldo;
  a.out_stride = out_stride;
  a.lower_tiles = 0;
  a.add_identity = 0;
  a.fp16 = fp16;
  a.scaleA = A.scale;
  a.scaleB = B.scale;
  a.unit = kBseUnit;
  a.err = d_err;
  QX_REQUIRE(nbatch <= 65535, QX_ERR_INVALID_INPUT, "at most 65535 batches");
  launch_tc<BN, EPI_STORE>(ctx, ah, al, bh, bl, a, dim3(a.m_blocks * ceil_div(N, BN), nbatch));
  check_tc_err(ctx, d_err);
}

// Block sweep, FP16X3 trailing update.  The panels T = M[:, K] D and P = the
// old M[:, K] ([nw][n][128] FP64; T is zero past column kb, P is zero in the
// rows of K) are split into the half of `base` selected by buf, so that one
// step can be split while the previous step's update still runs on the other
// sweep stream; the scales go to split slots 3 + 2 buf (T) and 4 + 2 buf (P).
SweepSplit launch_sweep_split(qx_ctx* ctx, cudaStream_t st, const double* Tp, const double* Pp, int n, int kb,
                              int nw, int buf, void* base) {
  const size_t elems = (size_t)nw * n * kSweepPanelCols;
  const size_t ps = (size_t)n * kSweepPanelCols;
  uint8_t* b = static_cast<uint8_t*>(base) + (size_t)buf * elems * 2 * 4;
  SweepSplit sp;
  sp.T.hi = b;
  sp.T.lo = b + elems * 2;
  sp.P.hi = b + elems * 4;
  sp.P.lo = b + elems * 6;
  // The bounds of T and P were accumulated by the panel and write kernels.
  split(ctx, Tp, n, kb, kSweepPanelCols, ps, sp.T.hi, sp.T.lo, kSweepPanelCols, ps, nw, nullptr, 0, 1, 3 + 2 * buf,
        &sp.T.scale, split_amax_words(ctx, 3 + 2 * buf), st);
  split(ctx, Pp, n, kb, kSweepPanelCols, ps, sp.P.hi, sp.P.lo, kSweepPanelCols, ps, nw, nullptr, 0, 1, 4 + 2 * buf,
        &sp.P.scale, split_amax_words(ctx, 4 + 2 * buf), st);
  return sp;
}

// M[w][r][c] -= sum_q T[w][r][q] P[w][c][q] on stream st over the lower
// 128 x 128 tiles outside tile row/column kblk (the K block), mirrored;
// mode / next_blk select the look-ahead subset (filter_mode of TcArgs).  err
// is one status word, zero on entry.
void launch_sweep_update_tc(qx_ctx* ctx, cudaStream_t st, double* eps, int n, int ldn, size_t stride, int nw,
                            int kblk, const SweepSplit& sp, int mode, int next_blk, int* err) {
  static_assert(kSweepPanelCols == TC_BM, "sweep block = tcgen05 tile");
  constexpr int BN = 128;
  constexpr int BK = TcPipe<EPI_UPDATE>::BK;
  const int K = kSweepPanelCols;
  CUtensorMap ah = make_map(sp.T.hi, K, n, K, nw, TC_BM, 3, 1, BK);
  CUtensorMap al = make_map(sp.T.lo, K, n, K, nw, TC_BM, 3, 1, BK);
  CUtensorMap bh = make_map(sp.P.hi, K, n, K, nw, BN, 3, 1, BK);
  CUtensorMap bl = make_map(sp.P.lo, K, n, K, nw, BN, 3, 1, BK);
  TcArgs a{};
  a.M = n;
  a.N = n;
  a.K = K;
  a.nbatch = nw;
  a.m_blocks = ceil_div(n, TC_BM);
  a.out = eps;
  a.ldo = ldn;
  a.out_stride = stride;
  a.lower_tiles = 1;
  a.subtract = 1;
  a.a_batched = 1;
  a.unit = kUpdateUnit;
  a.fp16 = 1;
  a.scaleA = sp.T.scale;
  a.scaleB = sp.P.scale;
  a.err = err;
  a.skip_tile = kblk;
  a.filter_mode = mode;
  a.filter_tile = next_blk;
  const int tiles = ceil_div(n, TC_BM);
  static_assert(kSweepPanelCols <= kUpdateUnit * TcPipe<EPI_UPDATE>::BK, "one accumulation unit covers the panel");
  QX_REQUIRE(nw <= 65535, QX_ERR_INVALID_INPUT, "at most 65535 matrices per sweep");
  launch_tc<BN, EPI_UPDATE>(ctx, ah, al, bh, bl, a, dim3(tiles * (tiles + 1) / 2, nw), st);
}

void launch_gsweep_update_tc(qx_ctx* ctx, const GMat* d_mats, const int* d_pre, int count, int ntiles, int step,
                             const TcOperand& T, const TcOperand& P, int rows, int* err) {
  constexpr int BN = 128;
  constexpr int BK = TcPipe<EPI_GUPDATE>::BK;
  const int K = kSweepPanelCols;
  CUtensorMap ah = make_map(T.hi, K, rows, K, 1, TC_BM, 2, 1, BK);
  CUtensorMap al = make_map(T.lo, K, rows, K, 1, TC_BM, 2, 1, BK);
  CUtensorMap bh = make_map(P.hi, K, rows, K, 1, BN, 3, 1, BK);
  CUtensorMap bl = make_map(P.lo, K, rows, K, 1, BN, 3, 1, BK);
  TcArgs a{};
  a.K = K;
  a.nbatch = 1;
  a.lower_tiles = 1;
  a.subtract = 1;
  a.fp16 = 1;
  a.unit = kUpdateUnit;
  a.scaleA = T.scale;
  a.scaleB = P.scale;
  a.err = err;
  a.skip_tile = step;
  a.gmats = d_mats;
  a.gpre = d_pre;
  a.gcount = count;
  a.items = ntiles;
  // Persistent: one CTA per SM walks the tiles of all matrices, so that the
  // loads and MMAs of its next tile run under the read-modify-write of this
  // one (the update is bound by that HBM traffic), with the two-group
  // epilogue.
  launch_tc<BN, EPI_GUPDATE>(ctx, ah, al, bh, bl, a, dim3(std::min(ntiles, ctx->sm_count)));
}

}  // namespace qx
