// Guarded eps inversion: pivot and growth checks around the block sweep, and
// the pivoted re-inversion of the matrices they flag.
//
// The block sweep (k_gw_f64.cu) is Gauss-Jordan elimination without pivoting.
// It is stable when eps >= I -- the imaginary axis with every occupied level
// below every virtual one, or real shifts below the smallest transition --
// and the callers that can show this run it unguarded.  Otherwise eps may be
// indefinite with a tiny or zero leading minor while still nonsingular, and
// the reference would then take its LU fallback: `invc` (Cholesky) fails and
// `inv` (LAPACK dgetrf/dgetri, partial pivoting) inverts it
// (quasix_core/src/selfenergy/correlation_ac.rs:383-399; the CD path calls
// `inv` directly, selfenergy/correlation_pyscf_cd.rs:126-159).
//
// A guarded inversion therefore
//   1. copies each eps aside and records amax = max |eps| (k_guard_backup);
//   2. sweeps, flagging a matrix whose pivot is below kGuardPivot * amax or
//      whose not-yet-swept entries grow past kGuardGrowth * amax;
//   2b. checks every result against its copy with one probe vector v of
//      +-1 entries: eta = max|eps X v - v| / (n amax max|X|) is the normwise
//      backward error of X in the direction v, ~1e-17 for a stable inverse
//      whatever the conditioning, and it exceeds kGuardResidual when the
//      unpivoted elimination lost digits to element growth that the pivot
//      and growth checks did not see;
//   3. re-inverts every flagged matrix from its copy by Gauss-Jordan
//      elimination with partial (row) pivoting, in super-panels of PIV_SB
//      columns, each worked as panels of PIV_NB (k_piv_panel: the pivoted
//      exchanges on a panel, one CTA per matrix; k_piv_update on the rest of
//      the super-panel); the columns outside the super-panel then take one
//      rank-PIV_SB update on DMMA tiles (k_piv_update with the super-panel's
//      pivot rows as they were before it, k_piv_gather), because consecutive
//      exchange steps compose: with C = A[:, panel](new) R^T, R the panel's
//      old pivot rows, a pivot row of the panel becomes -C and any other row
//      A - C, for any panel width.  k_piv_permute finally undoes the pivot
//      permutation into -eps^-1, the sweep's own output convention.
// A zero or non-finite pivot in step 3 leaves the matrix flagged singular
// (Wc = 0, the reference's identity fallback after a failed LU).
#include <algorithm>
#include <climits>

#include "gemm_f64.cuh"
#include "qx_internal.cuh"

namespace qx {

namespace {

constexpr int PIV_NB = 16;
// Super-panel width: one DMMA column tile, so the rank-PIV_SB update skips
// exactly the super-panel's own tile.
constexpr int PIV_SB = 64;
// Rows of a panel held in shared memory ([n][PIV_NB] doubles plus n row states).
constexpr int kPivSmemRows = 1700;
constexpr size_t kPivSmemBytes = (size_t)kPivSmemRows * (PIV_NB * sizeof(double) + sizeof(int)) + 1024;
using PivTile = F64Tile<64, 64, 2, 2, 3>;
static_assert(PivTile::BN == PIV_SB && PIV_SB % PIV_NB == 0, "a super-panel is one column tile of whole panels");

// Block-wide argmax of (v, r): largest v, ties to the smallest r (every
// thread calls it; the result is returned to all threads).
__device__ __forceinline__ void block_argmax(double& v, int& r, double* sv, int* sr) {
  for (int o = 16; o > 0; o >>= 1) {
    const double ov = __shfl_xor_sync(0xffffffffu, v, o);
    const int orr = __shfl_xor_sync(0xffffffffu, r, o);
    if (ov > v || (ov == v && orr < r)) {
      v = ov;
      r = orr;
    }
  }
  const int warp = threadIdx.x >> 5, nwarp = blockDim.x >> 5;
  __syncthreads();
  if ((threadIdx.x & 31) == 0) {
    sv[warp] = v;
    sr[warp] = r;
  }
  __syncthreads();
  v = sv[0];
  r = sr[0];
  for (int k = 1; k < nwarp; ++k)
    if (sv[k] > v || (sv[k] == v && sr[k] < r)) {
      v = sv[k];
      r = sr[k];
    }
}

__device__ __forceinline__ void atomic_max_abs(unsigned long long* out, double m) {
  // m >= 0 compares as its bit pattern.
  atomicMax(out, (unsigned long long)__double_as_longlong(m));
}

// bk = M over the n x n part, amax[idx] = max |M|.  grid (count, y).
__global__ void k_guard_backup(const GuardMat* __restrict__ tab, unsigned long long* __restrict__ amax) {
  const GuardMat g = tab[blockIdx.x];
  double m = 0.0;
  const size_t total = (size_t)g.n * g.n;
  for (size_t e = (size_t)blockIdx.y * blockDim.x + threadIdx.x; e < total; e += (size_t)gridDim.y * blockDim.x) {
    const size_t r = e / g.n, c = e % g.n;
    const double v = g.M[r * g.ldn + c];
    g.bk[r * g.ldn + c] = v;
    m = fmax(m, fabs(v));
    if (!isfinite(v)) m = INFINITY;
  }
  __shared__ double red[32];
  for (int o = 16; o > 0; o >>= 1) m = fmax(m, __shfl_xor_sync(0xffffffffu, m, o));
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = m;
  __syncthreads();
  if (threadIdx.x < 32) {
    m = threadIdx.x < (blockDim.x >> 5) ? red[threadIdx.x] : 0.0;
    for (int o = 16; o > 0; o >>= 1) m = fmax(m, __shfl_xor_sync(0xffffffffu, m, o));
    if (threadIdx.x == 0) atomic_max_abs(amax + g.idx, m);
  }
}

// Entry j of the probe vector: +-1 from a fixed integer hash of j.
__device__ __forceinline__ double probe_entry(int j) {
  unsigned h = (unsigned)j * 2654435761u;
  h ^= h >> 15;
  h *= 2246822519u;
  h ^= h >> 13;
  return (h & 1u) ? 1.0 : -1.0;
}

// y = X v with X = -M (the sweep's output is -eps^-1), xmax[idx] = max |X|.
// One warp per row; y in rbuf.  grid (count, y).
__global__ void k_guard_probe_xv(const GuardMat* __restrict__ tab, unsigned long long* __restrict__ xmax) {
  const GuardMat g = tab[blockIdx.x];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarp = blockDim.x >> 5;
  double mx = 0.0;
  for (int i = blockIdx.y * nwarp + warp; i < g.n; i += gridDim.y * nwarp) {
    const double* row = g.M + (size_t)i * g.ldn;
    double s = 0.0;
    for (int j = lane; j < g.n; j += 32) {
      const double x = -row[j];
      s += x * probe_entry(j);
      mx = fmax(mx, isfinite(x) ? fabs(x) : INFINITY);
    }
    for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    if (lane == 0) g.rbuf[i] = s;
  }
  for (int o = 16; o > 0; o >>= 1) mx = fmax(mx, __shfl_xor_sync(0xffffffffu, mx, o));
  if (lane == 0) atomic_max_abs(xmax + g.idx, mx);
}

// rmax[idx] = max_i |(eps y)_i - v_i| with eps the copy bk.  grid (count, y).
__global__ void k_guard_probe_res(const GuardMat* __restrict__ tab, unsigned long long* __restrict__ rmax) {
  const GuardMat g = tab[blockIdx.x];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarp = blockDim.x >> 5;
  double mx = 0.0;
  for (int i = blockIdx.y * nwarp + warp; i < g.n; i += gridDim.y * nwarp) {
    const double* row = g.bk + (size_t)i * g.ldn;
    double s = 0.0;
    for (int j = lane; j < g.n; j += 32) s += row[j] * g.rbuf[j];
    for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    const double r = s - probe_entry(i);
    mx = fmax(mx, isfinite(r) ? fabs(r) : INFINITY);
  }
  if (lane == 0) atomic_max_abs(rmax + g.idx, mx);
}

// Row state (-1: not yet a pivot row) for every flagged matrix; status
// cleared (the fallback decides it anew).
__global__ void k_piv_init(const GuardMat* __restrict__ tab) {
  const GuardMat g = tab[blockIdx.x];
  for (int r = threadIdx.x; r < g.n; r += blockDim.x) g.ints[r] = -1;
  if (threadIdx.x == 0) *g.status = 0;
}

// Panel [k0, k0 + kb) of the pivoted Gauss-Jordan exchange on bk, one CTA of
// 512 threads per matrix.  Exchange on pivot (p, c), d = T[p][c]:
//   T[p][c] = 1/d, T[p][j] = -T[p][j]/d, T[i][c] = T[i][c]/d,
//   T[i][j] -= T[i][c] T[p][j]/d        (i != p, j != c),
// applied here to the panel columns only (they depend on nothing else).  The
// pivot row of column c is the unused row of largest |T[r][c]| (ties to the
// lowest row).  SMEM: the panel and the row states sit in shared memory for
// the kb steps (n <= kPivSmemRows); otherwise every step works on bk itself.
// Each half-warp holds one row, a lane one column.  Afterwards rbuf[j][b] =
// the old row piv[k0 + b] outside the panel (zero inside), the operand of the
// update of the other columns.
template <bool SMEM>
__global__ void __launch_bounds__(512) k_piv_panel(const GuardMat* __restrict__ tab, int k0) {
  const GuardMat g = tab[blockIdx.x];
  const int n = g.n;
  if (k0 >= n || *g.status != 0) return;
  const int kb = min(PIV_NB, n - k0), lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int nwarp = blockDim.x >> 5;
  const int half = lane >> 4, col = lane & 15;
  int* gstate = g.ints;
  int* piv = g.ints + n;
  extern __shared__ __align__(16) uint8_t pan_smem[];
  double* P;  // panel element (r, c) at P[r * pld + c]
  int* state;
  size_t pld;
  if (SMEM) {
    P = reinterpret_cast<double*>(pan_smem);
    state = reinterpret_cast<int*>(P + (size_t)n * PIV_NB);
    pld = PIV_NB;
    for (int e = threadIdx.x; e < n * PIV_NB; e += blockDim.x) {
      const int r = e / PIV_NB, c = e % PIV_NB;
      P[e] = c < kb ? g.bk[(size_t)r * g.ldn + k0 + c] : 0.0;
    }
    for (int r = threadIdx.x; r < n; r += blockDim.x) state[r] = gstate[r];
    __syncthreads();
  } else {
    P = g.bk + k0;
    state = gstate;
    pld = g.ldn;
  }
  __shared__ double prow[PIV_NB];
  __shared__ double sv[32];
  __shared__ int sr[32];
  // Candidate pivot of the panel's first column.
  double best = -1.0;
  int bi = INT_MAX;
  for (int r = threadIdx.x; r < n; r += blockDim.x)
    if (state[r] < 0) {
      const double v = fabs(P[(size_t)r * pld]);
      if (v > best || (v == best && r < bi)) {
        best = v;
        bi = r;
      }
    }
  for (int j = 0; j < kb; ++j) {
    block_argmax(best, bi, sv, sr);
    const int p = bi;
    const double d = (p == INT_MAX) ? 0.0 : P[(size_t)p * pld + j];
    if (!(fabs(d) > 0.0) || !isfinite(d)) {  // uniform: p and d are the same in every thread
      if (threadIdx.x == 0) *g.status = 1;
      return;
    }
    if (threadIdx.x < PIV_NB) prow[threadIdx.x] = threadIdx.x < kb ? P[(size_t)p * pld + threadIdx.x] : 0.0;
    __syncthreads();
    if (threadIdx.x == 0) {
      state[p] = k0;
      piv[k0 + j] = p;
    }
    const double inv = 1.0 / d;
    best = -1.0;
    bi = INT_MAX;
    // Row r of this half-warp (the loop bound is warp-uniform: both halves
    // run every iteration, a half past n holding a dummy row).
    for (int r0 = 2 * warp; r0 < n; r0 += 2 * nwarp) {
      const int r = r0 + half;
      const bool live = r < n;
      double* row = P + (size_t)(live ? r : 0) * pld;
      double v = (live && col < kb) ? row[col] : 0.0;
      const double arj = __shfl_sync(0xffffffffu, v, (lane & 16) | j);
      if (r == p) {
        v = (col == j) ? inv : -prow[col] * inv;
      } else {
        const double t = arj * inv;
        v = (col == j) ? t : v - t * prow[col];
      }
      if (live && col < kb) row[col] = v;
      if (j + 1 < kb) {
        const double cv = fabs(__shfl_sync(0xffffffffu, v, (lane & 16) | (j + 1)));
        if (live && r != p && state[r] < 0 && (cv > best || (cv == best && r < bi))) {
          best = cv;
          bi = r;
        }
      }
    }
    __syncthreads();
  }
  if (SMEM) {
    for (int e = threadIdx.x; e < n * PIV_NB; e += blockDim.x) {
      const int r = e / PIV_NB, c = e % PIV_NB;
      if (c < kb) g.bk[(size_t)r * g.ldn + k0 + c] = P[e];
    }
    for (int r = threadIdx.x; r < n; r += blockDim.x) gstate[r] = state[r];
  }
}

// k_piv_panel with the panel in registers, for n <= 512 RPT, and the rest of
// its super-panel updated in the same kernel.  Thread t holds rows t + 512 i
// (i < RPT) across all PIV_NB columns.  A pivot step takes one block barrier:
// every warp reduces its candidates by shuffles and the lane owning the
// warp's best row publishes that row (value, index and its PIV_NB entries) in
// the warp's slot; after the barrier every thread picks the best slot (ties
// to the lowest row) and applies the exchange in registers.  The slots
// alternate between steps, so a slot is rewritten only after a barrier that
// follows every read of it.  The arithmetic is k_piv_panel's, operation for
// operation.  It also leaves in rbuf the old pivot rows of the super-panel's
// other columns (k_piv_gather's job for the other panel kernels), read only
// after the panel is written back: the panel's own columns are zero there.
template <int RPT>
__global__ void __launch_bounds__(512) k_piv_panel_reg(const GuardMat* __restrict__ tab, int k0) {
  constexpr int NWARP = 16;
  const GuardMat g = tab[blockIdx.x];
  const int n = g.n;
  if (k0 >= n || *g.status != 0) return;
  const int kb = min(PIV_NB, n - k0);
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  int* gstate = g.ints;
  int* piv = g.ints + n;
  __shared__ double slot_row[2][NWARP][PIV_NB];
  __shared__ double slot_val[2][NWARP];
  __shared__ int slot_idx[2][NWARP];
  __shared__ int pivs[PIV_NB];
  double v[RPT][PIV_NB];
  bool freer[RPT], mine[RPT];
#pragma unroll
  for (int i = 0; i < RPT; ++i) {
    const int r = threadIdx.x + 512 * i;
    const bool live = r < n;
    freer[i] = live && gstate[r] < 0;
    mine[i] = false;
    const double* src = g.bk + (size_t)(live ? r : 0) * g.ldn + k0;
    if (live && kb == PIV_NB && (g.ldn & 1) == 0) {
      // bk is 256-byte aligned, k0 a multiple of 16 and ldn even: 16-byte pairs.
#pragma unroll
      for (int c = 0; c < PIV_NB; c += 2) {
        const double2 x = __ldg(reinterpret_cast<const double2*>(src + c));
        v[i][c] = x.x;
        v[i][c + 1] = x.y;
      }
    } else {
#pragma unroll
      for (int c = 0; c < PIV_NB; ++c) v[i][c] = (live && c < kb) ? src[c] : 0.0;
    }
  }
  // This thread's candidate for column 0.
  double best = -1.0;
  int bi = INT_MAX;
#pragma unroll
  for (int i = 0; i < RPT; ++i) {
    const int r = threadIdx.x + 512 * i;
    const double a = fabs(v[i][0]);
    if (freer[i] && (a > best || (a == best && r < bi))) {
      best = a;
      bi = r;
    }
  }
  // Four pivot steps per loop iteration, then the registers rotate by four
  // columns, so that step s of an iteration works on column s and every
  // register index stays a compile-time constant.  (Sixteen unrolled steps
  // missed the instruction cache -- "no instruction" was the top stall --
  // and one step per iteration spent 32 register moves per row and pivot on
  // the rotation.)  Steps past kb only rotate.
  constexpr int UNR = 4;
  static_assert(PIV_NB % UNR == 0, "whole rotations");
#pragma unroll 1
  for (int j4 = 0; j4 < PIV_NB; j4 += UNR) {
#pragma unroll
    for (int s = 0; s < UNR; ++s) {
      const int j = j4 + s;
      if (j < kb) {  // uniform
        const int sl = j & 1;
        // Warp argmax, then the owner of the warp's best row publishes it.
        double wv = best;
        int wr = bi;
        for (int o = 16; o > 0; o >>= 1) {
          const double ov = __shfl_xor_sync(0xffffffffu, wv, o);
          const int orr = __shfl_xor_sync(0xffffffffu, wr, o);
          if (ov > wv || (ov == wv && orr < wr)) {
            wv = ov;
            wr = orr;
          }
        }
        if (lane == 0) {
          slot_val[sl][warp] = wv;
          slot_idx[sl][warp] = wr;
        }
#pragma unroll
        for (int i = 0; i < RPT; ++i)
          if (wr != INT_MAX && threadIdx.x + 512 * i == wr) {
#pragma unroll
            for (int c = 0; c < PIV_NB; ++c) slot_row[sl][warp][c] = v[i][c];
          }
        __syncthreads();
        // Block argmax over the warps' slots: lane k < NWARP holds slot k,
        // a shuffle tree picks the largest value (ties to the lowest row),
        // and lane 0's result goes to the whole warp.
        double gv = lane < NWARP ? slot_val[sl][lane] : -2.0;
        int gr = lane < NWARP ? slot_idx[sl][lane] : INT_MAX;
        int gw = lane;
        for (int o = NWARP / 2; o > 0; o >>= 1) {
          const double ov = __shfl_xor_sync(0xffffffffu, gv, o);
          const int orr = __shfl_xor_sync(0xffffffffu, gr, o);
          const int ow = __shfl_xor_sync(0xffffffffu, gw, o);
          if (ov > gv || (ov == gv && orr < gr)) {
            gv = ov;
            gr = orr;
            gw = ow;
          }
        }
        gr = __shfl_sync(0xffffffffu, gr, 0);
        gw = __shfl_sync(0xffffffffu, gw, 0);
        const int p = gr;
        const double d = (p == INT_MAX) ? 0.0 : slot_row[sl][gw][s];
        if (!(fabs(d) > 0.0) || !isfinite(d)) {  // uniform
          if (threadIdx.x == 0) *g.status = 1;
          return;
        }
        if (threadIdx.x == 0) {
          piv[k0 + j] = p;
          pivs[j] = p;
        }
        const double inv = 1.0 / d;
        double pr[PIV_NB];
#pragma unroll
        for (int c = 0; c < PIV_NB; ++c) pr[c] = slot_row[sl][gw][c];
        best = -1.0;
        bi = INT_MAX;
#pragma unroll
        for (int i = 0; i < RPT; ++i) {
          const int r = threadIdx.x + 512 * i;
          if (r == p) {
#pragma unroll
            for (int c = 0; c < PIV_NB; ++c) v[i][c] = (c == s) ? inv : -pr[c] * inv;
            freer[i] = false;
            mine[i] = true;
          } else {
            const double t = v[i][s] * inv;
#pragma unroll
            for (int c = 0; c < PIV_NB; ++c) v[i][c] = (c == s) ? t : v[i][c] - t * pr[c];
          }
          // The next step's column is v[.][s + 1] (before the rotation below).
          const double a = fabs(v[i][s + 1]);
          if (freer[i] && (a > best || (a == best && r < bi))) {
            best = a;
            bi = r;
          }
        }
      }
    }
#pragma unroll
    for (int i = 0; i < RPT; ++i) {
      double t0[UNR];
#pragma unroll
      for (int c = 0; c < UNR; ++c) t0[c] = v[i][c];
#pragma unroll
      for (int c = 0; c + UNR < PIV_NB; ++c) v[i][c] = v[i][c + UNR];
#pragma unroll
      for (int c = 0; c < UNR; ++c) v[i][PIV_NB - UNR + c] = t0[c];
    }
  }
  // Write the panel back, then the old pivot rows of the super-panel's other
  // columns into rbuf (zero inside the panel) for k_piv_update.
#pragma unroll
  for (int i = 0; i < RPT; ++i) {
    const int r = threadIdx.x + 512 * i;
    if (r >= n) continue;
    double* row = g.bk + (size_t)r * g.ldn + k0;
    if (kb == PIV_NB && (g.ldn & 1) == 0) {
#pragma unroll
      for (int c = 0; c < PIV_NB; c += 2) *reinterpret_cast<double2*>(row + c) = make_double2(v[i][c], v[i][c + 1]);
    } else {
#pragma unroll
      for (int c = 0; c < PIV_NB; ++c)
        if (c < kb) row[c] = v[i][c];
    }
    if (mine[i]) gstate[r] = k0;
  }
  const int ks = (k0 / PIV_SB) * PIV_SB, ce = min(ks + PIV_SB, n);
  __syncthreads();  // pivs complete
  for (int e = threadIdx.x; e < PIV_NB * PIV_SB; e += blockDim.x) {
    const int b = e / PIV_SB, c = ks + e % PIV_SB;
    if (b < kb && c < ce)
      g.rbuf[(size_t)c * PIV_SB + b] = (c >= k0 && c < k0 + kb) ? 0.0 : g.bk[(size_t)pivs[b] * g.ldn + c];
  }
}

// rbuf[c][b] = A[piv[k0 + b]][c] (row stride PIV_SB) for the columns c in
// [c_lo, min(c_hi, n)), zero inside [k0, k0 + kb): the old pivot rows of a
// panel (kbmax = PIV_NB) or of a super-panel (kbmax = PIV_SB), read before
// the update that consumes them.  One warp per pivot row.  grid (count, y).
__global__ void k_piv_gather(const GuardMat* __restrict__ tab, int k0, int kbmax, int c_lo, int c_hi) {
  const GuardMat g = tab[blockIdx.x];
  const int n = g.n;
  if (k0 >= n || *g.status != 0) return;
  const int kb = min(kbmax, n - k0), lane = threadIdx.x & 31;
  const int* piv = g.ints + n;
  const int ch = min(c_hi, n);
  for (int b = blockIdx.y * (blockDim.x >> 5) + (threadIdx.x >> 5); b < kb; b += gridDim.y * (blockDim.x >> 5)) {
    const double* src = g.bk + (size_t)piv[k0 + b] * g.ldn;
    for (int c = c_lo + lane; c < ch; c += 32)
      g.rbuf[(size_t)c * PIV_SB + b] = (c >= k0 && c < k0 + kb) ? 0.0 : src[c];
  }
}

// Columns c in [c_lo, min(c_hi, n)) outside the panel [k0, k0 + kb),
// kb = min(kbmax, n - k0): with C = A[:, panel] (new) rbuf^T,
//   A[r][c] = -C[r][c]         for the panel's pivot rows r (state in [pr_lo, pr_hi)),
//   A[r][c] -= C[r][c]         otherwise.
// grid (column tiles of [c_lo, c_hi), row tiles, count).
__global__ void __launch_bounds__(PivTile::THREADS)
    k_piv_update(const GuardMat* __restrict__ tab, int k0, int kbmax, int c_lo, int c_hi, int pr_lo, int pr_hi) {
  using T = PivTile;
  const GuardMat g = tab[blockIdx.z];
  const int n = g.n;
  if (k0 >= n || *g.status != 0) return;
  const int kb = min(kbmax, n - k0);
  const int ch = min(c_hi, n);
  const int m0 = blockIdx.y * T::BM, n0 = c_lo + blockIdx.x * T::BN;
  if (m0 >= n || n0 >= ch) return;
  if (n0 >= k0 && n0 + T::BN <= k0 + kb) return;
  extern __shared__ double smem[];
  double acc[T::MI][T::NJ][2];
#pragma unroll
  for (int i = 0; i < T::MI; ++i)
#pragma unroll
    for (int j = 0; j < T::NJ; ++j) acc[i][j][0] = acc[i][j][1] = 0.0;
  const size_t ld = g.ldn;
  f64_mainloop<T>(acc, smem, g.bk + (size_t)m0 * ld + k0, (int)ld, n - m0, g.rbuf + (size_t)n0 * PIV_SB, PIV_SB,
                  ch - n0, nullptr, kb);
  const int* state = g.ints;
#pragma unroll
  for (int i = 0; i < T::MI; ++i) {
    const int r = m0 + f64_row<T>(i);
    if (r >= n) continue;
    const bool prow = state[r] >= pr_lo && state[r] < pr_hi;
#pragma unroll
    for (int j = 0; j < T::NJ; ++j)
#pragma unroll
      for (int e = 0; e < 2; ++e) {
        const int c = n0 + f64_col<T>(j, e);
        if (c >= ch || (c >= k0 && c < k0 + kb)) continue;
        double* a = g.bk + (size_t)r * ld + c;
        *a = prow ? -acc[i][j][e] : *a - acc[i][j][e];
      }
  }
}

// pinv[piv[b]] = b.
__global__ void k_piv_inverse_perm(const GuardMat* __restrict__ tab) {
  const GuardMat g = tab[blockIdx.x];
  if (*g.status != 0) return;
  for (int b = threadIdx.x; b < g.n; b += blockDim.x) g.ints[2 * g.n + g.ints[g.n + b]] = b;
}

// After every exchange the element at (piv[a], b) is (eps^-1)[a][piv[b]], so
// M[a][c] = -bk[piv[a]][pinv[c]] is the sweep's -eps^-1.  grid (n, count).
__global__ void k_piv_permute(const GuardMat* __restrict__ tab) {
  const GuardMat g = tab[blockIdx.y];
  const int a = blockIdx.x;
  if (a >= g.n || *g.status != 0) return;
  const int* piv = g.ints + g.n;
  const int* pinv = g.ints + 2 * g.n;
  const double* src = g.bk + (size_t)piv[a] * g.ldn;
  double* dst = g.M + (size_t)a * g.ldn;
  for (int c = threadIdx.x; c < g.n; c += blockDim.x) dst[c] = -src[pinv[c]];
}

inline size_t align256(size_t b) { return (b + 255) & ~size_t(255); }

}  // namespace

size_t guard_bytes(int n, int ldn, int count) {
  const size_t per = align256((size_t)n * ldn * sizeof(double)) + align256((size_t)3 * n * sizeof(int)) +
                     align256((size_t)n * PIV_SB * sizeof(double));
  return per * count + align256(count * sizeof(GuardMat)) + 4 * align256(count * sizeof(unsigned long long)) + 256;
}

void guard_layout(GuardSet& gs, void* mem, size_t bytes) {
  size_t need = align256(gs.mats.size() * sizeof(GuardMat)) + 4 * align256(gs.nall * sizeof(unsigned long long));
  for (const GuardMat& g : gs.mats)
    need += align256((size_t)g.n * g.ldn * sizeof(double)) + align256((size_t)3 * g.n * sizeof(int)) +
            align256((size_t)g.n * PIV_SB * sizeof(double));
  QX_REQUIRE(need <= bytes, QX_ERR_INVALID_INPUT, "guarded inversion needs %zu bytes of workspace, have %zu", need,
             bytes);
  char* p = static_cast<char*>(mem);
  gs.d_tab = reinterpret_cast<GuardMat*>(p);
  p += align256(gs.mats.size() * sizeof(GuardMat));
  gs.amax = reinterpret_cast<unsigned long long*>(p);
  p += align256(gs.nall * sizeof(unsigned long long));
  gs.growth = reinterpret_cast<unsigned long long*>(p);
  p += align256(gs.nall * sizeof(unsigned long long));
  gs.xmax = reinterpret_cast<unsigned long long*>(p);
  p += align256(gs.nall * sizeof(unsigned long long));
  gs.rmax = reinterpret_cast<unsigned long long*>(p);
  p += align256(gs.nall * sizeof(unsigned long long));
  for (GuardMat& g : gs.mats) {
    g.bk = reinterpret_cast<double*>(p);
    p += align256((size_t)g.n * g.ldn * sizeof(double));
    g.ints = reinterpret_cast<int*>(p);
    p += align256((size_t)3 * g.n * sizeof(int));
    g.rbuf = reinterpret_cast<double*>(p);
    p += align256((size_t)g.n * PIV_SB * sizeof(double));
  }
}

void guard_begin(qx_ctx* ctx, GuardSet& gs) {
  if (gs.mats.empty()) return;
  static PerDeviceOnce attr_once;
  attr_once(ctx->device, [] {
    QX_CUDA(cudaFuncSetAttribute(k_piv_update, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)PivTile::SMEM));
    QX_CUDA(cudaFuncSetAttribute(k_piv_panel<true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)kPivSmemBytes));
  });
  QX_CUDA(cudaMemsetAsync(gs.amax, 0, gs.nall * sizeof(unsigned long long), ctx->stream));
  QX_CUDA(cudaMemsetAsync(gs.growth, 0, gs.nall * sizeof(unsigned long long), ctx->stream));
  QX_CUDA(cudaMemsetAsync(gs.xmax, 0, gs.nall * sizeof(unsigned long long), ctx->stream));
  QX_CUDA(cudaMemsetAsync(gs.rmax, 0, gs.nall * sizeof(unsigned long long), ctx->stream));
  QX_CUDA(cudaMemcpyAsync(gs.d_tab, gs.mats.data(), gs.mats.size() * sizeof(GuardMat), cudaMemcpyHostToDevice,
                          ctx->stream));
  int nmax = 0;
  for (const GuardMat& g : gs.mats) nmax = std::max(nmax, g.n);
  dim3 grid((unsigned)gs.mats.size(), std::max(1, std::min(ceil_div(nmax * nmax, 256 * 8), 512)));
  k_guard_backup<<<grid, 256, 0, ctx->stream>>>(gs.d_tab, gs.amax);
  check_launch(ctx);
}

int guard_end(qx_ctx* ctx, GuardSet& gs) {
  if (gs.mats.empty()) return 0;
  const int G = (int)gs.mats.size();
  // Probe residual of every result against its copy.
  int nmax = 0;
  for (const GuardMat& g : gs.mats) nmax = std::max(nmax, g.n);
  const dim3 pg((unsigned)G, std::max(1, std::min(ceil_div(nmax, 8), 64)));
  k_guard_probe_xv<<<pg, 256, 0, ctx->stream>>>(gs.d_tab, gs.xmax);
  check_launch(ctx);
  k_guard_probe_res<<<pg, 256, 0, ctx->stream>>>(gs.d_tab, gs.rmax);
  check_launch(ctx);
  // Read the flags: the status word of each guarded matrix and its bounds.
  std::vector<unsigned long long> amax(gs.nall), growth(gs.nall), xmax(gs.nall), rmax(gs.nall);
  std::vector<int> st(G);
  QX_CUDA(cudaMemcpyAsync(amax.data(), gs.amax, gs.nall * sizeof(unsigned long long), cudaMemcpyDeviceToHost,
                          ctx->stream));
  QX_CUDA(cudaMemcpyAsync(growth.data(), gs.growth, gs.nall * sizeof(unsigned long long), cudaMemcpyDeviceToHost,
                          ctx->stream));
  QX_CUDA(cudaMemcpyAsync(xmax.data(), gs.xmax, gs.nall * sizeof(unsigned long long), cudaMemcpyDeviceToHost,
                          ctx->stream));
  QX_CUDA(cudaMemcpyAsync(rmax.data(), gs.rmax, gs.nall * sizeof(unsigned long long), cudaMemcpyDeviceToHost,
                          ctx->stream));
  for (int i = 0; i < G; ++i)
    QX_CUDA(cudaMemcpyAsync(&st[i], gs.mats[i].status, sizeof(int), cudaMemcpyDeviceToHost, ctx->stream));
  QX_CUDA(cudaStreamSynchronize(ctx->stream));
  auto as_double = [](unsigned long long u) {
    double d;
    memcpy(&d, &u, sizeof d);
    return d;
  };
  std::vector<GuardMat> flagged;
  nmax = 0;
  for (int i = 0; i < G; ++i) {
    const GuardMat& g = gs.mats[i];
    const double a = as_double(amax[g.idx]), gr = as_double(growth[g.idx]);
    const double eta = as_double(rmax[g.idx]) / ((double)g.n * a * as_double(xmax[g.idx]));
    if (st[i] != 0 || !(gr <= kGuardGrowth * a) || !(eta <= kGuardResidual)) {
      flagged.push_back(g);
      nmax = std::max(nmax, g.n);
    }
  }
  gs.nflagged = (int)flagged.size();
  ctx->guard_matrices += G;
  ctx->guard_reinverted += gs.nflagged;
  if (flagged.empty()) return 0;
  const int F = (int)flagged.size();
  QX_REQUIRE(F <= 65535, QX_ERR_INVALID_INPUT, "%d matrices to re-invert in one call (at most 65535)", F);
  QX_CUDA(cudaMemcpyAsync(gs.d_tab, flagged.data(), F * sizeof(GuardMat), cudaMemcpyHostToDevice, ctx->stream));
  k_piv_init<<<F, 256, 0, ctx->stream>>>(gs.d_tab);
  check_launch(ctx);
  const int tiles = ceil_div(nmax, PivTile::BM);
  const bool smem_panel = nmax <= kPivSmemRows;
  const size_t panel_smem = (size_t)nmax * (PIV_NB * sizeof(double) + sizeof(int));
  for (int ks = 0; ks < nmax; ks += PIV_SB) {
    for (int k0 = ks; k0 < std::min(ks + PIV_SB, nmax); k0 += PIV_NB) {
      if (nmax <= 1024) {
        // The panel kernel also gathers the pivot rows for the update.
        if (nmax <= 512)
          k_piv_panel_reg<1><<<F, 512, 0, ctx->stream>>>(gs.d_tab, k0);
        else
          k_piv_panel_reg<2><<<F, 512, 0, ctx->stream>>>(gs.d_tab, k0);
        check_launch(ctx);
      } else {
        if (smem_panel)
          k_piv_panel<true><<<F, 512, panel_smem, ctx->stream>>>(gs.d_tab, k0);
        else
          k_piv_panel<false><<<F, 512, 0, ctx->stream>>>(gs.d_tab, k0);
        check_launch(ctx);
        k_piv_gather<<<dim3(F, 2), 256, 0, ctx->stream>>>(gs.d_tab, k0, PIV_NB, ks, ks + PIV_SB);
        check_launch(ctx);
      }
      // The rest of the super-panel (one column tile).
      k_piv_update<<<dim3(1, tiles, F), PivTile::THREADS, PivTile::SMEM, ctx->stream>>>(gs.d_tab, k0, PIV_NB, ks,
                                                                                        ks + PIV_SB, k0, k0 + 1);
      check_launch(ctx);
    }
    // Every column outside the super-panel: one rank-PIV_SB update.
    if (ks + PIV_SB < nmax || ks > 0) {
      k_piv_gather<<<dim3(F, 8), 256, 0, ctx->stream>>>(gs.d_tab, ks, PIV_SB, 0, nmax);
      check_launch(ctx);
      k_piv_update<<<dim3(tiles, tiles, F), PivTile::THREADS, PivTile::SMEM, ctx->stream>>>(
          gs.d_tab, ks, PIV_SB, 0, nmax, ks, ks + PIV_SB);
      check_launch(ctx);
    }
  }
  k_piv_inverse_perm<<<F, 256, 0, ctx->stream>>>(gs.d_tab);
  check_launch(ctx);
  k_piv_permute<<<dim3(nmax, F), 256, 0, ctx->stream>>>(gs.d_tab);
  check_launch(ctx);
  return F;
}

}  // namespace qx
