// qx_screened_interaction_noalloc: Wc = (I - Pi)^-1 - I on device arrays with
// all scratch in one file-scope device array (no allocation in the call).
//
// Same arithmetic as qx_screened_interaction (the guarded block sweep of
// launch_invert_wc with its pivoted fallback, correlation_ac.rs:377-401 in the
// reference), processed in frequency chunks that fit the scratch array.
// Scratch layout, each region 256-byte aligned:
//   status [kMaxFreq] int | eps [c][naux][ldn] | T panels [c][naux][128] | P panels [c][naux][128] |
//   D blocks [c][128][128] | guard (copies of eps and the fallback's work arrays, guard_bytes)
// with c the chunk length.  Only the status words and the guard's bound words
// must start at zero; both are cleared by every call before use.
#include <mutex>

#include "qx_internal.cuh"

using namespace qx;

namespace {

constexpr size_t kScratchBytes = QX_NOALLOC_SCRATCH_BYTES;
constexpr int kMaxFreq = QX_NOALLOC_MAX_NFREQ;
constexpr int kMaxNaux = QX_NOALLOC_MAX_NAUX;
constexpr int kMaxDevices = 64;
constexpr size_t kStatusBytes = (size_t)kMaxFreq * sizeof(int);

static_assert(kScratchBytes % 256 == 0 && kStatusBytes % 256 == 0, "scratch alignment");

static __device__ __align__(256) double qx_noalloc_scratch[kScratchBytes / sizeof(double)];

inline size_t align256(size_t b) { return (b + 255) & ~size_t(255); }

// Bytes one frequency of the sweep needs (eps, T and P panels, D block),
// each region rounded.
inline size_t per_freq_bytes(int n, int ldn) {
  return align256((size_t)n * ldn * sizeof(double)) + 2 * align256((size_t)n * kSweepPanelCols * sizeof(double)) +
         align256((size_t)kSweepPanelCols * kSweepPanelCols * sizeof(double));
}

// Bytes of a chunk of c frequencies: the sweep's regions plus the guard's.
inline size_t chunk_bytes(int n, int ldn, int c) { return (size_t)c * per_freq_bytes(n, ldn) + guard_bytes(n, ldn, c); }

// Device address of the scratch array, resolved once per device with that
// device current (the module holding it is loaded on first use).
double* scratch_for_device(int device) {
  static std::mutex mu;
  static double* addr[kMaxDevices] = {};
  QX_REQUIRE(device >= 0 && device < kMaxDevices, QX_ERR_INVALID_INPUT, "device %d out of range", device);
  std::lock_guard<std::mutex> lock(mu);
  if (!addr[device]) {
    void* p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, qx_noalloc_scratch);
    if (e != cudaSuccess || p == nullptr)
      throw Error(QX_ERR_CUDA, fmt("cudaGetSymbolAddress(scratch) failed on device %d: %s", device,
                                   cudaGetErrorString(e)));
    sweep_set_attributes();
    addr[device] = static_cast<double*>(p);
  }
  return addr[device];
}

// eps[w][r][c] = delta_rc - pi[w][r][c] for c < n, 0 in the padding columns.
__global__ void k_noalloc_load(const double* __restrict__ pi, int n, int ldn, size_t stride,
                               double* __restrict__ eps) {
  const int w = blockIdx.y;
  const double* P = pi + (size_t)w * n * n;
  double* E = eps + (size_t)w * stride;
  for (size_t idx = (size_t)blockIdx.x * blockDim.x + threadIdx.x; idx < (size_t)n * ldn;
       idx += (size_t)gridDim.x * blockDim.x) {
    const int r = (int)(idx / ldn), c = (int)(idx % ldn);
    E[idx] = (c < n) ? (r == c ? 1.0 : 0.0) - P[(size_t)r * n + c] : 0.0;
  }
}

// wc[w][r][c] = eps[w][r][c] for c < n.
__global__ void k_noalloc_store(const double* __restrict__ eps, int n, int ldn, size_t stride,
                                double* __restrict__ wc) {
  const int w = blockIdx.y;
  const double* E = eps + (size_t)w * stride;
  double* W = wc + (size_t)w * n * n;
  for (size_t idx = (size_t)blockIdx.x * blockDim.x + threadIdx.x; idx < (size_t)n * n;
       idx += (size_t)gridDim.x * blockDim.x) {
    const int r = (int)(idx / n), c = (int)(idx % n);
    W[idx] = E[(size_t)r * ldn + c];
  }
}

void screened_noalloc(qx_ctx* ctx, int nfreq, int naux, const double* pi, double* wc) {
  QX_REQUIRE(nfreq > 0 && naux > 0 && pi && wc, QX_ERR_INVALID_INPUT, "invalid arguments");
  QX_REQUIRE(naux <= kMaxNaux, QX_ERR_INVALID_INPUT,
             "naux=%d exceeds the scratch limit of qx_screened_interaction_noalloc (naux <= %d)", naux, kMaxNaux);
  QX_REQUIRE(nfreq <= kMaxFreq, QX_ERR_INVALID_INPUT,
             "nfreq=%d exceeds the scratch limit of qx_screened_interaction_noalloc (nfreq <= %d)", nfreq,
             kMaxFreq);
  // Device (or managed) memory of the context's device: a kernel handed a
  // pointer of another device, or a host pointer, would fault.
  for (const void* p : {static_cast<const void*>(pi), static_cast<const void*>(wc)}) {
    cudaPointerAttributes at;
    const cudaError_t e = cudaPointerGetAttributes(&at, p);
    if (e != cudaSuccess) cudaGetLastError();
    QX_REQUIRE(e == cudaSuccess && (at.type == cudaMemoryTypeManaged ||
                                    (at.type == cudaMemoryTypeDevice && at.device == ctx->device)),
               QX_ERR_INVALID_INPUT,
               "qx_screened_interaction_noalloc takes device pointers of the context's device (%d) only",
               ctx->device);
  }
  const int n = naux, ldn = round_up(naux, 8);
  const size_t stride = (size_t)n * ldn;
  const size_t avail = kScratchBytes - kStatusBytes;
  int chunk = (int)std::min<size_t>((size_t)nfreq, avail / per_freq_bytes(n, ldn));
  while (chunk > 0 && chunk_bytes(n, ldn, chunk) > avail) --chunk;
  QX_REQUIRE(chunk >= 1, QX_ERR_INVALID_INPUT, "naux=%d does not fit the %zu-byte scratch", naux, kScratchBytes);

  char* base = reinterpret_cast<char*>(scratch_for_device(ctx->device));
  int* status = reinterpret_cast<int*>(base);
  double* eps = reinterpret_cast<double*>(base + kStatusBytes);
  double* Tp = reinterpret_cast<double*>(base + kStatusBytes + align256((size_t)chunk * stride * sizeof(double)));
  double* Pp = reinterpret_cast<double*>(reinterpret_cast<char*>(Tp) +
                                         align256((size_t)chunk * n * kSweepPanelCols * sizeof(double)));
  double* Dp = reinterpret_cast<double*>(reinterpret_cast<char*>(Pp) +
                                         align256((size_t)chunk * n * kSweepPanelCols * sizeof(double)));
  char* guard_mem = reinterpret_cast<char*>(Dp) +
                    align256((size_t)chunk * kSweepPanelCols * kSweepPanelCols * sizeof(double));
  const size_t guard_len = guard_bytes(n, ldn, chunk);

  QX_CUDA(cudaMemsetAsync(status, 0, (size_t)nfreq * sizeof(int), ctx->stream));
  for (int w0 = 0; w0 < nfreq; w0 += chunk) {
    const int c = std::min(chunk, nfreq - w0);
    dim3 g(std::min(ceil_div(n * ldn, 256), 4096), c);
    k_noalloc_load<<<g, 256, 0, ctx->stream>>>(pi + (size_t)w0 * n * n, n, ldn, stride, eps);
    check_launch(ctx);
    // Pi comes from the caller: the sweep runs guarded (eps >= I cannot be assumed).
    launch_invert_wc_panels(ctx, eps, n, ldn, stride, c, Tp, Dp, Pp, status + w0, guard_mem, guard_len);
    k_noalloc_store<<<g, 256, 0, ctx->stream>>>(eps, n, ldn, stride, wc + (size_t)w0 * n * n);
    check_launch(ctx);
  }
  QX_CUDA(cudaStreamSynchronize(ctx->stream));
  // Singular eps: the reference substitutes the identity for eps^-1
  // (correlation_ac.rs:390-397); the device already set Wc = 0 there.
  int h[256];
  for (int w0 = 0; w0 < nfreq; w0 += 256) {
    const int c = std::min(256, nfreq - w0);
    QX_CUDA(cudaMemcpy(h, status + w0, c * sizeof(int), cudaMemcpyDeviceToHost));
    for (int i = 0; i < c; ++i)
      if (h[i]) fprintf(stderr, "WARNING: Matrix inversion failed at freq %d: singular eps, using Wc = 0\n", w0 + i);
  }
}

}  // namespace

extern "C" qx_status qx_screened_interaction_noalloc(qx_ctx* ctx, int nfreq, int naux, const double* pi,
                                                     double* wc) {
  if (!ctx) return QX_ERR_INVALID_INPUT;
  try {
    reset_pending(ctx);
    ctx->launches = 0;
    QX_CUDA(cudaSetDevice(ctx->device));
    screened_noalloc(ctx, nfreq, naux, pi, wc);
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
