// Allocation-free variant of the single-RHS FP32 fused matvec.
//
// Who needs it: callers that hold device buffers but cannot allocate device
// memory themselves -- for example a host that receives its input and output
// buffers from another framework's allocator and has no allocation API of its
// own to hand us, or a latency-critical loop where a cudaMalloc (which may
// synchronise the device and grow the memory pool) is not allowed.  Those
// callers cannot provide the workspace that laker_attn_matvec_f32 asks for,
// so this entry point keeps its scratch (the per-segment FP64 row partials and
// the device status word) in a fixed array that lives in the library itself.
//
// The array is a file-scope `static __device__` buffer of
// LAKER_NOALLOC_SCRATCH_BYTES: every GPU that loads this module holds it until
// the process exits.  Host code cannot use the array's name as a device
// address, so the first call on each device looks the address up with
// cudaGetSymbolAddress (with that device current) and caches it; that first
// call may load the module, so make it before any stream capture.  All calls
// share the one array, which keeps the previous call's contents: the status
// word is cleared at the start of every call (the partials are fully
// overwritten), and calls whose work overlaps on the GPU -- on different
// streams, or from different host threads without ordering -- race on it.
// A device-side failure (a bounded wait that expired) makes the call write
// NaN to y and leaves LAKER_ERR_TIMEOUT in the status word, which
// laker_noalloc_status reads back.  The cached address of the array is only
// valid in the device context it was looked up in: the entry point must not
// be used across a cudaDeviceReset.
#include <mutex>

#include "internal.cuh"

namespace laker {
namespace {

static __device__ __align__(256) unsigned char g_noalloc_scratch[LAKER_NOALLOC_SCRATCH_BYTES];

constexpr int kMaxDevices = 64;
std::mutex g_noalloc_mutex;
void* g_noalloc_ptr[kMaxDevices] = {};

// Device address of the scratch array on the current device (set-up on the
// first call per device).
cudaError_t noalloc_scratch(void** out) {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  if (dev < 0 || dev >= kMaxDevices) return cudaErrorInvalidDevice;
  std::lock_guard<std::mutex> lock(g_noalloc_mutex);
  if (!g_noalloc_ptr[dev]) {
    void* p = nullptr;
    e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess) return e;
    g_noalloc_ptr[dev] = p;
  }
  *out = g_noalloc_ptr[dev];
  return cudaSuccess;
}

// y from the segment partials; NaN everywhere when the matvec kernel recorded
// a failure (a CTA whose bounded wait expired left its partials unwritten, and
// the array still holds the previous call's).
__global__ void noalloc_finish_kernel(const double* __restrict__ part, int S, int64_t m, float lam,
                                      const float* __restrict__ x, float* __restrict__ y,
                                      int square, const int* status) {
  const bool failed = status_failed(status);
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < m;
       i += (int64_t)gridDim.x * blockDim.x) {
    double acc = square ? (double)lam * (double)x[i] : 0.0;
    for (int s = 0; s < S; ++s) acc += part[(int64_t)s * m + i];
    y[i] = failed ? nan_f32() : (float)acc;
  }
}

}  // namespace
}  // namespace laker

using namespace laker;

extern "C" int laker_attn_matvec_f32_noalloc(const float* rows32, int64_t m, const float* cols32,
                                             int64_t n, int d, float lam, int clamp,
                                             const float* x, float* y, void* stream) {
  if (m < 0 || n < 0 || d < 1 || d > 16) return LAKER_ERR_INVALID_ARG;
  if (m > LAKER_NOALLOC_MAX_ROWS) return LAKER_ERR_SCRATCH_LIMIT;
  if (m == 0) return LAKER_OK;
  if (!rows32 || !cols32 || !y || (n > 0 && !x) || (m == n && !x)) return LAKER_ERR_INVALID_ARG;

  void* base = nullptr;
  cudaError_t e = noalloc_scratch(&base);
  if (e != cudaSuccess) return fail_cuda(e);
  int* status = static_cast<int*>(base);
  double* part = reinterpret_cast<double*>(static_cast<char*>(base) + kWsHeader);
  const int64_t cap_rows = (int64_t)((LAKER_NOALLOC_SCRATCH_BYTES - kWsHeader) / sizeof(double));

  // The usual segment plan, with the segment count capped so that S x m
  // partials fit the fixed array (m <= LAKER_NOALLOC_MAX_ROWS keeps S >= 1).
  SegPlan plan = k1_plan(m, n, d);
  if ((int64_t)plan.S * m > cap_rows) {
    const int64_t tiles = ceil_div(n > 0 ? n : 1, kTileCols32);
    int64_t S = cap_rows / m;
    if (S < 1) return LAKER_ERR_SCRATCH_LIMIT;
    const int64_t tps = ceil_div(tiles, S);
    plan.S = (int)ceil_div(tiles, tps);
    plan.cols_per_seg = tps * kTileCols32;
  }

  cudaStream_t s = static_cast<cudaStream_t>(stream);
  e = cudaMemsetAsync(status, 0, sizeof(int), s);
  if (e != cudaSuccess) return fail_cuda(e);
  if (n > 0) {
    e = launch_k1(rows32, m, cols32, n, d, clamp, x, part, plan, status, nullptr, s);
    if (e != cudaSuccess) return fail_cuda(e);
  }
  int g = (int)ceil_div(m, 256);
  if (g > sm_count() * 8) g = sm_count() * 8;
  noalloc_finish_kernel<<<g, 256, 0, s>>>(part, n > 0 ? plan.S : 0, m, lam, x, y,
                                          (m == n) ? 1 : 0, status);
  e = cudaGetLastError();
  return e == cudaSuccess ? LAKER_OK : fail_cuda(e);
}

extern "C" int laker_noalloc_status(int* status, void* stream) {
  if (!status) return LAKER_ERR_INVALID_ARG;
  void* base = nullptr;
  cudaError_t e = noalloc_scratch(&base);
  if (e != cudaSuccess) return fail_cuda(e);
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  int h = 0;
  e = cudaMemcpyAsync(&h, base, sizeof(int), cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  if (e != cudaSuccess) return fail_cuda(e);
  *status = h;
  return LAKER_OK;
}
