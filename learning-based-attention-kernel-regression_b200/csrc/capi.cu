// Library-wide C ABI helpers: version, status strings, device queries, the
// column-segment planner and the roofline microbenchmarks.
#include "internal.cuh"

namespace laker {

static thread_local int g_last_cuda_error = 0;

int fail_cuda(cudaError_t e) {
  g_last_cuda_error = (int)e;
  return LAKER_ERR_CUDA;
}

int sm_count() {
  static int cache[64] = {0};
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0) return 148;
  if (dev < 64 && cache[dev] > 0) return cache[dev];
  int v = 0;
  if (cudaDeviceGetAttribute(&v, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || v < 1) v = 148;
  if (dev < 64) cache[dev] = v;
  return v;
}

SegPlan plan_segments(int64_t m, int64_t n, int rows_per_cta, int ctas_per_sm, int tile) {
  const int64_t RB = m > 0 ? ceil_div(m, rows_per_cta) : 1;
  const int64_t NT = n > 0 ? ceil_div(n, tile) : 1;
  const int64_t slots = (int64_t)sm_count() * ctas_per_sm;
  SegPlan best{1, NT * tile};
  double best_cost = 1e300;
  const int64_t smax = NT < 64 ? NT : 64;
  for (int64_t S = 1; S <= smax; ++S) {
    const int64_t tps = ceil_div(NT, S);
    const int64_t s_eff = ceil_div(NT, tps);
    if (s_eff != S) continue;  // another S gives the same split
    const int64_t ctas = RB * s_eff;
    if (ctas > 65535LL * 64) break;
    const int64_t waves = ceil_div(ctas, slots);
    // makespan in tiles: each wave lasts as long as its longest CTA, plus a
    // small per-CTA fixed cost (row loads, barrier set-up, partial store).
    const double cost = (double)waves * ((double)tps + 0.5);
    if (cost < best_cost - 1e-9) {
      best_cost = cost;
      best = SegPlan{(int)s_eff, tps * tile};
    }
  }
  return best;
}

namespace {

// ---- roofline microkernels -------------------------------------------------
// Register-resident dependent chains, 16 independent chains per thread.
constexpr int kPeakThreads = 256;

// 32 independent packed-pair chains, 4x unrolled: 128 FFMA2 per loop trip.
__global__ void __launch_bounds__(kPeakThreads) peak_ffma2_kernel(int iters, float seed, float* sink) {
  float2 a[32];
#pragma unroll
  for (int q = 0; q < 32; ++q) a[q] = make_float2(seed + q, seed - q);
  const float2 m = make_float2(0.9999f, 0.9998f), c = make_float2(1e-6f, 2e-6f);
  for (int it = 0; it < iters; it += 4) {
#pragma unroll
    for (int u = 0; u < 4; ++u)
#pragma unroll
      for (int q = 0; q < 32; ++q) a[q] = __ffma2_rn(a[q], m, c);
  }
  float s = 0.0f;
#pragma unroll
  for (int q = 0; q < 32; ++q) s += a[q].x + a[q].y;
  if (s == 1234.5678f) sink[0] = s;
}

// Same with scalar FFMA: 32 chains x 4 unroll.
__global__ void __launch_bounds__(kPeakThreads) peak_ffma_kernel(int iters, float seed, float* sink) {
  float a[32];
#pragma unroll
  for (int q = 0; q < 32; ++q) a[q] = seed + q;
  for (int it = 0; it < iters; it += 4) {
#pragma unroll
    for (int u = 0; u < 4; ++u)
#pragma unroll
      for (int q = 0; q < 32; ++q) a[q] = fmaf(a[q], 0.9999f, 1e-6f);
  }
  float s = 0.0f;
#pragma unroll
  for (int q = 0; q < 32; ++q) s += a[q];
  if (s == 1234.5678f) sink[0] = s;
}

__global__ void __launch_bounds__(kPeakThreads) peak_mufu_kernel(int iters, float seed, float* sink) {
  float a[16];
#pragma unroll
  for (int q = 0; q < 16; ++q) a[q] = -0.5f * (seed + 0.01f * q);
  for (int it = 0; it < iters; ++it) {
#pragma unroll
    for (int q = 0; q < 16; ++q) a[q] = ex2_approx(-a[q]);
  }
  float s = 0.0f;
#pragma unroll
  for (int q = 0; q < 16; ++q) s += a[q];
  if (s == 1234.5678f) sink[0] = s;
}

__global__ void __launch_bounds__(kPeakThreads) peak_dfma_kernel(int iters, double seed, double* sink) {
  double a[16];
#pragma unroll
  for (int q = 0; q < 16; ++q) a[q] = seed + q;
  for (int it = 0; it < iters; ++it) {
#pragma unroll
    for (int q = 0; q < 16; ++q) a[q] = fma(a[q], 0.9999999, 1e-9);
  }
  double s = 0.0;
#pragma unroll
  for (int q = 0; q < 16; ++q) s += a[q];
  if (s == 1234.5678) sink[0] = s;
}

template <typename F>
int time_kernel(F launch, cudaStream_t s, float* ms_out) {
  cudaEvent_t e0, e1;
  if (cudaEventCreate(&e0) != cudaSuccess) return fail_cuda(cudaGetLastError());
  if (cudaEventCreate(&e1) != cudaSuccess) {
    cudaEventDestroy(e0);
    return fail_cuda(cudaGetLastError());
  }
  launch();  // warm-up
  cudaEventRecord(e0, s);
  for (int r = 0; r < 3; ++r) launch();
  cudaEventRecord(e1, s);
  cudaError_t e = cudaEventSynchronize(e1);
  float ms = 0.0f;
  if (e == cudaSuccess) e = cudaEventElapsedTime(&ms, e0, e1);
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  if (e != cudaSuccess) return fail_cuda(e);
  *ms_out = ms / 3.0f;
  return LAKER_OK;
}

}  // namespace
}  // namespace laker

using namespace laker;

extern "C" int laker_version(void) { return 100; }

extern "C" int laker_workspace_status(const void* workspace, int* status, void* stream) {
  if (!workspace || !status) return LAKER_ERR_INVALID_ARG;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  int h = 0;
  cudaError_t e = cudaMemcpyAsync(&h, &static_cast<const WsHeader*>(workspace)->status, sizeof(int),
                                  cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  if (e != cudaSuccess) return fail_cuda(e);
  *status = h;
  return LAKER_OK;
}

extern "C" const char* laker_status_string(int status) {
  switch (status) {
    case LAKER_OK: return "ok";
    case LAKER_ERR_INVALID_ARG: return "invalid argument";
    case LAKER_ERR_CUDA: return "CUDA runtime error";
    case LAKER_ERR_BREAKDOWN: return "PCG breakdown: non-positive curvature";
    case LAKER_ERR_NOT_CONVERGED: return "PCG did not converge within max_iter";
    case LAKER_ERR_NONFINITE: return "non-finite value in a PCG inner product";
    case LAKER_ERR_TIMEOUT: return "bounded device wait expired";
    case LAKER_ERR_WORKSPACE: return "workspace too small";
    case LAKER_ERR_UNSUPPORTED: return "unsupported shape or dtype";
    case LAKER_ERR_CAPACITY: return "engine capacity exhausted (slots, points or block pairs)";
    case LAKER_ERR_SCRATCH_LIMIT:
      return "problem larger than the fixed scratch of the allocation-free entry point "
             "(m > LAKER_NOALLOC_MAX_ROWS)";
    default: return "unknown status";
  }
}

extern "C" int laker_last_cuda_error(void) { return g_last_cuda_error; }

extern "C" size_t laker_peaks_scratch_bytes(void) { return 256; }

extern "C" int laker_measure_peaks(void* scratch, double* ffma_tflops, double* mufu_tops,
                                   double* dfma_tflops, void* stream) {
  if (!scratch) return LAKER_ERR_INVALID_ARG;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  const int grid = sm_count() * 8;
  const double threads = (double)grid * kPeakThreads;
  float* f = static_cast<float*>(scratch);
  double* dd = static_cast<double*>(scratch);
  float ms = 0.0f;
  int st;
  if (ffma_tflops) {
    // best of packed (FFMA2) and scalar FFMA chains; 2 flops per FMA
    const int iters = 4096;
    st = time_kernel([&] { peak_ffma2_kernel<<<grid, kPeakThreads, 0, s>>>(iters, 1.0f, f); }, s, &ms);
    if (st) return st;
    const double packed = threads * iters * 32.0 * 2.0 * 2.0 / (ms * 1e-3) / 1e12;
    st = time_kernel([&] { peak_ffma_kernel<<<grid, kPeakThreads, 0, s>>>(iters, 1.0f, f); }, s, &ms);
    if (st) return st;
    const double scalar = threads * iters * 32.0 * 2.0 / (ms * 1e-3) / 1e12;
    *ffma_tflops = packed > scalar ? packed : scalar;
  }
  if (mufu_tops) {
    const int iters = 2048;
    st = time_kernel([&] { peak_mufu_kernel<<<grid, kPeakThreads, 0, s>>>(iters, 1.0f, f); }, s, &ms);
    if (st) return st;
    *mufu_tops = threads * iters * 16.0 / (ms * 1e-3) / 1e12;
  }
  if (dfma_tflops) {
    const int iters = 4096;
    st = time_kernel([&] { peak_dfma_kernel<<<grid, kPeakThreads, 0, s>>>(iters, 1.0, dd); }, s, &ms);
    if (st) return st;
    *dfma_tflops = threads * iters * 16.0 * 2.0 / (ms * 1e-3) / 1e12;
  }
  return LAKER_OK;
}
