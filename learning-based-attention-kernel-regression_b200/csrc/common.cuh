// Shared device helpers for the LAKER B200 solve path (sm_100a only).
//
// Everything here is header-only so that each translation unit of
// liblaker_b200.so can inline it; no relocatable device code is needed.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "../../include/laker_b200.h"

#if defined(__CUDA_ARCH__) && (__CUDA_ARCH__ < 1000)
#error "liblaker_b200 targets sm_100a (B200) only"
#endif

namespace laker {

// log2(e): the kernel entry exp(s) is evaluated as exp2(s * log2(e)), with
// log2(e) folded into the row-side embedding once per CTA.
constexpr float kLog2e = 1.4426950408889634f;

// The reference clamps the Gram entry at 80 (float32) before exp when
// max ||e_i||^2 >= 80 (laker/kernels.py:98-107, :181-185).  In the exp2
// domain that is 80 * log2(e).
constexpr float kClampLog2 = 80.0f * 1.4426950408889634f;
constexpr double kClamp64 = 700.0;

// Columns staged per shared-memory tile by the FP32 and FP64 matvecs.
constexpr int kTileCols32 = 256;  // 128 column pairs
constexpr int kTileCols64 = 128;

__host__ __device__ inline int64_t ceil_div(int64_t a, int64_t b) { return (a + b - 1) / b; }
__host__ __device__ inline int64_t round_up(int64_t a, int64_t b) { return ceil_div(a, b) * b; }

// Embedding dimension padded to an even count: the FP32 layout interleaves
// point pairs (see pack.cu), and every pair block must be 16-byte aligned.
__host__ __device__ inline int padded_dim(int d) { return (d + 1) & ~1; }

// Number of point pairs stored by the packed FP32 layout for n points: enough
// whole column tiles that every TMA bulk copy of a tile stays in bounds.
__host__ __device__ inline int64_t packed_pairs(int64_t n) {
  return round_up(ceil_div(n, 2) > 0 ? ceil_div(n, 2) : 1, kTileCols32 / 2);
}
// Number of rows stored by the packed FP64 layout.
__host__ __device__ inline int64_t packed_rows64(int64_t n) {
  return round_up(n > 0 ? n : 1, kTileCols64);
}

// ---------------------------------------------------------------------------
// Device status word.  Kernels never trap: a failed bounded wait records an
// error code here and the CTA returns; the host reads the word after the
// stream synchronises.
// ---------------------------------------------------------------------------
__device__ inline void record_status(int* status, int code) {
  if (status) atomicCAS(status, 0, code);
}

// Whether a product's status word reports a failure (its outputs are then
// written as NaN).
__device__ __forceinline__ bool status_failed(const int* status) {
  return status && *const_cast<volatile const int*>(status) != 0;
}
__device__ __forceinline__ float nan_f32() { return __int_as_float(0x7fc00000); }
__device__ __forceinline__ double nan_f64() { return __longlong_as_double(0x7ff8000000000000ll); }

// ---------------------------------------------------------------------------
// Fast exp2 on the MUFU pipe (PTX ex2.approx, flush-to-zero).
// ---------------------------------------------------------------------------
__device__ __forceinline__ float ex2_approx(float x) {
  float y;
  asm("ex2.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
  return y;
}

// ---------------------------------------------------------------------------
// Table-driven FP64 exp (Tang, "Table-driven implementation of the
// exponential function in IEEE floating-point arithmetic", ACM TOMS 15(2),
// 1989; constants by exp_table_gen.py).  exp(s) = 2^m 2^(j/64) exp(r) with
// k = rint(64 s / ln 2) = 64 m + j and r = s - k ln2/64, |r| <= ln2/128;
// exp(r) - 1 by its degree-5 Taylor polynomial (truncation 3.4e-17).  About
// half the FP64 operations of a general exp: the FP64 operator kernels spend
// half their time in the exponential.  Each CTA copies the 64-entry table
// into shared memory (exp_table_to_shared) before its first exp_tab.
// Results: ~1 ulp for s in [-708, 709]; 2^-1022 ... below (exp gives 0 or a
// subnormal there), overflow to +inf above; NaN gives NaN.
// ---------------------------------------------------------------------------
static __constant__ double c_exp2_64[64] = {
    1.0, 1.0108892860517005, 1.0218971486541166, 1.0330248790212284,
    1.0442737824274138, 1.0556451783605572, 1.0671404006768237, 1.0787607977571199,
    1.0905077326652577, 1.102382583307841, 1.1143867425958924, 1.1265216186082418,
    1.1387886347566916, 1.1511892299529827, 1.1637248587775775, 1.1763969916502812,
    1.189207115002721, 1.202156731452703, 1.215247359980469, 1.22848053610687,
    1.241857812073484, 1.255380757024691, 1.2690509571917332, 1.2828700160787783,
    1.2968395546510096, 1.3109612115247644, 1.3252366431597413, 1.339667524053303,
    1.3542555469368927, 1.3690024229745905, 1.383909881963832, 1.3989796725383112,
    1.4142135623730951, 1.42961333839197, 1.4451808069770467, 1.460917794180647,
    1.4768261459394993, 1.4929077282912648, 1.5091644275934228, 1.5255981507445384,
    1.5422108254079407, 1.559004400237837, 1.5759808451078865, 1.593142151342267,
    1.6104903319492543, 1.6280274218573478, 1.645755478153965, 1.6636765803267364,
    1.681792830507429, 1.7001063537185235, 1.718619298122478, 1.7373338352737062,
    1.7562521603732995, 1.7753764925265212, 1.7947090750031072, 1.8142521755003989,
    1.8340080864093424, 1.8539791250833855, 1.8741676341103, 1.8945759815869656,
    1.9152065613971474, 1.9360617934922943, 1.9571441241754002, 1.978456026387951};

__device__ __forceinline__ void exp_table_to_shared(double* s_tab, int tid, int nthreads) {
  for (int i = tid; i < 64; i += nthreads) s_tab[i] = c_exp2_64[i];
}

__device__ __forceinline__ double exp_tab(double s, const double* __restrict__ s_tab) {
  constexpr double kInvL = 92.33248261689366;      // 64 / ln 2
  constexpr double kLhi = 0.01083042469326756;     // ln2 / 64, leading 32 bits
  constexpr double kLlo = 2.9815858269852933e-12;  // ln2 / 64 - kLhi
  constexpr double kRound = 6755399441055744.0;    // 1.5 * 2^52
  const double t = fma(s, kInvL, kRound);          // low word of t: k (two's complement)
  const double kd = t - kRound;
  const int k = __double2loint(t);
  double r = fma(-kd, kLhi, s);  // exact: k kLhi has at most 49 bits for |s| < 2^10
  r = fma(-kd, kLlo, r);
  double q = fma(r, 1.0 / 120.0, 1.0 / 24.0);
  q = fma(q, r, 1.0 / 6.0);
  q = fma(q, r, 0.5);
  const double p = fma(r * r, q, r);  // exp(r) - 1
  const double tj = s_tab[k & 63];
  const int m = max(-1022, min(1023, k >> 6));
  return fma(tj, p, tj) * __hiloint2double((m + 1023) << 20, 0);
}

// ---------------------------------------------------------------------------
// mbarrier + 1-D TMA bulk copy (cp.async.bulk) wrappers.
// ---------------------------------------------------------------------------
__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}

__device__ __forceinline__ void mbar_fence_init() {
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t* bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.release.cta.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)),
               "r"(bytes)
               : "memory");
}

// Bulk global->shared copy completing on `bar`.  dst, src and bytes must be
// multiples of 16 (guaranteed by the packed layouts).
__device__ __forceinline__ void bulk_g2s(void* dst, const void* src, uint32_t bytes, uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
          smem_u32(dst)),
      "l"(src), "r"(bytes), "r"(smem_u32(bar))
      : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(ok)
      : "r"(smem_u32(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}

__device__ __forceinline__ uint64_t global_timer_ns() {
  uint64_t t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

// Time limit of the bounded waits in the pipelines' loops (ns).  Each
// translation unit has its own copy (the library is built without relocatable
// device code); laker_set_variant(LAKER_VARIANT_WAIT_LIMIT_US, ...) sets every
// unit's copy on the current device.  A limit of 0 makes every pipeline wait
// give up at once, without polling: the failure path (record the status,
// drain, return) then runs deterministically, with no fault and no hang.
static __constant__ unsigned long long c_wait_limit_ns = 2000000000ull;
// Drains after a failure (copies and MMAs still in flight) always get the
// full limit: a CTA must not exit while the copy engine or the tensor core may
// still write its shared memory.
constexpr unsigned long long kDrainLimitNs = 2000000000ull;

__device__ __forceinline__ unsigned long long wait_limit_ns() { return c_wait_limit_ns; }

// Sets this translation unit's wait limit on the current device.
[[maybe_unused]] static cudaError_t set_wait_limit_this_unit(unsigned long long ns) {
  return cudaMemcpyToSymbol(c_wait_limit_ns, &ns, sizeof(ns));
}

// Bounded wait on an mbarrier phase.  Returns false (and records
// LAKER_ERR_TIMEOUT) if the phase did not complete within `limit` ns, or at
// once for a limit of 0.
__device__ __forceinline__ bool mbar_wait_for(uint64_t* bar, uint32_t parity, int* status,
                                              unsigned long long limit) {
  if (limit == 0) {
    record_status(status, LAKER_ERR_TIMEOUT);
    return false;
  }
  if (mbar_try_wait(bar, parity)) return true;
  const uint64_t t0 = global_timer_ns();
  for (uint32_t it = 0; it < (1u << 30); ++it) {
    if (mbar_try_wait(bar, parity)) return true;
    if ((it & 255u) == 0 && global_timer_ns() - t0 >= limit) break;
  }
  record_status(status, LAKER_ERR_TIMEOUT);
  return false;
}

// A pipeline wait (the configurable limit, ~2 s by default).
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t* bar, uint32_t parity, int* status) {
  return mbar_wait_for(bar, parity, status, wait_limit_ns());
}

// A drain wait after a failure (always the full limit).
__device__ __forceinline__ bool mbar_wait_drain(uint64_t* bar, uint32_t parity, int* status) {
  return mbar_wait_for(bar, parity, status, kDrainLimitNs);
}

// ---------------------------------------------------------------------------
// Deterministic block reductions (fixed shuffle tree + fixed warp order).
// ---------------------------------------------------------------------------
template <typename V>
__device__ __forceinline__ V warp_sum(V v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

// Warp sums of V values per lane (V a power of two, 2..32) by recursive
// halving: at each of the first log2 V butterfly steps a lane keeps half of
// its values and sends the other half to its partner, so the step count and
// the additions fall from 5 V to V - 1 + 5 - log2 V.  On return v[0] of lane l
// holds the warp sum of value index l >> (5 - log2 V) (the same sum in the
// 32 / V lanes that share those bits).  Fixed order: deterministic.
template <int V, typename F>
__device__ __forceinline__ F warp_reduce_scatter(F (&v)[V], int lane) {
  static_assert(V >= 2 && V <= 32 && (V & (V - 1)) == 0, "V must be a power of two in [2, 32]");
  int o = 16;
#pragma unroll
  for (int h = V / 2; h >= 1; h >>= 1, o >>= 1) {
    const bool up = (lane & o) != 0;
#pragma unroll
    for (int i = 0; i < h; ++i) {
      const F keep = up ? v[i + h] : v[i];
      const F send = up ? v[i] : v[i + h];
      v[i] = keep + __shfl_xor_sync(0xffffffffu, send, o);
    }
  }
#pragma unroll
  for (; o > 0; o >>= 1) v[0] += __shfl_xor_sync(0xffffffffu, v[0], o);
  return v[0];
}

// Sums NV values over the block; result valid in every thread of warp 0.
// `scratch` must hold NV * (T/32) doubles.
template <int T, int NV>
__device__ __forceinline__ void block_sum(double (&v)[NV], double* scratch) {
  const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
#pragma unroll
  for (int q = 0; q < NV; ++q) v[q] = warp_sum(v[q]);
  if (l == 0) {
#pragma unroll
    for (int q = 0; q < NV; ++q) scratch[q * (T / 32) + w] = v[q];
  }
  __syncthreads();
  if (w == 0) {
#pragma unroll
    for (int q = 0; q < NV; ++q) {
      double t = (l < T / 32) ? scratch[q * (T / 32) + l] : 0.0;
      v[q] = warp_sum(t);
    }
  }
  __syncthreads();
}

// Completion detector for "last block finishes the reduction": each of
// `total` blocks publishes its partials, then calls this; exactly one block
// (the last to arrive) gets true.  The counter is reset by that block for
// reuse.
__device__ __forceinline__ bool arrive_last_of(unsigned int* counter, unsigned int total) {
  __shared__ bool s_last;
  __threadfence();
  __syncthreads();
  if (threadIdx.x == 0) {
    const unsigned int t = atomicAdd(counter, 1u);
    s_last = (t == total - 1);
    if (s_last) *counter = 0;  // every block has arrived; safe to rearm
  }
  __syncthreads();
  if (s_last) __threadfence();
  return s_last;
}

// Same over the whole grid.
__device__ __forceinline__ bool arrive_last_block(unsigned int* counter) {
  return arrive_last_of(counter, gridDim.x * gridDim.y * gridDim.z);
}

}  // namespace laker
