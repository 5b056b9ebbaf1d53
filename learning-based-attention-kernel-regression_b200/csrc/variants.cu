// Run-time kernel variant choices.  Each starts from its environment switch
// (read once) and can be changed between calls with laker_set_variant, which
// is what the autotuner (laker_b200.autotune) does after timing the candidates
// on the caller's problem size.
#include <atomic>
#include <cstdlib>

#include "internal.cuh"

namespace laker {
namespace {

constexpr int kNumVariants = 8;
std::atomic<int> g_variant[kNumVariants] = {{-1}, {-1}, {-1}, {-1}, {-1}, {-1}, {-1}, {-1}};

// Default bounded-wait limit: 2 s.
constexpr int kWaitLimitDefaultUs = 2000000;

int variant_default(int which) {
  if (which == LAKER_VARIANT_K1T_UNIT) {
    const char* e = getenv("LAKER_K1T_UNIT");
    return (e && e[0] == '2' && e[1] == 0) ? 2 : 4;
  }
  if (which == LAKER_VARIANT_SYM_MIN_BLOCKS) {
    // Measured at n = 2000 (4 blocks): 16.2 us per launch for the plain
    // kernel against 23.5 us for the tensor-core symmetric kernel, which then
    // has 10 block pairs for 148 SMs; the two are equal at n = 5000.
    const char* e = getenv("LAKER_SYM_MIN_BLOCKS");
    if (e && e[0]) {
      const int v = atoi(e);
      if (v >= 0 && v <= 64) return v;
    }
    return 6;
  }
  if (which == LAKER_VARIANT_K1T_LOGITS) {
    // split FP16 by default: n = 100k, 1.99 vs 2.10 ms per operator launch,
    // the same accuracy class as split TF32 (4.6e-7 vs 6.7e-7 relative at
    // n = 20k); LAKER_K1T_F16=0 selects split TF32
    const char* e = getenv("LAKER_K1T_F16");
    return (e && e[0] == '0') ? 0 : 1;
  }
  if (which == LAKER_VARIANT_WAIT_LIMIT_US) return kWaitLimitDefaultUs;
  if (which == LAKER_VARIANT_MULTI_FLASH_K) {
    const char* e = getenv("LAKER_MULTI_FLASH_K");
    if (e && e[0]) {
      const int v = atoi(e);
      if (v >= 0 && v <= 1 << 20) return v;
    }
    // measured on B200 (n = 50k, k = 16: 3.73 vs 7.75 ms for the CUDA-core-
    // logit kernel; n = 20k, k = 16: 0.70 vs 1.34 ms); wider products (one
    // exp2 per entry per chunk of 32) are faster on the CUDA-core-logit kernel
    return 32;
  }
  const char* e = getenv("LAKER_K2_LOGITS_TC");
  return (e && e[0] == '1') ? 1 : 0;
}

bool variant_valid(int which, int value) {
  if (which == LAKER_VARIANT_K1T_UNIT) return value == 2 || value == 4;
  if (which == LAKER_VARIANT_SYM_MIN_BLOCKS) return value >= 0 && value <= 64;
  if (which == LAKER_VARIANT_K1T_LOGITS) return value == 0 || value == 1;
  if (which == LAKER_VARIANT_WAIT_LIMIT_US) return value >= 0 && value <= kWaitLimitDefaultUs;
  if (which == LAKER_VARIANT_MULTI_FLASH_K) return value >= 0 && value <= 1 << 20;
  return value == 0 || value == 1;
}

// Writes the wait limit into every translation unit's copy on the current
// device.
cudaError_t apply_wait_limit(int us) {
  const unsigned long long ns = (unsigned long long)us * 1000ull;
  cudaError_t (*const setters[])(unsigned long long) = {set_wait_limit_f32, set_wait_limit_f64,
                                                        set_wait_limit_sym, set_wait_limit_symtc,
                                                        set_wait_limit_tc, set_wait_limit_flash};
  for (auto f : setters) {
    const cudaError_t e = f(ns);
    if (e != cudaSuccess) return e;
  }
  return cudaSuccess;
}

}  // namespace

int variant_get(int which) {
  if (which < 0 || which >= kNumVariants) return -1;
  int v = g_variant[which].load(std::memory_order_relaxed);
  if (v < 0) {
    v = variant_default(which);
    int expected = -1;
    if (!g_variant[which].compare_exchange_strong(expected, v)) v = expected;
  }
  return v;
}

}  // namespace laker

using namespace laker;

extern "C" int laker_set_variant(int which, int value) {
  if (which < 0 || which >= kNumVariants || !variant_valid(which, value)) return -1;
  const int prev = variant_get(which);
  if (which == LAKER_VARIANT_WAIT_LIMIT_US) {
    const cudaError_t e = apply_wait_limit(value);
    if (e != cudaSuccess) {
      fail_cuda(e);
      return -1;
    }
  }
  g_variant[which].store(value, std::memory_order_relaxed);
  return prev;
}

extern "C" int laker_get_variant(int which) { return variant_get(which); }
