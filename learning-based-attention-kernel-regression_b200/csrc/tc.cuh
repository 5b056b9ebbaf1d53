// tcgen05 (5th-generation tensor core) helpers shared by the tensor-core
// kernels: shared-memory matrix and instruction descriptors, MMA issue and
// commit, TMEM loads, proxy fences, and the bounded waits of the
// warp-specialised pipelines.
#pragma once

#include "common.cuh"

namespace laker {

// Every kernel of this library that allocates tensor memory takes all 512
// TMEM columns of its SM (tcgen05.alloc blocks while they are taken).  Each
// such kernel therefore keeps its shared memory above half of the SM's 228 KB,
// so no two of them (the same kernel or two different ones, e.g. the engine's
// operator and a variance product on another stream) are ever resident on
// one SM at once: a CTA never waits in tcgen05.alloc for another CTA that
// shares its SM.
constexpr uint32_t kTmemExclusiveSmem = 116u * 1024u;

// Shared-memory matrix descriptor of a K-major operand in a swizzled
// canonical layout: 8-row core groups `sbo` bytes apart, layout code 2
// (128-byte swizzle), 4 (64-byte swizzle) or 6 (32-byte swizzle), tiles
// aligned to the swizzle atom.  A K step inside the swizzled row advances the
// start address.
__device__ __forceinline__ uint64_t kmajor_desc_raw(uint32_t saddr, uint32_t sbo, uint32_t layout) {
  uint64_t d = 0;
  d |= (uint64_t)((saddr >> 4) & 0x3FFFu);  // start address [0,14)
  d |= (uint64_t)1u << 16;                   // LBO (unused when swizzled) [16,30)
  d |= (uint64_t)(sbo >> 4) << 32;           // SBO [32,46)
  d |= (uint64_t)1u << 46;                   // descriptor version (Blackwell) [46,48)
  d |= (uint64_t)layout << 61;               // swizzle mode [61,64)
  return d;
}

// Instruction descriptor: kind::tf32, D = FP32, A and B TF32 K-major.
__host__ __device__ constexpr uint32_t tf32_idesc_mn(int m, int n) {
  return (1u << 4)                      // D format F32
         | (2u << 7)                    // A format TF32
         | (2u << 10)                   // B format TF32
         | ((uint32_t)(n >> 3) << 17)   // N >> 3
         | ((uint32_t)(m >> 4) << 24);  // M >> 4
}

// Instruction descriptor: kind::f16, D = FP32, A and B both FP16 (format 0),
// K-major.
__host__ __device__ constexpr uint32_t f16_idesc_mn(int m, int n) {
  return (1u << 4)                      // D format F32
         | (0u << 7)                    // A format F16
         | (0u << 10)                   // B format F16
         | ((uint32_t)(n >> 3) << 17)   // N >> 3
         | ((uint32_t)(m >> 4) << 24);  // M >> 4
}

__device__ __forceinline__ void mma_f16(uint32_t tmem_d, uint64_t adesc, uint64_t bdesc,
                                        uint32_t idesc, uint32_t accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}\n"
      :
      : "r"(tmem_d), "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate));
}

__device__ __forceinline__ void mma_tf32(uint32_t tmem_d, uint64_t adesc, uint64_t bdesc,
                                         uint32_t idesc, uint32_t accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, p;\n\t}\n"
      :
      : "r"(tmem_d), "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate));
}

// kind::tf32 with the A operand in tensor memory (M = 128 lanes, K = 8
// consecutive 32-bit columns from tmem_a) and B from shared memory.
__device__ __forceinline__ void mma_tf32_ts(uint32_t tmem_d, uint32_t tmem_a, uint64_t bdesc,
                                            uint32_t idesc, uint32_t accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::tf32 [%0], [%1], %2, %3, p;\n\t}\n"
      :
      : "r"(tmem_d), "r"(tmem_a), "l"(bdesc), "r"(idesc), "r"(accumulate));
}

// Arrive on `bar` when every MMA issued so far by this thread has completed.
__device__ __forceinline__ void mma_commit(uint64_t* bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];"
               :
               : "r"(smem_u32(bar))
               : "memory");
}

__device__ __forceinline__ void fence_async_smem() {
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}
__device__ __forceinline__ void tc_fence_before() {
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
}
__device__ __forceinline__ void tc_fence_after() {
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
}

__device__ __forceinline__ uint32_t to_tf32(float x) {
  uint32_t r;
  asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(r) : "f"(x));
  return r;
}

// 16 / 32 consecutive FP32 TMEM columns of this warp's 32 lanes (one lane
// per thread), waited for before returning.
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float (&v)[16]) {
  uint32_t r[16];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, "
      "%12, %13, %14, %15}, [%16];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]),
        "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]),
        "=r"(r[14]), "=r"(r[15])
      : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
  for (int i = 0; i < 16; ++i) v[i] = __uint_as_float(r[i]);
}

__device__ __forceinline__ void tmem_ld32(uint32_t taddr, float (&v)[32]) {
  uint32_t r[32];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, "
      "%12, %13, %14, %15, %16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, %28, %29, "
      "%30, %31}, [%32];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]),
        "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]),
        "=r"(r[14]), "=r"(r[15]), "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]),
        "=r"(r[21]), "=r"(r[22]), "=r"(r[23]), "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]),
        "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
      : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
  for (int i = 0; i < 32; ++i) v[i] = __uint_as_float(r[i]);
}

// Two 16-column loads (two TMEM addresses) under one wait.
__device__ __forceinline__ void tmem_ld16x2(uint32_t ta, uint32_t tb, float (&va)[16], float (&vb)[16]) {
  uint32_t r[32];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, "
      "%12, %13, %14, %15}, [%32];\n\t"
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%16, %17, %18, %19, %20, %21, %22, %23, %24, %25, "
      "%26, %27, %28, %29, %30, %31}, [%33];\n\t"
      "tcgen05.wait::ld.sync.aligned;"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]),
        "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]),
        "=r"(r[14]), "=r"(r[15]), "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]),
        "=r"(r[21]), "=r"(r[22]), "=r"(r[23]), "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]),
        "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
      : "r"(ta), "r"(tb)
      : "memory");
#pragma unroll
  for (int i = 0; i < 16; ++i) {
    va[i] = __uint_as_float(r[i]);
    vb[i] = __uint_as_float(r[16 + i]);
  }
}

// Stores 16 consecutive 32-bit TMEM columns of this warp's 32 lanes (one
// lane per thread); tmem_st_wait() waits for this thread's stores.
__device__ __forceinline__ void tmem_st16(uint32_t taddr, const uint32_t (&v)[16]) {
  asm volatile(
      "tcgen05.st.sync.aligned.32x32b.x16.b32 [%0], {%1, %2, %3, %4, %5, %6, %7, %8, %9, %10, "
      "%11, %12, %13, %14, %15, %16};"
      :
      : "r"(taddr), "r"(v[0]), "r"(v[1]), "r"(v[2]), "r"(v[3]), "r"(v[4]), "r"(v[5]), "r"(v[6]),
        "r"(v[7]), "r"(v[8]), "r"(v[9]), "r"(v[10]), "r"(v[11]), "r"(v[12]), "r"(v[13]),
        "r"(v[14]), "r"(v[15])
      : "memory");
}

__device__ __forceinline__ void tmem_st32(uint32_t taddr, const uint32_t (&v)[32]) {
  asm volatile(
      "tcgen05.st.sync.aligned.32x32b.x32.b32 [%0], {%1, %2, %3, %4, %5, %6, %7, %8, %9, %10, "
      "%11, %12, %13, %14, %15, %16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, "
      "%28, %29, %30, %31, %32};"
      :
      : "r"(taddr), "r"(v[0]), "r"(v[1]), "r"(v[2]), "r"(v[3]), "r"(v[4]), "r"(v[5]), "r"(v[6]),
        "r"(v[7]), "r"(v[8]), "r"(v[9]), "r"(v[10]), "r"(v[11]), "r"(v[12]), "r"(v[13]),
        "r"(v[14]), "r"(v[15]), "r"(v[16]), "r"(v[17]), "r"(v[18]), "r"(v[19]), "r"(v[20]),
        "r"(v[21]), "r"(v[22]), "r"(v[23]), "r"(v[24]), "r"(v[25]), "r"(v[26]), "r"(v[27]),
        "r"(v[28]), "r"(v[29]), "r"(v[30]), "r"(v[31])
      : "memory");
}

__device__ __forceinline__ void tmem_st_wait() {
  asm volatile("tcgen05.wait::st.sync.aligned;" ::: "memory");
}

// try_wait that may suspend the thread until the phase completes or about
// `hint_ns` have passed (instead of returning at once), so a waiting warp
// stops taking issue slots from the warps doing the work.  The pipeline waits
// use 20 us (measured 1-2 % faster than polling for k1t and the flash
// multi-RHS kernel; each wait still checks the abort flag and its time limit
// after every suspension).
constexpr uint32_t kWaitHintNs = 20000;
__device__ __forceinline__ bool mbar_try_wait_hint(uint64_t* bar, uint32_t parity, uint32_t hint_ns) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2, %3;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(ok)
      : "r"(smem_u32(bar)), "r"(parity), "r"(hint_ns)
      : "memory");
  return ok != 0;
}

__device__ __forceinline__ void mbar_arrive(uint64_t* bar) {
  asm volatile("mbarrier.arrive.release.cta.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar)) : "memory");
}

// Wait for a phase, giving up on timeout (the wait limit, ~2 s by default, or
// at once for a limit of 0; sets *abort and records LAKER_ERR_TIMEOUT) or
// when another role has set *abort.
__device__ __forceinline__ bool wait_or_abort(uint64_t* bar, uint32_t parity, int* status,
                                              volatile int* abort) {
  const unsigned long long limit = wait_limit_ns();
  if (limit == 0) {
    record_status(status, LAKER_ERR_TIMEOUT);
    *abort = 1;
    return false;
  }
  if (mbar_try_wait(bar, parity)) return true;
  const uint64_t t0 = global_timer_ns();
  for (uint32_t it = 0; it < (1u << 30); ++it) {
    if (mbar_try_wait_hint(bar, parity, kWaitHintNs)) return true;
    if (*abort) return false;
    if (global_timer_ns() - t0 >= limit) break;
  }
  record_status(status, LAKER_ERR_TIMEOUT);
  *abort = 1;
  return false;
}

// Warp-wide wait: lane 0 polls (one poll per warp instead of 32), then every
// lane confirms the completed phase with its own try_wait, which also gives
// each lane the acquire ordering.  The phase cannot advance again before this
// warp releases the resource it guards, so the confirmation succeeds at once;
// should it not, the lane falls back to the bounded wait.  All 32 lanes must
// call it; the result is warp-uniform.
__device__ __forceinline__ bool warp_wait_or_abort(uint64_t* bar, uint32_t parity, int* status,
                                                   volatile int* abort, int lane) {
  bool ok = true;
  if (lane == 0) ok = wait_or_abort(bar, parity, status, abort);
  ok = __shfl_sync(0xffffffffu, ok ? 1 : 0, 0) != 0;
  if (ok && !mbar_try_wait(bar, parity)) ok = wait_or_abort(bar, parity, status, abort);
  return __all_sync(0xffffffffu, ok);
}

}  // namespace laker
