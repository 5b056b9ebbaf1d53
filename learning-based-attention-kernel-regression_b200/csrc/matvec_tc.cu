// Multi-RHS FP32 attention-kernel matvec on the 5th-generation tensor cores
// (tcgen05): Y = [lam X +] exp(E_rows E_cols^T) X for k right-hand sides.
//
// Each CTA owns 128 rows (one TMEM lane per row, two threads per row) and one
// chunk of N <= 256 right-hand sides (N TMEM columns of FP32 accumulators).
// It walks the columns (points) in tiles of 16:
//   * column embeddings (packed32, 16 points) and the matching 16 x N slice of
//     X, pre-split and pre-swizzled by k2_pack_x, arrive by TMA bulk copies
//     (one mbarrier transaction, double-buffered);
//   * every thread evaluates 16 kernel entries p of its row on the CUDA cores
//     (packed FFMA2 logits with log2 e folded into the row, MUFU ex2) and
//     writes p = p_hi + p_lo, both TF32, into the A tiles in the 128-byte
//     swizzled K-major layout the tensor core reads;
//   * one thread issues, per 8-point K step, the three split-TF32 products
//     P_hi X_hi + P_hi X_lo + P_lo X_hi (tcgen05.mma kind::tf32, M = 128,
//     N, FP32 accumulation in TMEM) and commits them to an mbarrier.
// TF32 alone (2^-11) or BF16 entries perturb A by far more than its smallest
// eigenvalue (lambda) and iterative refinement then diverges; the three
// products carry ~2^-21 relative error per term (the missing lo x lo term and
// the TF32 rounding of the lo parts), as accurate as FP32 entries need to be.
// The epilogue reads the accumulators with tcgen05.ld (warp w: lanes
// 32w..32w+31) and writes Y in row-major order.
//
// Tiles are TK = 32 points (128-byte swizzle) for N >= 128 and 16 points
// (64-byte swizzle) below.  Smem per CTA: A (hi + lo) 2 x 2 x 128 x 4 TK B, up
// to 160 KB of B stages, column embeddings per stage: one CTA per SM; TMEM:
// 256 columns.  The CTA
// evaluates the entries of tile t+1 while the tensor core works on tile t and
// the copies run several tiles ahead.
#include <cstdlib>

#include "internal.cuh"

namespace laker {
namespace {

constexpr int kTcRows = 128;          // M of the MMA, rows per CTA
constexpr int kTcThreads = 256;       // two threads per row (16 points of a tile each)
constexpr int kTcMaxN = 256;          // right-hand sides per CTA (TMEM columns)
constexpr int kTcMaxStages = 8;

// Column tiles of TK points: TK = 32 (one 128-byte swizzled TF32 row) for
// wide right-hand-side chunks, where fewer, larger tiles cost less per point;
// TK = 16 (64-byte swizzle) for narrow chunks, where more B stages fit.
template <int TK>
struct TileCfg {
  static_assert(TK == 16 || TK == 32, "tile width");
  static constexpr int kRowBytes = TK * 4;
  static constexpr int kABytes = kTcRows * kRowBytes;  // one A operand
  static constexpr uint32_t kSBO = 8u * kRowBytes;     // 8-row core group
  static constexpr uint32_t kLayout = TK == 32 ? 2u : 4u;  // SWIZZLE_128B / SWIZZLE_64B
  // byte offset of TF32 element (row, k) in the swizzled tile: address bits
  // [4, 4+log2(TK/4)) XOR the bits just above the 8-row group's row stride
  __host__ __device__ static constexpr uint32_t offset(uint32_t row, uint32_t k) {
    return TK == 32 ? row * 128u + ((((k >> 2) ^ (row & 7u)) << 4)) + (k & 3u) * 4u
                    : row * 64u + ((((k >> 2) ^ ((row >> 1) & 3u)) << 4)) + (k & 3u) * 4u;
  }
};

// ---- tcgen05 / descriptor helpers -------------------------------------------
__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

// Shared-memory matrix descriptor for a K-major operand in a swizzled
// canonical layout: rows of TK TF32, 8-row core groups SBO bytes apart, tiles
// 1024-byte aligned.  The K step inside the row advances the start address
// by 32 bytes per 8 TF32.
template <int TK>
__device__ __forceinline__ uint64_t kmajor_desc(uint32_t saddr) {
  uint64_t d = 0;
  d |= (uint64_t)((saddr >> 4) & 0x3FFFu);                  // start address [0,14)
  d |= (uint64_t)1u << 16;                                   // LBO (unused when swizzled) [16,30)
  d |= (uint64_t)(TileCfg<TK>::kSBO >> 4) << 32;             // SBO [32,46)
  d |= (uint64_t)1u << 46;                                   // descriptor version (Blackwell) [46,48)
  d |= (uint64_t)TileCfg<TK>::kLayout << 61;                 // swizzle mode [61,64)
  return d;
}

// Instruction descriptor: kind::tf32, D = FP32, A and B TF32 K-major, M = 128.
__host__ __device__ constexpr uint32_t tf32_idesc(int n) {
  return (1u << 4)                      // D format F32
         | (2u << 7)                    // A format TF32
         | (2u << 10)                   // B format TF32
         | ((uint32_t)(n >> 3) << 17)   // N >> 3
         | ((uint32_t)(kTcRows >> 4) << 24);  // M >> 4
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

// ---- X -> split, swizzled B tiles ---------------------------------------------
// Image of chunk c (N right-hand sides), column tile t: [hi: N rows x 4 TK B]
// [lo: N rows x 4 TK B], row = right-hand side, TK points per row.
template <int TK>
__global__ void k2_pack_x(const float* __restrict__ X, int64_t n, int64_t ldx, int k, int N,
                          int64_t ntiles, uint8_t* __restrict__ img) {
  constexpr int kTcTileK = TK;
  const int64_t total = (int64_t)ntiles * kTcTileK * ((k + N - 1) / N) * N;
  for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < total;
       e += (int64_t)gridDim.x * blockDim.x) {
    // e enumerates (point j, padded rhs q) with q fastest: coalesced reads of X
    const int kp = ((k + N - 1) / N) * N;
    const int64_t j = e / kp;
    const int q = (int)(e - j * kp);
    const float v = (j < n && q < k) ? X[j * ldx + q] : 0.0f;
    const uint32_t hi = to_tf32(v);
    const uint32_t lo = to_tf32(v - __uint_as_float(hi));
    const int64_t c = q / N, t = j / kTcTileK;
    const int r = q - (int)c * N, kk = (int)(j - t * kTcTileK);
    uint8_t* blk = img + ((c * ntiles + t) * (int64_t)N * (8 * TK));
    const uint32_t off = TileCfg<TK>::offset((uint32_t)r, (uint32_t)kk);
    *reinterpret_cast<uint32_t*>(blk + off) = hi;
    *reinterpret_cast<uint32_t*>(blk + (int64_t)N * (4 * TK) + off) = lo;
  }
}

// ---- the kernel ---------------------------------------------------------------
// 256 threads: thread t evaluates row t % 128, points (TK / 2)(t / 128) ..
// +TK/2-1 of each TK-point tile.  A is double-buffered, B (with the column embeddings)
// has S stages, so S - 1 tiles are in flight.  Per tile t:
//   all      wait MMA(t-2) (frees A[t&1]); wait TMA(t) (stage t % S)
//   all      entries of tile t -> A[t&1]; proxy fence; barrier
//   thread 0 MMAs(t) -> commit to mma_bar[t&1]; wait MMA(t-1) (frees stage
//            (t-1) % S); TMA(t+S-1) into it
// so the tensor core works on tile t while the CTA evaluates tile t+1 and
// the copies run S - 1 tiles ahead.  Every mbarrier is waited on at most one
// phase behind its latest completion.
template <int DP, bool CLAMP, int TK>
__global__ void __launch_bounds__(kTcThreads, 1)
    k2_tc_matvec(const float* __restrict__ rows32, int64_t m, const float* __restrict__ cols32,
                 int64_t n, const uint8_t* __restrict__ img, int N, int S, int64_t ntiles,
                 float lam, const float* __restrict__ X, int64_t ldx, int k, float* __restrict__ Y,
                 int64_t ldy, int* status) {
  constexpr int kTcTileK = TK;
  constexpr int kTcABytes = TileCfg<TK>::kABytes;
  extern __shared__ __align__(1024) uint8_t smem_raw[];
  uint8_t* base = reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
  const uint32_t bbytes = (uint32_t)N * (4u * TK);       // one B operand of a tile
  const uint32_t sbytes = (uint32_t)round_up(2 * bbytes, 1024);  // one stage (hi + lo)
  const uint32_t ecbytes = (uint32_t)(kTcTileK * DP * 4);
  uint8_t* sA = base;                                     // 2 x (hi, lo) x 8 KB
  uint8_t* sB = base + 4 * kTcABytes;                     // S stages
  float* sEc = reinterpret_cast<float*>(sB + (size_t)S * sbytes);       // S x 16 x DP
  uint64_t* bars = reinterpret_cast<uint64_t*>(sEc + (size_t)S * kTcTileK * DP);  // tma[S], mma[2]
  uint64_t* mma_bar = bars + S;
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(mma_bar + 2);

  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int row = tid & (kTcRows - 1), half = tid >> 7;
  const int64_t row0 = (int64_t)blockIdx.x * kTcRows;
  const int chunk = blockIdx.y;
  const uint32_t idesc = tf32_idesc(N);

  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;"
                 :
                 : "r"(smem_u32(tmem_slot)), "r"((uint32_t)kTcMaxN));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
  }
  if (tid == 0) {
    for (int i = 0; i < S + 2; ++i) mbar_init(&bars[i], 1);
    mbar_fence_init();
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem_d = *tmem_slot;

  float2 ev[DP];
  const bool row_ok = row0 + row < m;
  {
    const int64_t i = row0 + row;
    const float* blk = rows32 + (i >> 1) * (DP * 2) + (i & 1);
#pragma unroll
    for (int q = 0; q < DP; ++q) {
      const float v = row_ok ? blk[2 * q] * kLog2e : 0.0f;
      ev[q] = make_float2(v, v);
    }
  }

  auto issue = [&](int64_t t) {
    const int st = (int)(t % S);
    uint8_t* dB = sB + (size_t)st * sbytes;
    float* dE = sEc + (size_t)st * kTcTileK * DP;
    mbar_arrive_expect_tx(&bars[st], 2 * bbytes + ecbytes);
    bulk_g2s(dB, img + ((int64_t)chunk * ntiles + t) * (int64_t)N * (8 * TK), 2 * bbytes, &bars[st]);
    bulk_g2s(dE, cols32 + t * (kTcTileK * DP), ecbytes, &bars[st]);
  };

  int64_t issued = 0;
  if (tid == 0)
    for (; issued < ntiles && issued < S - 1; ++issued) issue(issued);
  bool failed = false;
  int64_t landed = 0, committed = 0;
  for (int64_t t = 0; t < ntiles; ++t) {
    const int abuf = (int)(t & 1);
    const int st = (int)(t % S);
    if (t >= 2) {
      const int ok = __syncthreads_and(
          mbar_wait_bounded(&mma_bar[abuf], (uint32_t)(((t - 2) >> 1) & 1), status) ? 1 : 0);
      if (!ok) {
        failed = true;
        break;
      }
    }
    {
      const int ok = __syncthreads_and(
          mbar_wait_bounded(&bars[st], (uint32_t)((t / S) & 1), status) ? 1 : 0);
      if (!ok) {
        failed = true;
        break;
      }
      ++landed;
    }
    // TK / 2 kernel entries of this row -> split TF32, swizzled into A[abuf]
    const float* ec = sEc + (size_t)st * kTcTileK * DP;
    uint8_t* a_hi = sA + abuf * 2 * kTcABytes;
    uint8_t* a_lo = a_hi + kTcABytes;
#pragma unroll
    for (int cc = 0; cc < TK / 8; ++cc) {
      const int c = (TK / 8) * half + cc;  // 16-byte chunk: points 4c .. 4c+3
      float p[4];
#pragma unroll
      for (int h = 0; h < 2; ++h) {
        const float* pe = ec + (2 * c + h) * (DP * 2);
        float2 sacc = __fmul2_rn(ev[0], make_float2(pe[0], pe[1]));
#pragma unroll
        for (int q = 1; q < DP; ++q) sacc = __ffma2_rn(ev[q], make_float2(pe[2 * q], pe[2 * q + 1]), sacc);
        if (CLAMP) {
          sacc.x = fminf(sacc.x, kClampLog2);
          sacc.y = fminf(sacc.y, kClampLog2);
        }
        p[2 * h] = row_ok ? ex2_approx(sacc.x) : 0.0f;
        p[2 * h + 1] = row_ok ? ex2_approx(sacc.y) : 0.0f;
      }
      uint4 hi, lo;
      hi.x = to_tf32(p[0]);
      hi.y = to_tf32(p[1]);
      hi.z = to_tf32(p[2]);
      hi.w = to_tf32(p[3]);
      lo.x = to_tf32(p[0] - __uint_as_float(hi.x));
      lo.y = to_tf32(p[1] - __uint_as_float(hi.y));
      lo.z = to_tf32(p[2] - __uint_as_float(hi.z));
      lo.w = to_tf32(p[3] - __uint_as_float(hi.w));
      const uint32_t off = TileCfg<TK>::offset((uint32_t)row, (uint32_t)(4 * c));
      *reinterpret_cast<uint4*>(a_hi + off) = hi;
      *reinterpret_cast<uint4*>(a_lo + off) = lo;
    }
    fence_async_smem();
    tc_fence_before();
    __syncthreads();
    if (tid == 0) {
      tc_fence_after();
      const uint8_t* bB = sB + (size_t)st * sbytes;
      const uint32_t ahi = smem_u32(a_hi), alo = smem_u32(a_lo);
      const uint32_t bhi = smem_u32(bB), blo = smem_u32(bB + bbytes);
#pragma unroll
      for (int kk = 0; kk < kTcTileK / 8; ++kk) {
        const uint32_t ko = (uint32_t)kk * 32u;
        mma_tf32(tmem_d, kmajor_desc<TK>(ahi + ko), kmajor_desc<TK>(bhi + ko), idesc,
                 (t > 0 || kk > 0) ? 1u : 0u);
        mma_tf32(tmem_d, kmajor_desc<TK>(ahi + ko), kmajor_desc<TK>(blo + ko), idesc, 1u);
        mma_tf32(tmem_d, kmajor_desc<TK>(alo + ko), kmajor_desc<TK>(bhi + ko), idesc, 1u);
      }
      mma_commit(&mma_bar[abuf]);
      // stage (t-1) % S was read by MMA(t-1): refill it with tile t+S-1
      if (issued < ntiles) {
        bool ok = true;
        if (t >= 1) ok = mbar_wait_bounded(&mma_bar[abuf ^ 1], (uint32_t)(((t - 1) >> 1) & 1), status);
        if (ok) issue(issued++);
      }
    }
    ++committed;
    // a refill that could not be issued shows up as a TMA wait that times out
  }

  // all committed MMAs (the last commit covers every earlier one)
  bool done_ok = false;
  if (committed > 0) {
    const int64_t last = committed - 1;
    done_ok = __syncthreads_and(
                  mbar_wait_bounded(&mma_bar[last & 1], (uint32_t)((last >> 1) & 1), status) ? 1 : 0) != 0;
  }
  if (failed) {
    // bounded drain of the copies still in flight (only thread 0 issued them
    // and knows how many)
    if (tid == 0)
      for (int64_t t = landed; t < issued; ++t)
        mbar_wait_bounded(&bars[t % S], (uint32_t)((t / S) & 1), status);
  } else if (done_ok) {
    tc_fence_after();
    const int64_t i = row0 + (warp & 3) * 32 + lane;
    const uint32_t lane_base = (uint32_t)((warp & 3) * 32) << 16;
    const int nh = N / 2, c_begin = (warp >> 2) * nh;
    for (int c0 = c_begin; c0 < c_begin + nh; c0 += 16) {
      float v[16];
      tmem_ld16(tmem_d + lane_base + (uint32_t)c0, v);
      if (i < m) {
#pragma unroll
        for (int u = 0; u < 16; ++u) {
          const int q = chunk * N + c0 + u;
          if (q < k) Y[i * ldy + q] = v[u] + (lam != 0.0f ? lam * X[i * ldx + q] : 0.0f);
        }
      }
    }
  }
  tc_fence_before();
  __syncthreads();
  if (warp == 0) {
    tc_fence_after();
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;"
                 :
                 : "r"(tmem_d), "r"((uint32_t)kTcMaxN));
  }
}

// Tile width for a chunk of N right-hand sides.
int k2_tile_points(int N) { return N >= 128 ? 32 : 16; }

// B stages for N right-hand sides, TK-point tiles and padded dimension DP:
// as many as fit next to the A tiles in 227 KB of shared memory, 2..8.
int k2_stages(int N, int TK, int DP) {
  const int sb = (int)round_up(2 * N * 4 * TK, 1024);
  const int avail = 227 * 1024 - 1024 - 4 * kTcRows * TK * 4 - 128;
  int S = avail / (sb + TK * DP * 4 + 8);
  if (S > kTcMaxStages) S = kTcMaxStages;
  return S;
}

size_t k2_smem_bytes(int N, int S, int TK, int DP) {
  const size_t sb = (size_t)round_up(2 * N * 4 * TK, 1024);
  return 1024 + 4 * (size_t)kTcRows * TK * 4 + (size_t)S * sb + (size_t)S * TK * DP * 4 +
         (size_t)(S + 2) * 8 + 16;
}

#define LAKER_DISPATCH_TC(dp, CALL)                     \
  switch (dp) {                                         \
    case 2: { constexpr int DPv = 2; CALL; } break;     \
    case 4: { constexpr int DPv = 4; CALL; } break;     \
    case 6: { constexpr int DPv = 6; CALL; } break;     \
    case 8: { constexpr int DPv = 8; CALL; } break;     \
    case 10: { constexpr int DPv = 10; CALL; } break;   \
    case 12: { constexpr int DPv = 12; CALL; } break;   \
    case 14: { constexpr int DPv = 14; CALL; } break;   \
    case 16: { constexpr int DPv = 16; CALL; } break;   \
    default: return cudaErrorInvalidValue;              \
  }

template <int DP, bool CLAMP, int TK>
cudaError_t launch_k2_t(const float* rows32, int64_t m, const float* cols32, int64_t n,
                        const uint8_t* img, int N, int64_t ntiles, int nchunks, float lam,
                        const float* X, int64_t ldx, int k, float* Y, int64_t ldy, int* status,
                        cudaStream_t s) {
  const int S = k2_stages(N, TK, DP);
  const size_t smem = k2_smem_bytes(N, S, TK, DP);
  if (S < 2 || smem > 227 * 1024) return cudaErrorInvalidConfiguration;
  auto fn = k2_tc_matvec<DP, CLAMP, TK>;
  cudaError_t e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
  dim3 grid((unsigned)ceil_div(m, kTcRows), (unsigned)nchunks);
  fn<<<grid, kTcThreads, smem, s>>>(rows32, m, cols32, n, img, N, S, ntiles, lam, X, ldx, k, Y,
                                    ldy, status);
  return cudaGetLastError();
}

template <int DP, bool CLAMP>
cudaError_t launch_k2_tk(const float* rows32, int64_t m, const float* cols32, int64_t n,
                         const uint8_t* img, int N, int64_t ntiles, int nchunks, float lam,
                         const float* X, int64_t ldx, int k, float* Y, int64_t ldy, int* status,
                         cudaStream_t s) {
  if (k2_tile_points(N) == 32)
    return launch_k2_t<DP, CLAMP, 32>(rows32, m, cols32, n, img, N, ntiles, nchunks, lam, X, ldx,
                                      k, Y, ldy, status, s);
  return launch_k2_t<DP, CLAMP, 16>(rows32, m, cols32, n, img, N, ntiles, nchunks, lam, X, ldx, k,
                                    Y, ldy, status, s);
}

}  // namespace

// RHS per CTA for k right-hand sides: a multiple of 32 (the MMA's N for M =
// 128 is a multiple of 16; each half of the epilogue reads 16-column groups),
// at most 256.
int k2_chunk_cols(int k) {
  const int kk = k < kTcMaxN ? k : kTcMaxN;
  return (int)round_up(kk, 32);
}

size_t k2_image_bytes(int64_t n, int k) {
  const int N = k2_chunk_cols(k);
  const int TK = k2_tile_points(N);
  const int64_t ntiles = ceil_div(n, TK);
  const int64_t nchunks = ceil_div(k, N);
  return (size_t)(nchunks * ntiles) * (size_t)N * 8 * TK;
}

bool k2_use_tensor_cores() {
  static int v = -1;
  if (v < 0) {
    const char* e = getenv("LAKER_K2_TENSOR_CORES");
    v = (e && e[0] == '0') ? 0 : 1;
  }
  return v == 1;
}

// Y (m x k, ldy) = lam X + exp(rows cols^T) X (lam = 0: rectangular product).
// img: k2_image_bytes(n, k) of workspace.
cudaError_t launch_k2(const float* rows32, int64_t m, const float* cols32, int64_t n, int d,
                      int clamp, float lam, const float* X, int64_t ldx, int k, float* Y,
                      int64_t ldy, uint8_t* img, int* status, cudaStream_t s) {
  const int N = k2_chunk_cols(k);
  const int TK = k2_tile_points(N);
  const int64_t ntiles = ceil_div(n, TK);
  const int nchunks = (int)ceil_div(k, N);
  {
    const int64_t total = ntiles * TK * (int64_t)nchunks * N;
    int64_t g = ceil_div(total, 256);
    if (g > (int64_t)sm_count() * 16) g = (int64_t)sm_count() * 16;
    if (TK == 32)
      k2_pack_x<32><<<(unsigned)g, 256, 0, s>>>(X, n, ldx, k, N, ntiles, img);
    else
      k2_pack_x<16><<<(unsigned)g, 256, 0, s>>>(X, n, ldx, k, N, ntiles, img);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
  }
  const int dp = padded_dim(d);
  if (clamp) {
    LAKER_DISPATCH_TC(dp, return (launch_k2_tk<DPv, true>(rows32, m, cols32, n, img, N, ntiles, nchunks, lam, X, ldx, k, Y, ldy, status, s)));
  } else {
    LAKER_DISPATCH_TC(dp, return (launch_k2_tk<DPv, false>(rows32, m, cols32, n, img, N, ntiles, nchunks, lam, X, ldx, k, Y, ldy, status, s)));
  }
  return cudaErrorInvalidValue;
}

}  // namespace laker
