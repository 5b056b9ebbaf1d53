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
#include "tc.cuh"

namespace laker {
namespace {

constexpr int kTcRows = 128;          // M of the MMA, rows per CTA
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

// K-major operand descriptor of a TK-point tile.
template <int TK>
__device__ __forceinline__ uint64_t kmajor_desc(uint32_t saddr) {
  return kmajor_desc_raw(saddr, TileCfg<TK>::kSBO, TileCfg<TK>::kLayout);
}

// Instruction descriptor: kind::tf32, D = FP32, A and B TF32 K-major, M = 128.
__host__ __device__ constexpr uint32_t tf32_idesc(int n) { return tf32_idesc_mn(kTcRows, n); }

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
// Work items are (row tile, right-hand-side chunk, column segment); a
// persistent grid takes items round-robin, so every SM stays busy whatever
// the number of row tiles.  Roles inside a CTA (no CTA-wide barrier in the
// main loop; full/empty mbarrier rings between the roles):
//   warps 0-7  entries: per tile, wait for the column embeddings, wait for a
//              free A slot, write the TK x 128 entries as split TF32 into it,
//              arrive on its "full" barrier; per item, after the last tile,
//              wait for the accumulators, read them from TMEM and write the
//              item's output (Y, or a segment partial), free the TMEM buffer
//   warp 8     copies: per tile, wait for a free B stage, TMA the X image
//              slice and the column embeddings into it
//   warp 9     MMA: per tile, wait for A and B, issue the three split-TF32
//              products per 8-point K step, commit to the A slot's and the B
//              stage's "empty" barriers; per item, commit to the TMEM
//              buffer's "full" barrier (two TMEM buffers: the epilogue of one
//              item overlaps the MMAs of the next)
// Every wait is bounded; a timeout raises a shared abort flag that every role
// checks, then the CTA drains its copies and MMAs and frees TMEM.
constexpr int kEntryThreads = 256;
constexpr int kTcThreadsWs = kEntryThreads + 64;  // + copy warp + MMA warp
constexpr int kASlots = 2;

struct K2Work {
  int64_t rtiles;   // row tiles (of 128)
  int chunks;       // RHS chunks (of N)
  int segs;         // column segments
  int64_t ntiles;   // column tiles (of TK)
  int64_t tps;      // tiles per segment
  int64_t items;    // rtiles * chunks * segs
};

template <int DP, bool CLAMP, int TK>
__global__ void __launch_bounds__(kTcThreadsWs, 1)
    k2_tc_matvec(const float* __restrict__ rows32, int64_t m, const float* __restrict__ cols32,
                 const uint8_t* __restrict__ img, int N, int S, K2Work wk, float lam,
                 const float* __restrict__ X, int64_t ldx, int k, float* __restrict__ Y,
                 int64_t ldy, float* __restrict__ part, int* status) {
  constexpr int kABytes = TileCfg<TK>::kABytes;
  extern __shared__ __align__(1024) uint8_t smem_raw[];
  uint8_t* base = reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
  const uint32_t bbytes = (uint32_t)N * (4u * TK);
  const uint32_t sbytes = (uint32_t)round_up(2 * bbytes, 1024);
  const uint32_t ecbytes = (uint32_t)(TK * DP * 4);
  uint8_t* sA = base;                                    // kASlots x (hi, lo)
  uint8_t* sB = base + kASlots * 2 * kABytes;            // S stages
  float* sEc = reinterpret_cast<float*>(sB + (size_t)S * sbytes);
  uint64_t* b_full = reinterpret_cast<uint64_t*>(sEc + (size_t)S * TK * DP);
  uint64_t* b_empty = b_full + S;
  uint64_t* a_full = b_empty + S;
  uint64_t* a_empty = a_full + kASlots;
  uint64_t* acc_full = a_empty + kASlots;
  uint64_t* acc_empty = acc_full + 2;
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(acc_empty + 2);
  volatile int* abort = reinterpret_cast<volatile int*>(tmem_slot + 1);

  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;"
                 :
                 : "r"(smem_u32(tmem_slot)), "r"(512u));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
  }
  if (tid == 0) {
    for (int i = 0; i < S; ++i) {
      mbar_init(&b_full[i], 1);
      mbar_init(&b_empty[i], 1);
    }
    // one arrival per entry warp (not per thread: arrivals on one mbarrier
    // serialise)
    for (int i = 0; i < kASlots; ++i) {
      mbar_init(&a_full[i], kEntryThreads / 32);
      mbar_init(&a_empty[i], 1);
    }
    for (int i = 0; i < 2; ++i) {
      mbar_init(&acc_full[i], 1);
      mbar_init(&acc_empty[i], kEntryThreads / 32);
    }
    *abort = 0;
    mbar_fence_init();
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem_base = *tmem_slot;
  const uint32_t idesc = tf32_idesc(N);

  // item -> (row tile, chunk, segment, tile range)
  auto item_of = [&](int64_t it, int64_t* rt, int* ch, int64_t* t0, int64_t* t1) {
    *rt = it % wk.rtiles;
    const int64_t rest = it / wk.rtiles;
    *ch = (int)(rest % wk.chunks);
    const int64_t sg = rest / wk.chunks;
    *t0 = sg * wk.tps;
    *t1 = *t0 + wk.tps < wk.ntiles ? *t0 + wk.tps : wk.ntiles;
  };

  int64_t b_issued = 0;     // copy role: tiles issued
  int64_t mma_tiles = 0;
  if (warp == 8) {
    // ---- copies ------------------------------------------------------------
    if (lane == 0) {
      int64_t g = 0;  // tile counter over this CTA's items
      for (int64_t it = blockIdx.x; it < wk.items && !*abort; it += gridDim.x) {
        int64_t rt, t0, t1;
        int ch;
        item_of(it, &rt, &ch, &t0, &t1);
        for (int64_t t = t0; t < t1; ++t, ++g) {
          const int st = (int)(g % S);
          if (!wait_or_abort(&b_empty[st], (uint32_t)(((g / S) & 1) ^ 1), status, abort)) break;
          mbar_arrive_expect_tx(&b_full[st], 2 * bbytes + ecbytes);
          bulk_g2s(sB + (size_t)st * sbytes, img + ((int64_t)ch * wk.ntiles + t) * (int64_t)N * (8 * TK),
                   2 * bbytes, &b_full[st]);
          bulk_g2s(sEc + (size_t)st * TK * DP, cols32 + t * (TK * DP), ecbytes, &b_full[st]);
        }
      }
      b_issued = g;
    }
  } else if (warp == 9) {
    // ---- MMA issue -----------------------------------------------------------
    if (lane == 0) {
      int64_t g = 0, ni = 0;
      for (int64_t it = blockIdx.x; it < wk.items && !*abort; it += gridDim.x, ++ni) {
        int64_t rt, t0, t1;
        int ch;
        item_of(it, &rt, &ch, &t0, &t1);
        const int ab = (int)(ni & 1);
        if (!wait_or_abort(&acc_empty[ab], (uint32_t)(((ni >> 1) & 1) ^ 1), status, abort)) break;
        tc_fence_after();
        const uint32_t tmem_d = tmem_base + (uint32_t)(ab * 256);
        bool ok = true;
        for (int64_t t = t0; t < t1; ++t, ++g) {
          const int st = (int)(g % S), as = (int)(g % kASlots);
          if (!wait_or_abort(&b_full[st], (uint32_t)((g / S) & 1), status, abort) ||
              !wait_or_abort(&a_full[as], (uint32_t)((g / kASlots) & 1), status, abort)) {
            ok = false;
            break;
          }
          tc_fence_after();
          const uint8_t* bB = sB + (size_t)st * sbytes;
          const uint32_t ahi = smem_u32(sA + as * 2 * kABytes), alo = ahi + kABytes;
          const uint32_t bhi = smem_u32(bB), blo = bhi + bbytes;
#pragma unroll
          for (int kk = 0; kk < TK / 8; ++kk) {
            const uint32_t ko = (uint32_t)kk * 32u;
            mma_tf32(tmem_d, kmajor_desc<TK>(ahi + ko), kmajor_desc<TK>(bhi + ko), idesc,
                     (t > t0 || kk > 0) ? 1u : 0u);
            mma_tf32(tmem_d, kmajor_desc<TK>(ahi + ko), kmajor_desc<TK>(blo + ko), idesc, 1u);
            mma_tf32(tmem_d, kmajor_desc<TK>(alo + ko), kmajor_desc<TK>(bhi + ko), idesc, 1u);
          }
          mma_commit(&a_empty[as]);
          mma_commit(&b_empty[st]);
        }
        if (!ok) break;
        mma_commit(&acc_full[ab]);
      }
      mma_tiles = g;
    }
  } else {
    // ---- entries + epilogue (warps 0-7) ------------------------------------
    const int row = tid & 127, half = tid >> 7;
    int64_t g = 0, ni = 0;
    // waits are made warp-uniform (__all_sync) so that a warp reaches the
    // .sync.aligned TMEM loads with all its lanes or not at all
    for (int64_t it = blockIdx.x; it < wk.items; it += gridDim.x, ++ni) {
      if (__any_sync(0xffffffffu, *abort != 0)) break;
      int64_t rt, t0, t1;
      int ch;
      item_of(it, &rt, &ch, &t0, &t1);
      const int64_t i = rt * kTcRows + row;
      const bool row_ok = i < m;
      float2 ev[DP];
      {
        const float* blk = rows32 + (i >> 1) * (DP * 2) + (i & 1);
#pragma unroll
        for (int q = 0; q < DP; ++q) {
          const float v = row_ok ? blk[2 * q] * kLog2e : 0.0f;
          ev[q] = make_float2(v, v);
        }
      }
      bool ok = true;
      for (int64_t t = t0; t < t1; ++t, ++g) {
        const int st = (int)(g % S), as = (int)(g % kASlots);
        bool w = wait_or_abort(&b_full[st], (uint32_t)((g / S) & 1), status, abort);
        w = w && wait_or_abort(&a_empty[as], (uint32_t)(((g / kASlots) & 1) ^ 1), status, abort);
        if (!__all_sync(0xffffffffu, w)) {
          ok = false;
          break;
        }
        const float* ec = sEc + (size_t)st * TK * DP;
        uint8_t* a_hi = sA + as * 2 * kABytes;
        uint8_t* a_lo = a_hi + kABytes;
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
        fence_async_smem();  // this thread's entries -> visible to the tensor core
        __syncwarp();
        if (lane == 0) mbar_arrive(&a_full[as]);
      }
      if (!ok) break;
      // epilogue: this item's accumulators
      const int ab = (int)(ni & 1);
      if (!__all_sync(0xffffffffu, wait_or_abort(&acc_full[ab], (uint32_t)((ni >> 1) & 1), status, abort)))
        break;
      tc_fence_after();
      const int64_t r = rt * kTcRows + (warp & 3) * 32 + lane;
      const uint32_t lane_base = (uint32_t)((warp & 3) * 32) << 16;
      const int nh = N / 2, c_begin = (warp >> 2) * nh;
      const int sg = (int)(t0 / wk.tps);
      for (int c0 = c_begin; c0 < c_begin + nh; c0 += 16) {
        float v[16];
        tmem_ld16(tmem_base + (uint32_t)(ab * 256) + lane_base + (uint32_t)c0, v);
        if (r < m) {
#pragma unroll
          for (int u = 0; u < 16; ++u) {
            const int q = ch * N + c0 + u;
            if (q < k) {
              if (wk.segs == 1)
                Y[r * ldy + q] = v[u] + (lam != 0.0f ? lam * X[r * ldx + q] : 0.0f);
              else
                part[((int64_t)sg * m + r) * k + q] = v[u];
            }
          }
        }
      }
      tc_fence_before();
      __syncwarp();
      if (lane == 0) mbar_arrive(&acc_empty[ab]);
    }
  }

  // ---- teardown: every role has left its loop ---------------------------------
  __syncthreads();
  if (*abort) {
    // bounded drains: the copies the copy role issued and the MMAs the MMA
    // role committed (the last commit of each barrier covers earlier ones)
    if (warp == 8 && lane == 0) {
      // the latest copy of every stage (earlier ones were consumed)
      const int64_t from = b_issued > S ? b_issued - S : 0;
      for (int64_t gg = from; gg < b_issued; ++gg)
        mbar_wait_bounded(&b_full[gg % S], (uint32_t)((gg / S) & 1), status);
    }
    if (warp == 9 && lane == 0 && mma_tiles > 0) {
      // the last commit completes when every MMA issued before it has
      const int64_t gg = mma_tiles - 1;
      mbar_wait_bounded(&b_empty[gg % S], (uint32_t)((gg / S) & 1), status);
    }
  }
  tc_fence_before();
  __syncthreads();
  if (warp == 0) {
    tc_fence_after();
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" : : "r"(tmem_base), "r"(512u));
  }
}

// Y = lam X + sum over segments of the partials, in segment order.
__global__ void k2_reduce_kernel(const float* __restrict__ part, int segs, int64_t m, int k,
                                 float lam, const float* __restrict__ X, int64_t ldx,
                                 float* __restrict__ Y, int64_t ldy) {
  const int64_t total = m * (int64_t)k;
  for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < total;
       e += (int64_t)gridDim.x * blockDim.x) {
    const int64_t i = e / k;
    const int q = (int)(e - i * k);
    float s = 0.0f;
    for (int sg = 0; sg < segs; ++sg) s += part[(int64_t)sg * total + e];
    Y[i * ldy + q] = s + (lam != 0.0f ? lam * X[i * ldx + q] : 0.0f);
  }
}

// Tile width for a chunk of N right-hand sides.
int k2_tile_points(int N) { return N >= 128 ? 32 : 16; }

// B stages for N right-hand sides, TK-point tiles and padded dimension DP:
// as many as fit next to the A slots in 227 KB of shared memory, 2..8.
int k2_stages(int N, int TK, int DP) {
  const int sb = (int)round_up(2 * N * 4 * TK, 1024);
  const int avail = 227 * 1024 - 1024 - kASlots * 2 * kTcRows * TK * 4 - 256;
  int S = avail / (sb + TK * DP * 4 + 16);
  if (S > kTcMaxStages) S = kTcMaxStages;
  return S;
}

size_t k2_smem_bytes(int N, int S, int TK, int DP) {
  const size_t sb = (size_t)round_up(2 * N * 4 * TK, 1024);
  return 1024 + (size_t)kASlots * 2 * kTcRows * TK * 4 + (size_t)S * sb + (size_t)S * TK * DP * 4 +
         (size_t)(2 * S + 2 * kASlots + 4) * 8 + 64;
}

// Work split: column segments so that the items fill the SMs several times
// over (each segment at least 8 tiles).
K2Work k2_work(int64_t m, int64_t n, int k, int N, int TK) {
  K2Work w{};
  w.rtiles = ceil_div(m, kTcRows);
  w.chunks = (int)ceil_div(k, N);
  w.ntiles = ceil_div(n, TK);
  const int64_t base = w.rtiles * w.chunks;
  const int64_t want = 8 * (int64_t)sm_count();
  int64_t segs = base >= want ? 1 : ceil_div(want, base);
  const int64_t max_segs = w.ntiles / 8 > 1 ? w.ntiles / 8 : 1;
  if (segs > max_segs) segs = max_segs;
  if (segs > 64) segs = 64;
  w.tps = ceil_div(w.ntiles, segs);
  w.segs = (int)ceil_div(w.ntiles, w.tps);
  w.items = base * w.segs;
  return w;
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
cudaError_t launch_k2_t(const float* rows32, int64_t m, const float* cols32, const uint8_t* img,
                        int N, const K2Work& wk, float lam, const float* X, int64_t ldx, int k,
                        float* Y, int64_t ldy, float* part, int* status, cudaStream_t s) {
  const int S = k2_stages(N, TK, DP);
  const size_t smem = k2_smem_bytes(N, S, TK, DP);
  if (S < 2 || smem > 227 * 1024) return cudaErrorInvalidConfiguration;
  auto fn = k2_tc_matvec<DP, CLAMP, TK>;
  cudaError_t e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
  const int64_t grid = wk.items < (int64_t)sm_count() ? wk.items : (int64_t)sm_count();
  fn<<<(unsigned)grid, kTcThreadsWs, smem, s>>>(rows32, m, cols32, img, N, S, wk, lam, X, ldx, k, Y,
                                                ldy, part, status);
  return cudaGetLastError();
}

template <int DP, bool CLAMP>
cudaError_t launch_k2_tk(const float* rows32, int64_t m, const float* cols32, const uint8_t* img,
                         int N, int TK, const K2Work& wk, float lam, const float* X, int64_t ldx,
                         int k, float* Y, int64_t ldy, float* part, int* status, cudaStream_t s) {
  if (TK == 32)
    return launch_k2_t<DP, CLAMP, 32>(rows32, m, cols32, img, N, wk, lam, X, ldx, k, Y, ldy, part,
                                      status, s);
  return launch_k2_t<DP, CLAMP, 16>(rows32, m, cols32, img, N, wk, lam, X, ldx, k, Y, ldy, part,
                                    status, s);
}

}  // namespace

// RHS per CTA for k right-hand sides: a multiple of 32 (the MMA's N for M =
// 128 is a multiple of 16; each half of the epilogue reads 16-column groups),
// at most 256.
int k2_chunk_cols(int k) {
  const int kk = k < kTcMaxN ? k : kTcMaxN;
  return (int)round_up(kk, 32);
}

// Workspace of one multi-RHS product: the split X image, then the segment
// partials when the column range is split.
size_t k2_image_bytes(int64_t m, int64_t n, int k) {
  const int N = k2_chunk_cols(k);
  const int TK = k2_tile_points(N);
  const K2Work w = k2_work(m, n, k, N, TK);
  size_t b = (size_t)round_up((int64_t)((size_t)(w.chunks * w.ntiles) * (size_t)N * 8 * TK), 256);
  if (w.segs > 1) b += (size_t)w.segs * (size_t)m * (size_t)k * 4;
  return b;
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
// img: k2_image_bytes(m, n, k) of workspace.
cudaError_t launch_k2(const float* rows32, int64_t m, const float* cols32, int64_t n, int d,
                      int clamp, float lam, const float* X, int64_t ldx, int k, float* Y,
                      int64_t ldy, uint8_t* img, int* status, cudaStream_t s) {
  const int N = k2_chunk_cols(k);
  const int TK = k2_tile_points(N);
  const K2Work wk = k2_work(m, n, k, N, TK);
  float* part = wk.segs > 1
                    ? reinterpret_cast<float*>(img + round_up((int64_t)((size_t)(wk.chunks * wk.ntiles) *
                                                                        (size_t)N * 8 * TK), 256))
                    : nullptr;
  {
    const int64_t total = wk.ntiles * TK * (int64_t)wk.chunks * N;
    int64_t g = ceil_div(total, 256);
    if (g > (int64_t)sm_count() * 16) g = (int64_t)sm_count() * 16;
    if (TK == 32)
      k2_pack_x<32><<<(unsigned)g, 256, 0, s>>>(X, n, ldx, k, N, wk.ntiles, img);
    else
      k2_pack_x<16><<<(unsigned)g, 256, 0, s>>>(X, n, ldx, k, N, wk.ntiles, img);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
  }
  const int dp = padded_dim(d);
  cudaError_t e = cudaErrorInvalidValue;
  if (clamp) {
    LAKER_DISPATCH_TC(dp, e = (launch_k2_tk<DPv, true>(rows32, m, cols32, img, N, TK, wk, lam, X, ldx, k, Y, ldy, part, status, s)));
  } else {
    LAKER_DISPATCH_TC(dp, e = (launch_k2_tk<DPv, false>(rows32, m, cols32, img, N, TK, wk, lam, X, ldx, k, Y, ldy, part, status, s)));
  }
  if (e != cudaSuccess || wk.segs == 1) return e;
  int64_t g = ceil_div(m * (int64_t)k, 256);
  if (g > (int64_t)sm_count() * 16) g = (int64_t)sm_count() * 16;
  k2_reduce_kernel<<<(unsigned)g, 256, 0, s>>>(part, wk.segs, m, k, lam, X, ldx, Y, ldy);
  return cudaGetLastError();
}

}  // namespace laker
