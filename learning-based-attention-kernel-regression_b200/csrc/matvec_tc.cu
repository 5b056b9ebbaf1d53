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
#include "sym.cuh"
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
                          int64_t ntiles, uint8_t* __restrict__ img, const int* gate) {
  if (gate && *gate == 0) return;
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
                 int64_t ldy, float* __restrict__ part, int* status, const int* gate) {
  if (gate && *gate == 0) return;
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
          // P_hi by truncation (an AND), P_lo the exact remainder rounded to
          // TF32: |error| <= 2^-22 |p|
          hi.x = __float_as_uint(p[0]) & 0xffffe000u;
          hi.y = __float_as_uint(p[1]) & 0xffffe000u;
          hi.z = __float_as_uint(p[2]) & 0xffffe000u;
          hi.w = __float_as_uint(p[3]) & 0xffffe000u;
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
        mbar_wait_drain(&b_full[gg % S], (uint32_t)((gg / S) & 1), status);
    }
    if (warp == 9 && lane == 0 && mma_tiles > 0) {
      // the last commit completes when every MMA issued before it has
      const int64_t gg = mma_tiles - 1;
      mbar_wait_drain(&b_empty[gg % S], (uint32_t)((gg / S) & 1), status);
    }
  }
  tc_fence_before();
  __syncthreads();
  if (warp == 0) {
    tc_fence_after();
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" : : "r"(tmem_base), "r"(512u));
  }
}

// ---- logits on the tensor cores (k2t) ------------------------------------------
// The same items, X image, segment partials and epilogue as k2_tc_matvec, but
// the kernel entries' logits come from the tensor core too: per column tile
// the MMA warp issues the six split-TF32 logit MMAs (rows' E, scaled by log2 e,
// against the tile's points' E, K = 16; operands from the k1t operand image)
// into one of kSBufs TMEM logit buffers, then the P X products of the previous
// tile into the O accumulator.  The entry warps read a logit tile from TMEM,
// apply exp2 (MUFU), split into TF32 hi / lo and write the A operand of P X to
// shared memory -- no FMAs and no embedding loads per entry on the CUDA cores.
// TMEM: O in columns [0, 256), logit buffers from column 256.
constexpr int kSBufs = 4;
// 16 entry warps in two groups that take alternate tiles (two tiles in flight
// per row quadrant); group 0 also runs the epilogue.  Then the copy and MMA warps.
constexpr int kK2tEntry = 512, kK2tThreads = kK2tEntry + 64, kK2tCopyWarp = 16, kK2tMmaWarp = 17;
constexpr uint32_t kImgVar = 512 * 64;  // one variant of one 512-point image block
constexpr uint32_t kImgBlock = 4 * kImgVar;

template <bool CLAMP, int TK>
__global__ void __launch_bounds__(kK2tThreads, 1)
    k2t_matvec(const uint8_t* __restrict__ rimg, int64_t m, const uint8_t* __restrict__ cimg,
               const uint8_t* __restrict__ img, int N, int S, int AS, K2Work wk, float lam,
               const float* __restrict__ X, int64_t ldx, int k, float* __restrict__ Y, int64_t ldy,
               float* __restrict__ part, int* status, const int* gate) {
  if (gate && *gate == 0) return;
  constexpr int kABytes = TileCfg<TK>::kABytes;
  constexpr uint32_t kArBytes = kTcRows * 64;   // one variant of the rows' operand
  constexpr uint32_t kBcBytes = TK * 64;        // one variant of a tile's points' operand
  static_assert(TK == 32, "logit tiles of 32 points (TMEM buffers of 32 columns)");
  extern __shared__ __align__(1024) uint8_t smem_raw[];
  uint8_t* base = reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
  const uint32_t bbytes = (uint32_t)N * (4u * TK);
  const uint32_t sbytes = (uint32_t)round_up(2 * bbytes + 2 * kBcBytes, 1024);
  uint8_t* sA = base;                                 // AS P slots x (hi, lo)
  uint8_t* sAr = sA + (size_t)AS * 2 * kABytes;       // rows' operand (hi, lo)
  uint8_t* sB = sAr + 2 * kArBytes;                   // S stages: X (hi, lo), points (hi, lo)
  uint64_t* b_full = reinterpret_cast<uint64_t*>(sB + (size_t)S * sbytes);
  uint64_t* b_empty = b_full + S;
  uint64_t* a_full = b_empty + S;
  uint64_t* a_empty = a_full + AS;
  uint64_t* s_full = a_empty + AS;
  uint64_t* s_empty = s_full + kSBufs;
  uint64_t* acc_full = s_empty + kSBufs;
  uint64_t* acc_empty = acc_full + 1;
  uint64_t* ar_full = acc_empty + 1;
  uint64_t* ar_empty = ar_full + 1;
  uint64_t* drain = ar_empty + 1;
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(drain + 1);
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
    for (int i = 0; i < AS; ++i) {
      mbar_init(&a_full[i], kEntryThreads / 32);
      mbar_init(&a_empty[i], 1);
    }
    for (int i = 0; i < kSBufs; ++i) {
      mbar_init(&s_full[i], 1);
      mbar_init(&s_empty[i], kEntryThreads / 32);
    }
    mbar_init(acc_full, 1);
    mbar_init(acc_empty, kEntryThreads / 32);  // group 0 runs the epilogue
    mbar_init(ar_full, 1);
    mbar_init(ar_empty, 1);
    mbar_init(drain, 1);
    *abort = 0;
    mbar_fence_init();
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem_base = *tmem_slot;

  auto item_of = [&](int64_t it, int64_t* rt, int* ch, int64_t* t0, int64_t* t1) {
    *rt = it % wk.rtiles;
    const int64_t rest = it / wk.rtiles;
    *ch = (int)(rest % wk.chunks);
    const int64_t sg = rest / wk.chunks;
    *t0 = sg * wk.tps;
    *t1 = *t0 + wk.tps < wk.ntiles ? *t0 + wk.tps : wk.ntiles;
  };
  // byte offset of variant v (0, 1: rows scaled hi / lo; 2, 3: points hi / lo)
  // of point p in the operand image
  auto img_off = [](int64_t p, int v) -> int64_t {
    return (p >> 9) * (int64_t)kImgBlock + (int64_t)v * kImgVar + (p & 511) * 64;
  };

  int64_t b_issued = 0, ar_issued = 0;  // copy role
  bool mma_any = false;                 // MMA role
  if (warp == kK2tCopyWarp) {
    // ---- copies ------------------------------------------------------------
    if (lane == 0) {
      int64_t g = 0, ni = 0;
      for (int64_t it = blockIdx.x; it < wk.items && !*abort; it += gridDim.x, ++ni) {
        int64_t rt, t0, t1;
        int ch;
        item_of(it, &rt, &ch, &t0, &t1);
        // the rows' operand of this item (released by the MMA after its logits)
        if (!wait_or_abort(ar_empty, (uint32_t)((ni & 1) ^ 1), status, abort)) break;
        mbar_arrive_expect_tx(ar_full, 2 * kArBytes);
        bulk_g2s(sAr, rimg + img_off(rt * kTcRows, 0), kArBytes, ar_full);
        bulk_g2s(sAr + kArBytes, rimg + img_off(rt * kTcRows, 1), kArBytes, ar_full);
        ++ar_issued;
        bool ok = true;
        for (int64_t t = t0; t < t1; ++t, ++g) {
          const int st = (int)(g % S);
          if (!wait_or_abort(&b_empty[st], (uint32_t)(((g / S) & 1) ^ 1), status, abort)) {
            ok = false;
            break;
          }
          uint8_t* stg = sB + (size_t)st * sbytes;
          mbar_arrive_expect_tx(&b_full[st], 2 * bbytes + 2 * kBcBytes);
          bulk_g2s(stg, img + ((int64_t)ch * wk.ntiles + t) * (int64_t)N * (8 * TK), 2 * bbytes, &b_full[st]);
          bulk_g2s(stg + 2 * bbytes, cimg + img_off(t * TK, 2), kBcBytes, &b_full[st]);
          bulk_g2s(stg + 2 * bbytes + kBcBytes, cimg + img_off(t * TK, 3), kBcBytes, &b_full[st]);
          b_issued = g + 1;
        }
        if (!ok) break;
      }
    }
  } else if (warp == kK2tMmaWarp) {
    // ---- MMA issue -----------------------------------------------------------
    if (lane == 0) {
      const uint32_t idesc_s = tf32_idesc(TK);  // logits: N = TK points
      const uint32_t idesc_o = tf32_idesc(N);   // P X: N right-hand sides
      // descriptors built once and advanced by adds (the start-address field
      // holds address >> 4; shared addresses stay below 256 KB, so no carry)
      const uint64_t ar_hi = kmajor_desc_raw(smem_u32(sAr), 512u, 4u);
      const uint64_t ar_lo = ar_hi + (kArBytes >> 4);
      const uint64_t p_desc0 = kmajor_desc<TK>(smem_u32(sA));
      const uint64_t x_desc0 = kmajor_desc<TK>(smem_u32(sB));
      const uint64_t bc_desc0 = kmajor_desc_raw(smem_u32(sB + 2 * bbytes), 512u, 4u);
      const uint64_t p_slot_step = (2 * kABytes) >> 4, p_lo_step = kABytes >> 4;
      const uint64_t stage_step = sbytes >> 4, x_lo_step = bbytes >> 4;
      int64_t g = 0, ni = 0;
      bool ok = true;
      // P X of tile gp (stage / P slot of counter gp); first: the item's first tile
      auto issue_px = [&](int64_t gp, bool first) -> bool {
        const int st = (int)(gp % S), as = (int)(gp % AS);
        if (!wait_or_abort(&a_full[as], (uint32_t)((gp / AS) & 1), status, abort)) return false;
        tc_fence_after();
        const uint64_t ahi = p_desc0 + (uint64_t)as * p_slot_step, alo = ahi + p_lo_step;
        const uint64_t bhi = x_desc0 + (uint64_t)st * stage_step, blo = bhi + x_lo_step;
#pragma unroll
        for (int kk = 0; kk < TK / 8; ++kk) {
          const uint64_t ko = (uint64_t)kk * 2u;  // 32 bytes per 8-point K step
          mma_tf32(tmem_base, ahi + ko, bhi + ko, idesc_o, (!first || kk > 0) ? 1u : 0u);
          mma_tf32(tmem_base, ahi + ko, blo + ko, idesc_o, 1u);
          mma_tf32(tmem_base, alo + ko, bhi + ko, idesc_o, 1u);
        }
        mma_commit(&a_empty[as]);
        mma_commit(&b_empty[st]);
        return true;
      };
      for (int64_t it = blockIdx.x; it < wk.items && ok && !*abort; it += gridDim.x, ++ni) {
        int64_t rt, t0, t1;
        int ch;
        item_of(it, &rt, &ch, &t0, &t1);
        (void)rt;
        (void)ch;
        if (!wait_or_abort(ar_full, (uint32_t)(ni & 1), status, abort) ||
            !wait_or_abort(acc_empty, (uint32_t)((ni & 1) ^ 1), status, abort)) {
          ok = false;
          break;
        }
        tc_fence_after();
        // logits run up to L tiles ahead of the P X products (L <= S: a tile's
        // stage is held from its logits to its P X; L <= kSBufs: TMEM buffers)
        const int L = S < kSBufs ? S : kSBufs;
        const int64_t g0 = g, n_t = t1 - t0;
        int64_t gl = g0;  // next tile (counter) whose logits are issued
        for (int64_t gp = g0; gp < g0 + n_t; ++gp) {
          for (; gl < g0 + n_t && gl < gp + L; ++gl) {
            const int st = (int)(gl % S), sb = (int)(gl % kSBufs);
            if (!wait_or_abort(&b_full[st], (uint32_t)((gl / S) & 1), status, abort) ||
                !wait_or_abort(&s_empty[sb], (uint32_t)(((gl / kSBufs) & 1) ^ 1), status, abort)) {
              ok = false;
              break;
            }
            tc_fence_after();
            const uint64_t bc_hi = bc_desc0 + (uint64_t)st * stage_step, bc_lo = bc_hi + (kBcBytes >> 4);
            const uint32_t ds = tmem_base + 256u + (uint32_t)(sb * TK);
#pragma unroll
            for (int kk = 0; kk < 2; ++kk) {
              const uint64_t ko = (uint64_t)kk * 2u;  // 32 bytes in the start-address field
              mma_tf32(ds, ar_hi + ko, bc_hi + ko, idesc_s, kk > 0 ? 1u : 0u);
              mma_tf32(ds, ar_hi + ko, bc_lo + ko, idesc_s, 1u);
              mma_tf32(ds, ar_lo + ko, bc_hi + ko, idesc_s, 1u);
            }
            mma_any = true;
            mma_commit(&s_full[sb]);
            if (gl + 1 == g0 + n_t) mma_commit(ar_empty);  // last logits of the item issued
          }
          if (!ok || !issue_px(gp, gp == g0)) {
            ok = false;
            break;
          }
        }
        g = g0 + n_t;
        if (!ok) break;
        mma_commit(acc_full);
      }
    }
  } else {
    // ---- entries (warps 0-15: group warp >> 3 takes tiles g with g & 1 ==
    // group) + epilogue (group 0) -------------------------------------------
    const int grp = warp >> 3;
    const int q = warp & 3, h = (warp >> 2) & 1;
    const int row = q * 32 + lane;  // TMEM lane = row of the tile
    const uint32_t lane_base = (uint32_t)(q * 32) << 16;
    int64_t g = 0, ni = 0;
    for (int64_t it = blockIdx.x; it < wk.items; it += gridDim.x, ++ni) {
      if (__any_sync(0xffffffffu, *abort != 0)) break;
      int64_t rt, t0, t1;
      int ch;
      item_of(it, &rt, &ch, &t0, &t1);
      bool ok = true;
      for (int64_t t = t0; t < t1; ++t, ++g) {
        if ((int)(g & 1) != grp) continue;
        const int as = (int)(g % AS), sb = (int)(g % kSBufs);
        if (!__all_sync(0xffffffffu, wait_or_abort(&s_full[sb], (uint32_t)((g / kSBufs) & 1), status, abort))) {
          ok = false;
          break;
        }
        tc_fence_after();
        float v[16];
        tmem_ld16(tmem_base + lane_base + 256u + (uint32_t)(sb * TK + h * 16), v);
        tc_fence_before();
        __syncwarp();
        if (lane == 0) mbar_arrive(&s_empty[sb]);
        if (!__all_sync(0xffffffffu,
                        wait_or_abort(&a_empty[as], (uint32_t)(((g / AS) & 1) ^ 1), status, abort))) {
          ok = false;
          break;
        }
        uint8_t* a_hi = sA + (size_t)as * 2 * kABytes;
        uint8_t* a_lo = a_hi + kABytes;
#pragma unroll
        for (int c4 = 0; c4 < 4; ++c4) {
          uint4 hi, lo;
          uint32_t* ph = &hi.x;
          uint32_t* pl = &lo.x;
#pragma unroll
          for (int u = 0; u < 4; ++u) {
            const float sv = v[4 * c4 + u];
            const float p = ex2_approx(CLAMP ? fminf(sv, kClampLog2) : sv);
            ph[u] = __float_as_uint(p) & 0xffffe000u;  // truncation, as in k2_tc_matvec
            pl[u] = to_tf32(p - __uint_as_float(ph[u]));
          }
          const uint32_t off = TileCfg<TK>::offset((uint32_t)row, (uint32_t)(h * 16 + 4 * c4));
          *reinterpret_cast<uint4*>(a_hi + off) = hi;
          *reinterpret_cast<uint4*>(a_lo + off) = lo;
        }
        fence_async_smem();  // this thread's entries -> visible to the tensor core
        __syncwarp();
        if (lane == 0) mbar_arrive(&a_full[as]);
      }
      if (!ok) break;
      if (grp != 0) continue;
      // epilogue: this item's accumulators
      if (!__all_sync(0xffffffffu, wait_or_abort(acc_full, (uint32_t)(ni & 1), status, abort))) break;
      tc_fence_after();
      const int64_t r = rt * kTcRows + row;
      const int nh = N / 2, c_begin = h * nh;
      const int sg = (int)(t0 / wk.tps);
      for (int c0 = c_begin; c0 < c_begin + nh; c0 += 16) {
        float o[16];
        tmem_ld16(tmem_base + lane_base + (uint32_t)c0, o);
        if (r < m) {
#pragma unroll
          for (int u = 0; u < 16; ++u) {
            const int qq = ch * N + c0 + u;
            if (qq < k) {
              if (wk.segs == 1)
                Y[r * ldy + qq] = o[u] + (lam != 0.0f ? lam * X[r * ldx + qq] : 0.0f);
              else
                part[((int64_t)sg * m + r) * k + qq] = o[u];
            }
          }
        }
      }
      tc_fence_before();
      __syncwarp();
      if (lane == 0) mbar_arrive(acc_empty);
    }
  }

  // ---- teardown: every role has left its loop ---------------------------------
  __syncthreads();
  if (*abort) {
    // bounded drains of the copies in flight and of the MMAs issued
    if (warp == kK2tCopyWarp && lane == 0) {
      if (ar_issued > 0) mbar_wait_drain(ar_full, (uint32_t)((ar_issued - 1) & 1), status);
      const int64_t from = b_issued > S ? b_issued - S : 0;
      for (int64_t gg = from; gg < b_issued; ++gg)
        mbar_wait_drain(&b_full[gg % S], (uint32_t)((gg / S) & 1), status);
    }
    if (warp == kK2tMmaWarp && lane == 0 && mma_any) {
      mma_commit(drain);
      mbar_wait_drain(drain, 0u, status);
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
                                 float* __restrict__ Y, int64_t ldy, const int* gate) {
  if (gate && *gate == 0) return;
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
                        float* Y, int64_t ldy, float* part, int* status, cudaStream_t s,
                        const int* gate) {
  const int S = k2_stages(N, TK, DP);
  size_t smem = k2_smem_bytes(N, S, TK, DP);
  if (S < 2 || smem > 227 * 1024) return cudaErrorInvalidConfiguration;
  if (smem <= kTmemExclusiveSmem) smem = kTmemExclusiveSmem + 1024;  // one TMEM owner per SM
  auto fn = k2_tc_matvec<DP, CLAMP, TK>;
  cudaError_t e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
  const int64_t grid = wk.items < (int64_t)sm_count() ? wk.items : (int64_t)sm_count();
  fn<<<(unsigned)grid, kTcThreadsWs, smem, s>>>(rows32, m, cols32, img, N, S, wk, lam, X, ldx, k, Y,
                                                ldy, part, status, gate);
  return cudaGetLastError();
}

template <int DP, bool CLAMP>
cudaError_t launch_k2_tk(const float* rows32, int64_t m, const float* cols32, const uint8_t* img,
                         int N, int TK, const K2Work& wk, float lam, const float* X, int64_t ldx,
                         int k, float* Y, int64_t ldy, float* part, int* status, cudaStream_t s,
                         const int* gate) {
  if (TK == 32)
    return launch_k2_t<DP, CLAMP, 32>(rows32, m, cols32, img, N, wk, lam, X, ldx, k, Y, ldy, part,
                                      status, s, gate);
  return launch_k2_t<DP, CLAMP, 16>(rows32, m, cols32, img, N, wk, lam, X, ldx, k, Y, ldy, part,
                                    status, s, gate);
}

// Logit-on-tensor-core variant: P slots (2 for wide chunks, 4 for narrow
// ones) and as many B stages as fit, 2..8.
int k2t_pslots(int N) { return N > 128 ? 2 : 4; }

int k2t_stages(int N, int AS) {
  const int sb = (int)round_up(2 * N * 4 * 32 + 2 * 32 * 64, 1024);
  const int avail = 227 * 1024 - 1024 - AS * 2 * kTcRows * 32 * 4 - 2 * kTcRows * 64 - 512;
  int S = avail / sb;
  if (S > kTcMaxStages) S = kTcMaxStages;
  return S;
}

size_t k2t_smem_bytes(int N, int S, int AS) {
  const size_t sb = (size_t)round_up(2 * N * 4 * 32 + 2 * 32 * 64, 1024);
  return 1024 + (size_t)AS * 2 * kTcRows * 32 * 4 + 2 * kTcRows * 64 + (size_t)S * sb +
         (size_t)(2 * S + 2 * AS + 2 * kSBufs + 5) * 8 + 16;
}

template <bool CLAMP>
cudaError_t launch_k2t_t(const uint8_t* rimg, int64_t m, const uint8_t* cimg, const uint8_t* img,
                         int N, const K2Work& wk, float lam, const float* X, int64_t ldx, int k,
                         float* Y, int64_t ldy, float* part, int* status, cudaStream_t s,
                         const int* gate) {
  const int AS = k2t_pslots(N);
  const int S = k2t_stages(N, AS);
  size_t smem = k2t_smem_bytes(N, S, AS);
  if (S < 2 || smem > 227 * 1024) return cudaErrorInvalidConfiguration;
  if (smem <= kTmemExclusiveSmem) smem = kTmemExclusiveSmem + 1024;  // one TMEM owner per SM
  auto fn = k2t_matvec<CLAMP, 32>;
  cudaError_t e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
  const int64_t grid = wk.items < (int64_t)sm_count() ? wk.items : (int64_t)sm_count();
  fn<<<(unsigned)grid, kK2tThreads, smem, s>>>(rimg, m, cimg, img, N, S, AS, wk, lam, X, ldx, k, Y,
                                               ldy, part, status, gate);
  return cudaGetLastError();
}

}  // namespace

// RHS per CTA for k right-hand sides: a multiple of 32 (the MMA's N for M =
// 128 is a multiple of 16; each half of the epilogue reads 16-column groups),
// at most 256.
int k2_chunk_cols(int k) {
  const int kk = k < kTcMaxN ? k : kTcMaxN;
  return (int)round_up(kk, 32);
}

// Whether the multi-RHS kernel for chunks of N right-hand sides takes its
// logits from the tensor cores too (k2t; LAKER_K2_LOGITS_TC=1 or
// laker_set_variant per chunk-width class).  Off by default: measured on B200
// it matches k2_tc_matvec for narrow chunks (n = 50k, k = 16: 7.07 vs 7.31 ms)
// and is slower for wide ones (n = 20k, k = 256: 2.17 vs 1.49 ms); both are
// bound by their pipelines (mbarrier polling dominates the issued
// instructions), not by the entry arithmetic that k2t moves to the tensor
// cores.  The autotuner picks per class on the caller's sizes.
bool k2_logits_tc(int N) {
  const int which = N <= 32 ? LAKER_VARIANT_K2_LOGITS_N32
                            : (N <= 128 ? LAKER_VARIANT_K2_LOGITS_N128 : LAKER_VARIANT_K2_LOGITS_WIDE);
  return variant_get(which) == 1;
}

namespace {
int k2_tk_for(int N) { return k2_logits_tc(N) ? 32 : k2_tile_points(N); }
size_t k2_x_image_bytes(const K2Work& w, int N, int TK) {
  return (size_t)round_up((int64_t)((size_t)(w.chunks * w.ntiles) * (size_t)N * 8 * TK), 256);
}
}  // namespace

// Workspace of one multi-RHS product: the split X image, the segment
// partials when the column range is split, and (tensor-core logits) the
// operand images of the rows' and the points' embeddings.
size_t k2_image_bytes(int64_t m, int64_t n, int k) {
  const int N = k2_chunk_cols(k);
  const int TK = k2_tk_for(N);
  const K2Work w = k2_work(m, n, k, N, TK);
  size_t b = k2_x_image_bytes(w, N, TK);
  if (w.segs > 1) b += (size_t)round_up((int64_t)((size_t)w.segs * (size_t)m * (size_t)k * 4), 1024);
  if (k2_logits_tc(N)) b += k1t_image_bytes(m) + k1t_image_bytes(n);
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
                      int64_t ldy, uint8_t* img, int* status, cudaStream_t s, const int* gate) {
  const int N = k2_chunk_cols(k);
  const int TK = k2_tk_for(N);
  const K2Work wk = k2_work(m, n, k, N, TK);
  const size_t xbytes = k2_x_image_bytes(wk, N, TK);
  float* part = wk.segs > 1 ? reinterpret_cast<float*>(img + xbytes) : nullptr;
  const size_t pbytes =
      wk.segs > 1 ? (size_t)round_up((int64_t)((size_t)wk.segs * (size_t)m * (size_t)k * 4), 1024) : 0;
  {
    const int64_t total = wk.ntiles * TK * (int64_t)wk.chunks * N;
    int64_t g = ceil_div(total, 256);
    if (g > (int64_t)sm_count() * 16) g = (int64_t)sm_count() * 16;
    if (TK == 32)
      k2_pack_x<32><<<(unsigned)g, 256, 0, s>>>(X, n, ldx, k, N, wk.ntiles, img, gate);
    else
      k2_pack_x<16><<<(unsigned)g, 256, 0, s>>>(X, n, ldx, k, N, wk.ntiles, img, gate);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
  }
  const int dp = padded_dim(d);
  cudaError_t e = cudaErrorInvalidValue;
  if (k2_logits_tc(N)) {
    // operand images of the rows and of the points (one image for a square
    // product with the same embeddings)
    uint8_t* rimg = img + xbytes + pbytes;
    uint8_t* cimg = rimg;
    const int64_t rrows = round_up(m > 0 ? m : 1, 512), crows = round_up(n > 0 ? n : 1, 512);
    e = launch_k1t_pack(rows32, m, d, rimg, rrows, s);
    if (e == cudaSuccess && !(rows32 == cols32 && m == n)) {
      cimg = rimg + k1t_image_bytes(m);
      e = launch_k1t_pack(cols32, n, d, cimg, crows, s);
    }
    if (e == cudaSuccess)
      e = clamp ? launch_k2t_t<true>(rimg, m, cimg, img, N, wk, lam, X, ldx, k, Y, ldy, part, status, s, gate)
                : launch_k2t_t<false>(rimg, m, cimg, img, N, wk, lam, X, ldx, k, Y, ldy, part, status, s, gate);
  } else if (clamp) {
    LAKER_DISPATCH_TC(dp, e = (launch_k2_tk<DPv, true>(rows32, m, cols32, img, N, TK, wk, lam, X, ldx, k, Y, ldy, part, status, s, gate)));
  } else {
    LAKER_DISPATCH_TC(dp, e = (launch_k2_tk<DPv, false>(rows32, m, cols32, img, N, TK, wk, lam, X, ldx, k, Y, ldy, part, status, s, gate)));
  }
  if (e != cudaSuccess || wk.segs == 1) return e;
  int64_t g = ceil_div(m * (int64_t)k, 256);
  if (g > (int64_t)sm_count() * 16) g = (int64_t)sm_count() * 16;
  k2_reduce_kernel<<<(unsigned)g, 256, 0, s>>>(part, wk.segs, m, k, lam, X, ldx, Y, ldy, gate);
  return cudaGetLastError();
}

cudaError_t set_wait_limit_tc(unsigned long long ns) { return set_wait_limit_this_unit(ns); }

cudaError_t launch_pack_x32(const float* X, int64_t n, int64_t ldx, int k, int N, int64_t ntiles,
                            uint8_t* img, const int* gate, cudaStream_t s) {
  const int64_t total = ntiles * 32 * ceil_div(k, N) * N;
  int64_t g = ceil_div(total, 256);
  if (g > (int64_t)sm_count() * 16) g = (int64_t)sm_count() * 16;
  if (g < 1) g = 1;
  k2_pack_x<32><<<(unsigned)g, 256, 0, s>>>(X, n, ldx, k, N, ntiles, img, gate);
  return cudaGetLastError();
}

cudaError_t launch_seg_reduce(const float* part, int segs, int64_t m, int k, float lam,
                              const float* X, int64_t ldx, float* Y, int64_t ldy, const int* gate,
                              cudaStream_t s) {
  int64_t g = ceil_div(m * (int64_t)k, 256);
  if (g > (int64_t)sm_count() * 16) g = (int64_t)sm_count() * 16;
  if (g < 1) g = 1;
  k2_reduce_kernel<<<(unsigned)g, 256, 0, s>>>(part, segs, m, k, lam, X, ldx, Y, ldy, gate);
  return cudaGetLastError();
}

}  // namespace laker
