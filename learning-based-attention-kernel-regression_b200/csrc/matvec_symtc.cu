// Symmetric FP32 fused matvec with the logits on the tensor cores:
// y = lam x + exp(E E^T) x, each off-diagonal kernel entry evaluated once.
//
// Same work decomposition and partial-sum layout as the CUDA-core symmetric
// kernel (matvec_sym.cu): blocks of 512 points, block pairs (a, b), a <= b,
// row-major over the upper triangle, one 512-vector of row sums (double) and
// one of column sums (float) per pair, and the same fixed-order finish.  What
// changes is where the work runs:
//   * logits: the 512 x 512 Gram block of a pair is 4 row tiles x 8 column
//     slabs of tcgen05.mma kind::tf32 (M = 128, N = 64, K = 16: d padded to
//     16), split TF32 (E = E_hi + E_lo, three products E_hi E_hi + E_hi E_lo +
//     E_lo E_hi, ~2^-21 relative per term like FP32), accumulated in TMEM;
//     log2 e is folded into the row-side copy, so TMEM holds exp2 arguments;
//   * CUDA cores: per entry one MUFU ex2, one FFMA for the row sum and one
//     for the column sum; a column slab keeps the four row tiles in TMEM, so
//     a thread adds its four rows' column contributions in registers and the
//     warp reduce-scatter (shuffles) runs once per 4 x 32 rows.
// The per-entry CUDA-core work falls from d + 2 FMAs + 1 exp2 (logits on the
// FMA pipe) to 2 FMAs + 1 exp2: the kernel is bound by the MUFU ex2 rate.
//
// Operand image (k1t_pack): per 512-point block 128 KB, four variants of the
// block's points, 64 bytes (16 TF32) per point in the 64-byte-swizzled
// K-major layout the tensor core reads: rows scaled by log2 e (hi, lo), then
// columns unscaled (hi, lo).  One bulk copy brings a block's row operands
// (64 KB), one its column operands (64 KB).
// FP16 format (unclamped operators, LAKER_VARIANT_K1T_LOGITS = 1): six
// variants of 32 bytes (16 FP16) per point in the 32-byte-swizzled K-major
// layout, rows scaled by log2 e (H, L, Hs), then columns (H, L, Hs), with
// H = fp16(v), L = fp16((v - H) 2^12), Hs = fp16(H 2^-12); the logits are
// H H' + Hs L' + L Hs' (= H H' + H lo' + lo H'), three kind::f16 MMAs of K =
// 16 per row tile instead of six kind::tf32 MMAs of K = 8, half the operand
// bytes (48 KB per side) and the f16 tensor rate.
// Two-MMA FP16 format (the same, for at most 10 padded dimensions): four
// variants, V0 = [H | Hs_0..], V1 = [Hs_P.. | L], W0 = [H' | L'_0..],
// W1 = [L'_P.. | Hs'] (k1t_pack16x2_kernel), so that V0 W0 + V1 W1 gives the
// same three products in two MMAs (32 KB per side).
//
// Roles in a CTA of 576 threads (one CTA per SM: 512 TMEM columns, up to
// 221 KB of shared memory), no CTA-wide barrier in the main loop:
//   warps 0-15 epilogue: warp w reads TMEM lanes 32 (w & 3) .. + 31 (its rows
//             in each row tile) and 16 of a slab's 64 columns (column group
//             w >> 2); four epilogue warps per SM sub-partition hide the
//             TMEM-load and shuffle latencies.  Per pair, row sums and column
//             sums are combined over the warps in shared memory in a fixed
//             order and stored;
//   warp 16   copies: the row block's operands when the row block changes,
//             the column block's operands per pair (two stages);
//   warp 17   MMA (lane 0): per TMEM unit (UT row tiles of one slab), 6 MMAs
//             per row tile into one of 8 / UT buffers, committed to that
//             buffer's "full" barrier.
// Every wait is bounded; a timeout sets a shared abort flag that every role
// checks; the CTA then drains its copies and MMAs and frees TMEM.  The
// epilogue warps keep walking their pairs after an abort (without waits or
// TMEM reads) so that their named barriers always match.
#include <cuda_fp16.h>

#include <cstdlib>

#include "sym.cuh"
#include "tc.cuh"

namespace laker {
namespace {

constexpr int kTB = 512;                       // points per block
constexpr int kTRowTiles = kTB / 128;          // M = 128 row tiles per block
constexpr int kTSlabN = 64;                    // N of one MMA (columns per slab)
constexpr int kTSlabs = kTB / kTSlabN;         // column slabs per block
constexpr uint32_t kTRowBytes = 64;            // 16 TF32 per point
constexpr uint32_t kTVar = kTB * kTRowBytes;   // one operand variant of a block (32 KB)
constexpr uint32_t kTImgBlock = 4 * kTVar;     // image bytes per block (128 KB)
constexpr uint32_t kTHalf = 2 * kTVar;         // hi + lo of one side (64 KB)
constexpr uint32_t kTSBO = 8 * kTRowBytes;     // 8-row core group
constexpr uint32_t kTLayout = 4;               // SWIZZLE_64B
constexpr int kTEpi = 512;                     // epilogue threads (16 warps)
constexpr int kTThreads = kTEpi + 64;          // + copy warp + MMA warp
constexpr int kTCopyWarp = kTEpi / 32, kTMmaWarp = kTEpi / 32 + 1;
constexpr int kTNcg = 4;                       // column groups (warps per row quadrant)
constexpr int kTCW = kTSlabN / kTNcg;          // columns per warp per slab (16)
static_assert(kTB == 512, "the finish and the engine use 512-point blocks");
// FP16 image format
constexpr uint32_t kTRowBytes16 = 32;              // 16 FP16 per point
constexpr uint32_t kTVar16 = kTB * kTRowBytes16;   // one FP16 variant of a block (16 KB)
constexpr uint32_t kTHalf16 = 3 * kTVar16;         // H, L, Hs of one side (48 KB)
constexpr uint32_t kTSBO16 = 8 * kTRowBytes16;     // 8-row core group
constexpr uint32_t kTLayout16 = 6;                 // SWIZZLE_32B
static_assert(2 * kTHalf16 <= kTImgBlock, "the FP16 image fits the block's 128 KB");

// Plan for TMEM units of UT row tiles (UT x 64 accumulator columns, 512 / (64
// UT) buffers): UT = 4 holds a whole slab per buffer (2 buffers), UT = 2 half
// a slab (4 buffers, more MMA look-ahead, twice the handshakes).  Offsets are
// from a 1024-byte aligned base.
template <int UT, int FMT>
struct K1tCfg {
  static_assert(UT == 2 || UT == 4, "row tiles per unit");
  static constexpr int kBufs = 8 / UT;
  static constexpr uint32_t kHalf = FMT == kK1tF16 ? kTHalf16
                                    : FMT == kK1tF16x2 ? 2 * kTVar16
                                                       : kTHalf;  // one side of a block
  // mbarrier slots: row operands full / empty, column stages full [2] /
  // empty [2], TMEM buffers full [kBufs] / empty [kBufs], MMA drain
  static constexpr int kBarAFull = 0, kBarAEmpty = 1, kBarBFull = 2, kBarBEmpty = 4,
                       kBarAccFull = 6, kBarAccEmpty = kBarAccFull + kBufs,
                       kBarDrain = kBarAccEmpty + kBufs, kNumBars = kBarDrain + 1;
  static constexpr uint32_t kOffA = 0;                        // row operands (hi | lo)
  static constexpr uint32_t kOffB = kOffA + kHalf;            // 2 stages of column operands
  static constexpr uint32_t kOffXb = kOffB + 2 * kHalf;       // 2 x 512 floats: x of the column block
  static constexpr uint32_t kOffRow = kOffXb + 2 * kTB * 4;   // 4 x 512 doubles: row sums per column group
  static constexpr uint32_t kOffCol = kOffRow + kTNcg * kTB * 8;  // 4 x 512 floats: column sums per row quadrant
  static constexpr uint32_t kOffBar = kOffCol + 4 * kTB * 4;  // barriers, TMEM slot, abort flag
  static constexpr uint32_t kSmemBytes = kOffBar + kNumBars * 8 + 16 + 1024;  // + alignment slack
  static_assert(kSmemBytes <= 227 * 1024, "shared memory budget");
  static_assert(kSmemBytes > kTmemExclusiveSmem, "one TMEM-owning CTA per SM");
};

// Byte offset of TF32 element k of point row r inside a block variant
// (64-byte swizzle: 16-byte chunk index XOR bits 1-2 of the row).
__host__ __device__ inline uint32_t k1t_offset(uint32_t r, uint32_t k) {
  return r * kTRowBytes + ((((k >> 2) ^ ((r >> 1) & 3u)) << 4)) + (k & 3u) * 4u;
}

// Byte offset of FP16 element k of point row r inside an FP16 block variant
// (32-byte swizzle: 16-byte chunk index XOR bit 2 of the row).
__host__ __device__ inline uint32_t k1t16_offset(uint32_t r, uint32_t k) {
  return r * kTRowBytes16 + ((((k >> 3) ^ ((r >> 2) & 1u)) << 4)) + (k & 7u) * 2u;
}

__device__ __forceinline__ void split_f16(float v, uint16_t& h, uint16_t& l, uint16_t& hs) {
  const __half hh = __float2half_rn(v);
  const float hf = __half2float(hh);
  h = __half_as_ushort(hh);
  l = __half_as_ushort(__float2half_rn((v - hf) * 4096.0f));
  hs = __half_as_ushort(__float2half_rn(hf * (1.0f / 4096.0f)));
}

// FP16-format image of `rows` points: one thread per point and 8-dimension
// chunk (one 16-byte chunk of each of the six variants).
__global__ void k1t_pack16_kernel(const float* __restrict__ packed32, int DP, int64_t npts,
                                  int64_t rows, uint8_t* __restrict__ img) {
  for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < rows * 2;
       e += (int64_t)gridDim.x * blockDim.x) {
    const int64_t r = e >> 1;
    const int c = (int)(e & 1);
    uint16_t h[6][8];
#pragma unroll
    for (int u = 0; u < 8; ++u) {
      const int k = 8 * c + u;
      const float v = (r < npts && k < DP) ? packed32[(r >> 1) * (2 * DP) + 2 * k + (r & 1)] : 0.0f;
      split_f16(v * kLog2e, h[0][u], h[1][u], h[2][u]);
      split_f16(v, h[3][u], h[4][u], h[5][u]);
    }
    const int64_t blk = r / kTB;
    const uint32_t rr = (uint32_t)(r - blk * kTB);
    uint8_t* base = img + blk * (int64_t)kTImgBlock + k1t16_offset(rr, 8u * c);
#pragma unroll
    for (int vv = 0; vv < 6; ++vv) {
      uint4 q;
      q.x = (uint32_t)h[vv][0] | ((uint32_t)h[vv][1] << 16);
      q.y = (uint32_t)h[vv][2] | ((uint32_t)h[vv][3] << 16);
      q.z = (uint32_t)h[vv][4] | ((uint32_t)h[vv][5] << 16);
      q.w = (uint32_t)h[vv][6] | ((uint32_t)h[vv][7] << 16);
      *reinterpret_cast<uint4*>(base + vv * kTVar16) = q;
    }
  }
}

// Two-MMA FP16 image (DP <= 10) of `rows` points: one thread per point.
// Per side two variants of 16 FP16: V0 = [H_0..H_DP-1 | Hs_0..Hs_P-1] and
// V1 = [Hs_P..Hs_DP-1 | L_0..L_DP-1 | 0 ...] for the row side (scaled by
// log2 e), W0 = [H' | L'_0..L'_P-1] and W1 = [L'_P..L'_DP-1 | Hs' | 0 ...]
// for the column side, with P = min(16 - DP, DP): V0 W0 + V1 W1 =
// H H' + Hs L' + L Hs', the three products of the split-FP16 format.
__global__ void k1t_pack16x2_kernel(const float* __restrict__ packed32, int DP, int64_t npts,
                                    int64_t rows, uint8_t* __restrict__ img) {
  for (int64_t r = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; r < rows;
       r += (int64_t)gridDim.x * blockDim.x) {
    uint16_t hr[3][16], hc[3][16];  // [H, L, Hs] of the row and column sides
#pragma unroll
    for (int k = 0; k < 16; ++k) {
      const float v = (r < npts && k < DP) ? packed32[(r >> 1) * (2 * DP) + 2 * k + (r & 1)] : 0.0f;
      split_f16(v * kLog2e, hr[0][k], hr[1][k], hr[2][k]);
      split_f16(v, hc[0][k], hc[1][k], hc[2][k]);
    }
    const int P = (16 - DP) < DP ? 16 - DP : DP;
    uint16_t out[4][16];
#pragma unroll
    for (int k = 0; k < 16; ++k) {
      // V0 / W0: H, then the first P correction terms in H's padding
      const bool lead = k < DP;
      const int kp = k - DP;  // index into the padding
      out[0][k] = lead ? hr[0][k] : (kp < P ? hr[2][kp] : 0);
      out[2][k] = lead ? hc[0][k] : (kp < P ? hc[1][kp] : 0);
      // V1 / W1: the remaining DP - P correction terms, then the second product
      const int rest = DP - P;
      const int k2 = k - rest;
      out[1][k] = k < rest ? hr[2][P + k] : (k2 < DP ? hr[1][k2] : 0);
      out[3][k] = k < rest ? hc[1][P + k] : (k2 < DP ? hc[2][k2] : 0);
    }
    const int64_t blk = r / kTB;
    const uint32_t rr = (uint32_t)(r - blk * kTB);
    uint8_t* base = img + blk * (int64_t)kTImgBlock;
#pragma unroll
    for (int vv = 0; vv < 4; ++vv) {
      // variants 0, 1 on the row side; 2, 3 start the column side (2 * kTVar16)
      uint8_t* vb = base + vv * kTVar16;
#pragma unroll
      for (int c = 0; c < 2; ++c) {
        uint4 q;
        q.x = (uint32_t)out[vv][8 * c + 0] | ((uint32_t)out[vv][8 * c + 1] << 16);
        q.y = (uint32_t)out[vv][8 * c + 2] | ((uint32_t)out[vv][8 * c + 3] << 16);
        q.z = (uint32_t)out[vv][8 * c + 4] | ((uint32_t)out[vv][8 * c + 5] << 16);
        q.w = (uint32_t)out[vv][8 * c + 6] | ((uint32_t)out[vv][8 * c + 7] << 16);
        *reinterpret_cast<uint4*>(vb + k1t16_offset(rr, 8u * c)) = q;
      }
    }
  }
}

// Image of `rows` points (a multiple of 512) from the packed FP32 layout
// (point pairs interleaved, DP floats per point; see pack.cu); points at or
// past npts and dimensions at or past DP are zero.
__global__ void k1t_pack_kernel(const float* __restrict__ packed32, int DP, int64_t npts,
                                int64_t rows, uint8_t* __restrict__ img) {
  for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < rows * 4;
       e += (int64_t)gridDim.x * blockDim.x) {
    const int64_t r = e >> 2;
    const int c = (int)(e & 3);
    float v[4];
#pragma unroll
    for (int u = 0; u < 4; ++u) {
      const int k = 4 * c + u;
      v[u] = (r < npts && k < DP) ? packed32[(r >> 1) * (2 * DP) + 2 * k + (r & 1)] : 0.0f;
    }
    uint4 ahi, alo, bhi, blo;
    uint32_t* pah = &ahi.x;
    uint32_t* pal = &alo.x;
    uint32_t* pbh = &bhi.x;
    uint32_t* pbl = &blo.x;
#pragma unroll
    for (int u = 0; u < 4; ++u) {
      const float a = v[u] * kLog2e;
      pah[u] = to_tf32(a);
      pal[u] = to_tf32(a - __uint_as_float(pah[u]));
      pbh[u] = to_tf32(v[u]);
      pbl[u] = to_tf32(v[u] - __uint_as_float(pbh[u]));
    }
    const int64_t blk = r / kTB;
    const uint32_t rr = (uint32_t)(r - blk * kTB);
    uint8_t* base = img + blk * (int64_t)kTImgBlock + k1t_offset(rr, 4u * c);
    *reinterpret_cast<uint4*>(base) = ahi;
    *reinterpret_cast<uint4*>(base + kTVar) = alo;
    *reinterpret_cast<uint4*>(base + 2 * kTVar) = bhi;
    *reinterpret_cast<uint4*>(base + 3 * kTVar) = blo;
  }
}

// A CTA's walk over its pairs (single instance or the running instances of
// a batch).  `slot` is the pair's index in the partial arrays.
struct PairWalk {
  int64_t p, p_end;
  int j;
  int64_t a, b;
  int64_t nb, npts, seg, pstart, pend, gp0;

  template <bool BATCHED>
  __device__ __forceinline__ void load_inst(const SymPlan& sp, const BatchMap& bm, int64_t n) {
    if (BATCHED) {
      const SlotInfo& si = bm.slots[bm.act_inst[j]];
      nb = si.nblk;
      npts = si.npts;
      seg = si.seg;
      pstart = bm.act_ps[j];
      pend = bm.act_ps[j + 1];
      gp0 = si.pair_start;
    } else {
      nb = sp.nb;
      npts = n;
      seg = 0;
      pstart = 0;
      pend = sp.npairs;
      gp0 = 0;
    }
  }
  // place on pair p (moving to the instance that holds it)
  template <bool BATCHED>
  __device__ __forceinline__ bool settle(const SymPlan& sp, const BatchMap& bm, int64_t n) {
    if (p >= p_end) return false;
    if (BATCHED) {
      while (p >= pend) {
        ++j;
        load_inst<BATCHED>(sp, bm, n);
      }
    }
    sym_pair_coords(p - pstart, nb, &a, &b);
    return true;
  }
  template <bool BATCHED>
  __device__ __forceinline__ bool next(const SymPlan& sp, const BatchMap& bm, int64_t n) {
    ++p;
    if (p >= p_end) return false;
    if (p < pend) {
      if (++b >= nb) {
        ++a;
        b = a;
      }
      return true;
    }
    return settle<BATCHED>(sp, bm, n);
  }
  __device__ __forceinline__ int64_t slot() const { return gp0 + p - pstart; }
  // global image blocks of the pair's row and column blocks
  __device__ __forceinline__ int64_t row_block() const { return seg / kTB + a; }
  __device__ __forceinline__ int64_t col_block() const { return seg / kTB + b; }
  // column slabs holding points
  __device__ __forceinline__ int slabs() const {
    const int64_t rem = npts - b * kTB;
    const int64_t s = (rem + kTSlabN - 1) / kTSlabN;
    return s < kTSlabs ? (int)s : kTSlabs;
  }
};

// Named barrier 1 over the N epilogue threads.
template <int N>
__device__ __forceinline__ void epi_bar_sync() {
  asm volatile("bar.sync 1, %0;" ::"n"(N) : "memory");
}

template <int UT, int FMT, bool CLAMP, bool BATCHED>
__global__ void __launch_bounds__(kTThreads, 1)
    k1t_matvec(const uint8_t* __restrict__ img, int64_t n, const float* __restrict__ x,
               float* __restrict__ colpart, double* __restrict__ rowpart, SymPlan sp, BatchMap bm,
               int* status, const int* gate) {
  using Cfg = K1tCfg<UT, FMT>;
  constexpr bool F16 = FMT != kK1tTf32;   // both FP16 formats
  constexpr bool F16X2 = FMT == kK1tF16x2;  // the two-MMA FP16 format
  constexpr int CW = kTCW;
  constexpr int kTBufs = Cfg::kBufs;
  if (gate && *gate == 0) return;
  extern __shared__ __align__(1024) uint8_t smem_raw[];
  uint8_t* sm = reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
  float* sXb = reinterpret_cast<float*>(sm + Cfg::kOffXb);
  double* sRow = reinterpret_cast<double*>(sm + Cfg::kOffRow);
  float* sCol = reinterpret_cast<float*>(sm + Cfg::kOffCol);
  uint64_t* bars = reinterpret_cast<uint64_t*>(sm + Cfg::kOffBar);
  uint64_t* a_full = bars + Cfg::kBarAFull;
  uint64_t* a_empty = bars + Cfg::kBarAEmpty;
  uint64_t* b_full = bars + Cfg::kBarBFull;        // [2]
  uint64_t* b_empty = bars + Cfg::kBarBEmpty;      // [2]
  uint64_t* acc_full = bars + Cfg::kBarAccFull;    // [kTBufs]
  uint64_t* acc_empty = bars + Cfg::kBarAccEmpty;  // [kTBufs]
  uint64_t* drain = bars + Cfg::kBarDrain;
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(bars + Cfg::kNumBars);  // after the last barrier
  volatile int* abort = reinterpret_cast<volatile int*>(tmem_slot + 1);

  // ---- this CTA's pair range ------------------------------------------------
  const int64_t c = blockIdx.x;
  PairWalk w0;
  w0.j = 0;
  if (BATCHED) {
    const int nact = *bm.act_count;
    if (nact <= 0) return;
    const int64_t total = bm.act_ps[nact];
    const int64_t q = total / gridDim.x, rem = total % gridDim.x;
    w0.p = c * q + (c < rem ? c : rem);
    w0.p_end = w0.p + q + (c < rem ? 1 : 0);
    if (w0.p >= w0.p_end) return;
    int lo = 0, hi = nact - 1;
    while (lo < hi) {
      const int mid = (lo + hi + 1) >> 1;
      if (bm.act_ps[mid] <= w0.p) lo = mid; else hi = mid - 1;
    }
    w0.j = lo;
  } else {
    w0.p = c * sp.q + (c < sp.rem ? c : sp.rem);
    w0.p_end = w0.p + sp.q + (c < sp.rem ? 1 : 0);
    if (w0.p >= w0.p_end) return;
  }
  w0.load_inst<BATCHED>(sp, bm, n);
  if (!w0.settle<BATCHED>(sp, bm, n)) return;  // uniform over the CTA

  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;"
                 :
                 : "r"(smem_u32(tmem_slot)), "r"(512u));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
  }
  if (tid == 0) {
    mbar_init(a_full, 1);
    mbar_init(a_empty, 1);
    for (int i = 0; i < 2; ++i) {
      mbar_init(&b_full[i], 1);
      mbar_init(&b_empty[i], 1);
    }
    for (int i = 0; i < kTBufs; ++i) {
      mbar_init(&acc_full[i], 1);
      mbar_init(&acc_empty[i], kTEpi);
    }
    mbar_init(drain, 1);
    *abort = 0;
    mbar_fence_init();
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem_base = *tmem_slot;

  int64_t b_issued = 0, a_issued = 0;  // copy role
  bool mma_any = false;                // MMA role
  if (warp == kTCopyWarp) {
    // ---- copies ---------------------------------------------------------------
    if (lane == 0) {
      PairWalk wk = w0;
      int64_t prev_a = -1;
      bool more = true;
      while (more && !*abort) {
        const int64_t ab = wk.row_block();
        if (ab != prev_a) {
          if (!wait_or_abort(a_empty, (uint32_t)((a_issued & 1) ^ 1), status, abort)) break;
          mbar_arrive_expect_tx(a_full, Cfg::kHalf);
          bulk_g2s(sm + Cfg::kOffA, img + ab * (int64_t)kTImgBlock, Cfg::kHalf, a_full);
          ++a_issued;
          prev_a = ab;
        }
        const int bs = (int)(b_issued & 1);
        if (!wait_or_abort(&b_empty[bs], (uint32_t)(((b_issued >> 1) & 1) ^ 1), status, abort)) break;
        mbar_arrive_expect_tx(&b_full[bs], Cfg::kHalf);
        bulk_g2s(sm + Cfg::kOffB + bs * Cfg::kHalf,
                 img + wk.col_block() * (int64_t)kTImgBlock + Cfg::kHalf, Cfg::kHalf, &b_full[bs]);
        ++b_issued;
        more = wk.next<BATCHED>(sp, bm, n);
      }
    }
  } else if (warp == kTMmaWarp) {
    // ---- MMA issue --------------------------------------------------------------
    if (lane == 0) {
      const uint32_t idesc = F16 ? f16_idesc_mn(128, kTSlabN) : tf32_idesc_mn(128, kTSlabN);
      // descriptors built once: the start-address field holds address >> 4,
      // so an operand offset is added to the descriptor as offset >> 4 (no
      // carry: shared addresses stay below 256 KB)
      constexpr uint32_t kRB = F16 ? kTRowBytes16 : kTRowBytes;
      const uint64_t a_hi0 = kmajor_desc_raw(smem_u32(sm + Cfg::kOffA), F16 ? kTSBO16 : kTSBO,
                                             F16 ? kTLayout16 : kTLayout);
      const uint64_t b_hi0 = kmajor_desc_raw(smem_u32(sm + Cfg::kOffB), F16 ? kTSBO16 : kTSBO,
                                             F16 ? kTLayout16 : kTLayout);
      constexpr uint64_t kRowTileStep = (128u * kRB) >> 4;           // next row tile
      constexpr uint64_t kSlabStep = (kTSlabN * kRB) >> 4;           // next column slab
      constexpr uint64_t kLoStep = (F16 ? kTVar16 : kTVar) >> 4;     // next variant
      constexpr uint64_t kStageStep = Cfg::kHalf >> 4;               // next column stage
      constexpr uint64_t kKStep = 32u >> 4;                          // TF32: second 8-wide K step
      PairWalk wk = w0;
      int64_t prev_a = -1, na = 0, pc = 0, g = 0;
      bool more = true;
      while (more && !*abort) {
        const int64_t ab = wk.row_block();
        if (ab != prev_a) {
          if (!wait_or_abort(a_full, (uint32_t)(na & 1), status, abort)) break;
          ++na;
          prev_a = ab;
        }
        const int bs = (int)(pc & 1);
        if (!wait_or_abort(&b_full[bs], (uint32_t)((pc >> 1) & 1), status, abort)) break;
        tc_fence_after();
        const uint64_t b_stage = b_hi0 + (uint64_t)bs * kStageStep;
        const int nsl = wk.slabs();
        bool ok = true;
        // units (slab s, row tiles UT hp .. UT hp + UT - 1), one TMEM buffer each
        constexpr int kUnitsPerSlab = kTRowTiles / UT;
        for (int un = 0; un < kUnitsPerSlab * nsl; ++un, ++g) {
          const int s = un / kUnitsPerSlab, hp = un % kUnitsPerSlab;
          const int buf = (int)(g % kTBufs);
          if (!wait_or_abort(&acc_empty[buf], (uint32_t)(((g / kTBufs) & 1) ^ 1), status, abort)) {
            ok = false;
            break;
          }
          tc_fence_after();
          const uint64_t bhi = b_stage + (uint64_t)s * kSlabStep, blo = bhi + kLoStep;
#pragma unroll
          for (int r2 = 0; r2 < UT; ++r2) {
            const int rt = UT * hp + r2;
            const uint32_t d = tmem_base + (uint32_t)(buf * (UT * kTSlabN) + r2 * kTSlabN);
            const uint64_t ahi = a_hi0 + (uint64_t)rt * kRowTileStep, alo = ahi + kLoStep;
            if constexpr (F16X2) {
              // V0 W0 + V1 W1 = H H' + Hs L' + L Hs'
              mma_f16(d, ahi, bhi, idesc, 0u);
              mma_f16(d, alo, blo, idesc, 1u);
            } else if constexpr (F16) {
              // variants H, L, Hs: H H' + Hs L' + L Hs'
              mma_f16(d, ahi, bhi, idesc, 0u);
              mma_f16(d, ahi + 2 * kLoStep, blo, idesc, 1u);
              mma_f16(d, alo, bhi + 2 * kLoStep, idesc, 1u);
            } else {
              mma_tf32(d, ahi, bhi, idesc, 0u);
              mma_tf32(d, ahi, blo, idesc, 1u);
              mma_tf32(d, alo, bhi, idesc, 1u);
              mma_tf32(d, ahi + kKStep, bhi + kKStep, idesc, 1u);
              mma_tf32(d, ahi + kKStep, blo + kKStep, idesc, 1u);
              mma_tf32(d, alo + kKStep, bhi + kKStep, idesc, 1u);
            }
          }
          mma_any = true;
          mma_commit(&acc_full[buf]);
        }
        if (!ok) break;
        mma_commit(&b_empty[bs]);
        ++pc;
        more = wk.next<BATCHED>(sp, bm, n);
        if (!more || wk.row_block() != prev_a) mma_commit(a_empty);
      }
    }
  } else {
    // ---- epilogue (warps 0 .. 15) -------------------------------------------------
    const int q = warp & 3, cg = warp >> 2;
    const uint32_t lane_base = (uint32_t)(q * 32) << 16;
    constexpr int XPT = kTB / kTEpi;  // x values of the column block per thread
    PairWalk wk = w0;
    int64_t pc = 0, g = 0;
    bool dead = false;  // warp-uniform: stop waiting and reading TMEM after an abort
    // x of the pair's column block (XPT per thread) and of this thread's rows,
    // loaded one pair ahead
    auto load_x = [&](const PairWalk& w, float (&xbv)[XPT], float (&xav)[kTRowTiles]) {
#pragma unroll
      for (int t = 0; t < XPT; ++t) {
        const int64_t li = w.b * kTB + tid + t * kTEpi;
        xbv[t] = li < w.npts ? x[w.seg + li] : 0.0f;
      }
#pragma unroll
      for (int rt = 0; rt < kTRowTiles; ++rt) {
        const int64_t li = w.a * kTB + rt * 128 + q * 32 + lane;
        xav[rt] = li < w.npts ? x[w.seg + li] : 0.0f;
      }
    };
    float xb_next[XPT], xa_next[kTRowTiles];
    load_x(wk, xb_next, xa_next);
    bool more = true;
    while (more) {
      const int64_t slot = wk.slot();
      const bool off = wk.a != wk.b;
      const int nsl = wk.slabs();
      float* xb = sXb + (pc & 1) * kTB;
#pragma unroll
      for (int t = 0; t < XPT; ++t) xb[tid + t * kTEpi] = xb_next[t];
      float xa[kTRowTiles];
#pragma unroll
      for (int rt = 0; rt < kTRowTiles; ++rt) xa[rt] = xa_next[rt];
      {
        PairWalk nx = wk;
        if (nx.next<BATCHED>(sp, bm, n)) load_x(nx, xb_next, xa_next);
      }
      epi_bar_sync<kTEpi>();
      // a thread's share of a row sum (128 entries of the pair) in FP32, like
      // the column sums (512 rows per pair), widened to FP64 once per pair:
      // the per-chunk F2F + DADD chain cost 5 % of the kernel
      float racc[kTRowTiles];
#pragma unroll
      for (int rt = 0; rt < kTRowTiles; ++rt) racc[rt] = 0.0f;
      for (int s = 0; s < nsl; ++s) {
        float xj[CW];
        {
          const float4* xs = reinterpret_cast<const float4*>(xb + s * kTSlabN + cg * CW);
#pragma unroll
          for (int u = 0; u < CW / 4; ++u) {
            const float4 t = xs[u];
            xj[4 * u] = t.x;
            xj[4 * u + 1] = t.y;
            xj[4 * u + 2] = t.z;
            xj[4 * u + 3] = t.w;
          }
        }
        float2 cacc[CW / 2];
#pragma unroll
        for (int u = 0; u < CW / 2; ++u) cacc[u] = make_float2(0.0f, 0.0f);
        // one tile's entries: exp2, row sum (packed pairs, fixed order) and
        // column contributions (packed FFMA2: half the FMA-pipe instructions)
        auto consume = [&](const float (&v)[CW], int rt) {
          float2 ra = make_float2(0.0f, 0.0f);
          const float2 xr = make_float2(xa[rt], xa[rt]);
#pragma unroll
          for (int u = 0; u < CW / 2; ++u) {
            float2 e;
            e.x = ex2_approx(CLAMP ? fminf(v[2 * u], kClampLog2) : v[2 * u]);
            e.y = ex2_approx(CLAMP ? fminf(v[2 * u + 1], kClampLog2) : v[2 * u + 1]);
            ra = __ffma2_rn(e, make_float2(xj[2 * u], xj[2 * u + 1]), ra);
            cacc[u] = __ffma2_rn(e, xr, cacc[u]);
          }
          racc[rt] += ra.x + ra.y;
        };
#pragma unroll
        for (int hp = 0; hp < kTRowTiles / UT; ++hp, ++g) {
          const int buf = (int)(g % kTBufs);
          if (!dead)
            dead = !warp_wait_or_abort(&acc_full[buf], (uint32_t)((g / kTBufs) & 1), status, abort, lane);
          if (!dead) {
            tc_fence_after();
            const uint32_t t0 = tmem_base + lane_base + (uint32_t)(buf * (UT * kTSlabN) + cg * CW);
            // tiles in pairs under one TMEM wait; the buffer is released after
            // its last load, before the last pair is consumed
#pragma unroll
            for (int r2 = 0; r2 < UT; r2 += 2) {
              float va[16], vb[16];
              tmem_ld16x2(t0 + (uint32_t)(r2 * kTSlabN), t0 + (uint32_t)((r2 + 1) * kTSlabN), va, vb);
              if (r2 + 2 == UT) {
                tc_fence_before();
                mbar_arrive(&acc_empty[buf]);
              }
              consume(va, UT * hp + r2);
              consume(vb, UT * hp + r2 + 1);
            }
          }
        }
        if (off) {
          // warp sums over its 4 x 32 rows; CW = 16: lanes 2c, 2c + 1 hold column c
          float cv[CW];
#pragma unroll
          for (int u = 0; u < CW / 2; ++u) {
            cv[2 * u] = cacc[u].x;
            cv[2 * u + 1] = cacc[u].y;
          }
          const float cs = warp_reduce_scatter<CW>(cv, lane);
          if (CW == 32 || (lane & 1) == 0)
            sCol[q * kTB + s * kTSlabN + cg * CW + (CW == 32 ? lane : (lane >> 1))] = cs;
        }
      }
      if (off && (CW == 32 || (lane & 1) == 0)) {
        for (int s = nsl; s < kTSlabs; ++s)
          sCol[q * kTB + s * kTSlabN + cg * CW + (CW == 32 ? lane : (lane >> 1))] = 0.0f;
      }
#pragma unroll
      for (int rt = 0; rt < kTRowTiles; ++rt) sRow[cg * kTB + rt * 128 + q * 32 + lane] = (double)racc[rt];
      epi_bar_sync<kTEpi>();
      for (int j = tid; j < kTB; j += kTEpi) {
        double r = sRow[j];
#pragma unroll
        for (int c = 1; c < kTNcg; ++c) r += sRow[c * kTB + j];
        rowpart[slot * kTB + j] = r;
        if (off)
          colpart[slot * kTB + j] = ((sCol[j] + sCol[kTB + j]) + sCol[2 * kTB + j]) + sCol[3 * kTB + j];
      }
      ++pc;
      more = wk.next<BATCHED>(sp, bm, n);
    }
  }

  // ---- teardown: every role has left its loop ---------------------------------
  __syncthreads();
  if (*abort) {
    // bounded drains of the copies in flight and of the MMAs issued
    if (warp == kTCopyWarp && lane == 0) {
      if (a_issued > 0) mbar_wait_drain(a_full, (uint32_t)((a_issued - 1) & 1), status);
      for (int64_t gg = b_issued > 2 ? b_issued - 2 : 0; gg < b_issued; ++gg)
        mbar_wait_drain(&b_full[gg & 1], (uint32_t)((gg >> 1) & 1), status);
    }
    if (warp == kTMmaWarp && lane == 0 && mma_any) {
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

template <int UT, int FMT, bool CLAMP, bool BATCHED>
cudaError_t launch_k1t_t(const uint8_t* img, int64_t n, const float* x, double* rowpart,
                         float* colpart, const SymPlan& sp, const BatchMap& bm, int* status,
                         const int* gate, cudaStream_t s) {
  using Cfg = K1tCfg<UT, FMT>;
  static bool attr = false;
  if (!attr) {
    const cudaError_t e = cudaFuncSetAttribute(k1t_matvec<UT, FMT, CLAMP, BATCHED>,
                                               cudaFuncAttributeMaxDynamicSharedMemorySize,
                                               (int)Cfg::kSmemBytes);
    if (e != cudaSuccess) return e;
    attr = true;
  }
  k1t_matvec<UT, FMT, CLAMP, BATCHED><<<sp.grid, kTThreads, Cfg::kSmemBytes, s>>>(
      img, n, x, colpart, rowpart, sp, bm, status, gate);
  return cudaGetLastError();
}

// Row tiles per TMEM unit: 4 (default) or 2 (LAKER_K1T_UNIT=2 or
// laker_set_variant).
int k1t_unit_tiles() { return variant_get(LAKER_VARIANT_K1T_UNIT); }

template <bool CLAMP, bool BATCHED>
cudaError_t launch_k1t_ut(const uint8_t* img, int64_t n, const float* x, double* rowpart,
                          float* colpart, const SymPlan& sp, const BatchMap& bm, int* status,
                          const int* gate, cudaStream_t s, int fmt) {
  if (fmt == kK1tF16 || fmt == kK1tF16x2) {
    // FP16 operands only for unclamped operators (|e_k| < 9: no overflow)
    if (CLAMP) return cudaErrorInvalidValue;
    if (fmt == kK1tF16x2)
      return launch_k1t_t<4, kK1tF16x2, false, BATCHED>(img, n, x, rowpart, colpart, sp, bm,
                                                         status, gate, s);
    return launch_k1t_t<4, kK1tF16, false, BATCHED>(img, n, x, rowpart, colpart, sp, bm, status,
                                                     gate, s);
  }
  return k1t_unit_tiles() == 2
             ? launch_k1t_t<2, kK1tTf32, CLAMP, BATCHED>(img, n, x, rowpart, colpart, sp, bm, status, gate, s)
             : launch_k1t_t<4, kK1tTf32, CLAMP, BATCHED>(img, n, x, rowpart, colpart, sp, bm, status, gate, s);
}

}  // namespace

bool k1t_enabled(int d) {
  static int v = -1;
  if (v < 0) {
    const char* e = getenv("LAKER_K1_TC");
    v = (e && e[0] == '0') ? 0 : 1;
  }
  return v == 1 && d >= 1 && d <= 16;
}

int k1t_format(int clamp, int d) {
  if (clamp || variant_get(LAKER_VARIANT_K1T_LOGITS) != 1) return kK1tTf32;
  return padded_dim(d) <= 10 ? kK1tF16x2 : kK1tF16;
}

size_t k1t_image_bytes(int64_t points) {
  const int64_t nb = points > 0 ? ceil_div(points, kTB) : 1;
  return (size_t)nb * kTImgBlock;
}

SymPlan k1t_plan_pairs(int64_t nb, int64_t npairs) {
  SymPlan sp{};
  sp.B = kTB;
  sp.nb = nb;
  sp.npairs = npairs;
  const int64_t slots = sm_count();
  sp.grid = (int)(npairs < slots ? (npairs > 0 ? npairs : 1) : slots);
  sp.q = npairs / sp.grid;
  sp.rem = npairs % sp.grid;
  sp.cfg = 1;
  return sp;
}

SymPlan k1t_plan(int64_t n) {
  const int64_t nb = n > 0 ? ceil_div(n, kTB) : 1;
  return k1t_plan_pairs(nb, nb * (nb + 1) / 2);
}

cudaError_t launch_k1t_pack(const float* packed32, int64_t npts, int d, uint8_t* img, int64_t rows,
                            cudaStream_t s, int fmt) {
  if (rows % kTB != 0 || d < 1 || d > 16 || (fmt != kK1tTf32 && fmt != kK1tF16 && fmt != kK1tF16x2))
    return cudaErrorInvalidValue;
  if (fmt == kK1tF16x2 && padded_dim(d) > 10) return cudaErrorInvalidValue;
  const int per_point = fmt == kK1tF16 ? 2 : fmt == kK1tF16x2 ? 1 : 4;  // threads per point
  int g = (int)ceil_div(rows * per_point, 256);
  if (g > sm_count() * 8) g = sm_count() * 8;
  if (g < 1) g = 1;
  if (fmt == kK1tF16x2)
    k1t_pack16x2_kernel<<<g, 256, 0, s>>>(packed32, padded_dim(d), npts, rows, img);
  else if (fmt == kK1tF16)
    k1t_pack16_kernel<<<g, 256, 0, s>>>(packed32, padded_dim(d), npts, rows, img);
  else
    k1t_pack_kernel<<<g, 256, 0, s>>>(packed32, padded_dim(d), npts, rows, img);
  return cudaGetLastError();
}

cudaError_t launch_k1t(const uint8_t* img, int64_t n, int clamp, const float* x, double* rowpart,
                       float* colpart, const SymPlan& sp, int* status, const int* gate,
                       cudaStream_t s, int fmt) {
  const BatchMap none{};
  return clamp ? launch_k1t_ut<true, false>(img, n, x, rowpart, colpart, sp, none, status, gate, s, fmt)
               : launch_k1t_ut<false, false>(img, n, x, rowpart, colpart, sp, none, status, gate, s, fmt);
}

cudaError_t launch_k1t_batched(const uint8_t* img, int clamp, const float* x, double* rowpart,
                               float* colpart, const SymPlan& sp, const BatchMap& bm, int* status,
                               const int* gate, cudaStream_t s, int fmt) {
  return clamp ? launch_k1t_ut<true, true>(img, 0, x, rowpart, colpart, sp, bm, status, gate, s, fmt)
               : launch_k1t_ut<false, true>(img, 0, x, rowpart, colpart, sp, bm, status, gate, s, fmt);
}

cudaError_t set_wait_limit_symtc(unsigned long long ns) { return set_wait_limit_this_unit(ns); }

}  // namespace laker
