// Flash-style multi-RHS FP32 attention-kernel matvec on the tensor cores:
//   Y = [lam X +] exp(E_rows E_cols^T) X        (X: n x k, k <= 32 per chunk)
// for operators whose Gram entries need no clamp.
//
// The shape is FlashAttention's forward without the softmax normalisation
// (the exp arguments are bounded, so no running maximum is needed): per
// 128-row tile and 64-point column slab
//   S = E_r E_c^T      three kind::f16 MMAs of K = 16 from the split-FP16
//                      operand image of the symmetric kernel (k1t_pack: rows
//                      scaled by log2 e), two with its two-MMA format when
//                      d <= 10, M = 128, N = 64, into TMEM;
//   P = exp2(S)        CUDA cores: each thread loads 16 logits of its row from
//                      TMEM, one MUFU ex2 each, splits P into TF32 hi + lo and
//                      stores both back into TMEM (P never touches shared
//                      memory);
//   O += P X           kind::tf32 MMAs with A = P from TMEM (K = 8 columns per
//                      MMA), B = the slab's pre-split X tiles from shared
//                      memory: P_hi X_hi + P_hi X_lo + P_lo X_hi (~2^-21
//                      relative per product, as FP32 entries; plain TF32
//                      would perturb A by more than lambda), FP32 accumulation
//                      in TMEM.  The X tile stores X_hi's N rows right above
//                      X_lo's, so P_hi [X_hi | X_lo] is one MMA of width 2 N
//                      and P_lo X_hi a second one into the first N columns:
//                      two MMAs per K step; the output is the sum of the two
//                      column halves.
// Per kernel entry the CUDA cores do one ex2 and a few conversions: the kernel
// is bound by the MUFU ex2 rate, where the CUDA-core-logit multi-RHS kernel
// (k2_tc_matvec) spends d FMAs, embedding loads and a shared-memory write per
// entry.  Each entry is evaluated once per chunk of up to 32 right-hand sides.
//
// Work items: (row tile, RHS chunk, column segment), rows fastest, taken by a
// persistent grid; segments of the column range keep every SM busy and their
// partial outputs are added in a fixed order (launch_seg_reduce), so the
// result does not depend on scheduling.
//
// Roles in a CTA of 576 threads (one CTA per SM: all 512 TMEM columns taken,
// more than half of the SM's shared memory):
//   warps 0-15 epilogue, two groups of eight that take alternate slabs (two
//             slabs' exp2 in flight, so one group's TMEM and barrier latencies
//             hide behind the other's work): warp w owns TMEM lanes
//             32 (w & 3) .. + 31 and 32 of a slab's 64 columns ((w >> 2) & 1):
//             exp2 and the split into P; the four warps of group 0, column
//             half 0 also read the item's accumulators and write its rows;
//   warp 16   copies: the item's row operands (double-buffered), per slab the
//             column operands and the X tiles (S stages);
//   warp 17   MMA (lane 0): the slab's logits one slab ahead of its P X
//             products, three TMEM logit / P buffers.
// Every wait is bounded; a timeout raises a shared abort flag, the CTA drains
// its copies and MMAs, frees TMEM and returns (status LAKER_ERR_TIMEOUT).
#include <cstdlib>

#include "internal.cuh"
#include "sym.cuh"
#include "tc.cuh"

namespace laker {
namespace {

constexpr int kFRows = 128;                       // rows per item (MMA M)
constexpr int kFSlab = 64;                        // points per column slab
constexpr int kFEpiWarps = 16;
constexpr int kFThreads = kFEpiWarps * 32 + 64;   // + copy warp + MMA warp
constexpr int kFCopyWarp = kFEpiWarps, kFMmaWarp = kFEpiWarps + 1;
constexpr int kFBufs = 3;                         // TMEM logit / P buffers
constexpr int kFMaxN = 32;                        // right-hand sides per chunk
constexpr int kFGroupWarps = 8;                   // epilogue warps per slab group
constexpr int kFMaxStages = 8;
// TMEM columns: buffer b holds S, then P_hi, at [128 b, 128 b + 64) and P_lo
// at [128 b + 64, 128 b + 128); accumulator a at [384 + 64 a, + 2 N).
constexpr uint32_t kFAccCol = 128u * kFBufs;
// Split-FP16 operand image of k1t_pack: per 512-point block 128 KB, row side
// (H, L, Hs) then column side (H, L, Hs), 16 KB per variant, 32 bytes per
// point (32-byte swizzle, K-major).
constexpr uint32_t kFVar = 512u * 32u;
constexpr uint32_t kFImgBlock = 128u * 1024u;
constexpr uint32_t kFRowVar = kFRows * 32u;        // one variant of a row tile (4 KB)
constexpr uint32_t kFColVar = kFSlab * 32u;        // one variant of a slab (2 KB)
constexpr uint32_t kFRowOps = 3u * kFRowVar;       // 12 KB
constexpr uint32_t kFColOps = 3u * kFColVar;       // 6 KB
constexpr uint32_t kFSBO16 = 8u * 32u;             // 8-row core group, FP16 operands
constexpr uint32_t kFLayout16 = 6u;                // SWIZZLE_32B
constexpr uint32_t kFSBO32 = 8u * 128u;            // 8-row core group, X tiles
constexpr uint32_t kFLayout128 = 2u;               // SWIZZLE_128B
static_assert(kFAccCol + 2 * (2 * kFMaxN) <= 512, "TMEM budget");

struct K2fWork {
  int64_t rtiles;  // row tiles of 128
  int chunks;      // RHS chunks of N
  int segs;        // column segments
  int64_t nslabs;  // column slabs of 64 points
  int64_t sps;     // slabs per segment
  int64_t items;   // rtiles * chunks * segs
};

// Bytes of one stage: X tiles (2 tiles x [hi, lo] x N rows x 128 B) then the
// slab's three FP16 column operands, rounded to the 1024-byte swizzle atom.
__host__ __device__ inline uint32_t k2f_stage_bytes(int N) {
  return (uint32_t)round_up(512 * N + (int64_t)kFColOps, 1024);
}

__global__ void __launch_bounds__(kFThreads, 1)
    k2f_matvec(const uint8_t* __restrict__ rimg, int64_t m, const uint8_t* __restrict__ cimg,
               const uint8_t* __restrict__ ximg, int N, int S, K2fWork wk, float lam,
               const float* __restrict__ X, int64_t ldx, int k, float* __restrict__ Y,
               int64_t ldy, float* __restrict__ part, int nv, int* status, const int* gate) {
  // nv: operand variants per side of the image, 3 (split FP16) or 2 (the
  // same products in two MMAs, d <= 10); the shared-memory slots hold three
  if (gate && *gate == 0) return;
  extern __shared__ __align__(1024) uint8_t smem_raw[];
  uint8_t* base =
      reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
  const uint32_t sbytes = k2f_stage_bytes(N);
  uint8_t* sRow = base;                                 // 2 x row operands (12 KB)
  uint8_t* sStage = base + 2 * kFRowOps;                // S stages
  uint64_t* bars = reinterpret_cast<uint64_t*>(sStage + (size_t)S * sbytes);
  uint64_t* a_full = bars;                              // [2]
  uint64_t* a_empty = a_full + 2;                       // [2]
  uint64_t* b_full = a_empty + 2;                       // [S]
  uint64_t* b_empty = b_full + S;                       // [S]
  uint64_t* s_full = b_empty + S;                       // [kFBufs]
  uint64_t* s_empty = s_full + kFBufs;                  // [kFBufs]
  uint64_t* p_full = s_empty + kFBufs;                  // [kFBufs]
  uint64_t* acc_full = p_full + kFBufs;                 // [2]
  uint64_t* acc_empty = acc_full + 2;                   // [2]
  uint64_t* drain = acc_empty + 2;
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
    for (int i = 0; i < 2; ++i) {
      mbar_init(&a_full[i], 1);
      mbar_init(&a_empty[i], 1);
      mbar_init(&acc_full[i], 1);
      mbar_init(&acc_empty[i], 4);  // the four warps of column group 0
    }
    for (int i = 0; i < S; ++i) {
      mbar_init(&b_full[i], 1);
      mbar_init(&b_empty[i], 1);
    }
    for (int i = 0; i < kFBufs; ++i) {
      mbar_init(&s_full[i], 1);
      mbar_init(&s_empty[i], 1);
      mbar_init(&p_full[i], kFGroupWarps);  // one arrival per warp of the slab's group
    }
    mbar_init(drain, 1);
    *abort = 0;
    mbar_fence_init();
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem_base = *tmem_slot;

  // item -> (row tile, chunk, segment) and its slab range [s0, s1)
  auto item_of = [&](int64_t it, int64_t* rt, int* ch, int* sg, int64_t* s0, int64_t* s1) {
    *rt = it % wk.rtiles;
    const int64_t rest = it / wk.rtiles;
    *ch = (int)(rest % wk.chunks);
    *sg = (int)(rest / wk.chunks);
    *s0 = (int64_t)*sg * wk.sps;
    *s1 = *s0 + wk.sps < wk.nslabs ? *s0 + wk.sps : wk.nslabs;
  };

  int64_t a_issued = 0, b_issued = 0;  // copy role
  bool mma_any = false;                // MMA role
  if (warp == kFCopyWarp) {
    // ---- copies -------------------------------------------------------------
    if (lane == 0) {
      int64_t g = 0, ni = 0;
      for (int64_t it = blockIdx.x; it < wk.items && !*abort; it += gridDim.x, ++ni) {
        int64_t rt, s0, s1;
        int ch, sg;
        item_of(it, &rt, &ch, &sg, &s0, &s1);
        const int ab = (int)(ni & 1);
        if (!wait_or_abort(&a_empty[ab], (uint32_t)(((ni >> 1) & 1) ^ 1), status, abort)) break;
        mbar_arrive_expect_tx(&a_full[ab], (uint32_t)nv * kFRowVar);
        const uint8_t* rsrc = rimg + (rt >> 2) * (int64_t)kFImgBlock + (rt & 3) * (int64_t)kFRowVar;
        for (int v = 0; v < nv; ++v)
          bulk_g2s(sRow + ab * kFRowOps + v * kFRowVar, rsrc + v * kFVar, kFRowVar, &a_full[ab]);
        ++a_issued;
        bool ok = true;
        for (int64_t s = s0; s < s1; ++s, ++g) {
          const int st = (int)(g % S);
          if (!wait_or_abort(&b_empty[st], (uint32_t)(((g / S) & 1) ^ 1), status, abort)) {
            ok = false;
            break;
          }
          uint8_t* dst = sStage + (size_t)st * sbytes;
          mbar_arrive_expect_tx(&b_full[st], (uint32_t)(512 * N) + (uint32_t)nv * kFColVar);
          bulk_g2s(dst, ximg + ((int64_t)ch * 2 * wk.nslabs + 2 * s) * (int64_t)(256 * N),
                   (uint32_t)(512 * N), &b_full[st]);
          const uint8_t* csrc =
              cimg + (s >> 3) * (int64_t)kFImgBlock + (int64_t)nv * kFVar + (s & 7) * (int64_t)kFColVar;
          for (int v = 0; v < nv; ++v)
            bulk_g2s(dst + 512 * N + v * kFColVar, csrc + v * kFVar, kFColVar, &b_full[st]);
          ++b_issued;
        }
        if (!ok) break;
      }
    }
  } else if (warp == kFMmaWarp) {
    // ---- MMA issue ------------------------------------------------------------
    if (lane == 0) {
      const uint32_t idesc_s = f16_idesc_mn(kFRows, kFSlab);
      const uint32_t idesc_p = tf32_idesc_mn(kFRows, N);
      const uint32_t idesc_p2 = tf32_idesc_mn(kFRows, 2 * N);
      int64_t g = 0, ni = 0;
      // the logits of global slab gg (row operands of buffer ab), into its buffer
      auto logits = [&](int64_t gg, int ab) -> bool {
        const int st = (int)(gg % S), buf = (int)(gg % kFBufs);
        if (!wait_or_abort(&b_full[st], (uint32_t)((gg / S) & 1), status, abort)) return false;
        if (!wait_or_abort(&s_empty[buf], (uint32_t)(((gg / kFBufs) & 1) ^ 1), status, abort))
          return false;
        tc_fence_after();
        const uint32_t ra = smem_u32(sRow + ab * kFRowOps);
        const uint32_t cb = smem_u32(sStage + (size_t)st * sbytes + 512 * N);
        const uint32_t d = tmem_base + (uint32_t)(buf * 128);
        mma_f16(d, kmajor_desc_raw(ra, kFSBO16, kFLayout16), kmajor_desc_raw(cb, kFSBO16, kFLayout16),
                idesc_s, 0u);
        if (nv == 2) {
          // V0 W0 + V1 W1 = H H' + Hs L' + L Hs'
          mma_f16(d, kmajor_desc_raw(ra + kFRowVar, kFSBO16, kFLayout16),
                  kmajor_desc_raw(cb + kFColVar, kFSBO16, kFLayout16), idesc_s, 1u);
        } else {
          // H H' + Hs L' + L Hs' (variants 0 = H, 1 = L, 2 = Hs)
          mma_f16(d, kmajor_desc_raw(ra + 2 * kFRowVar, kFSBO16, kFLayout16),
                  kmajor_desc_raw(cb + kFColVar, kFSBO16, kFLayout16), idesc_s, 1u);
          mma_f16(d, kmajor_desc_raw(ra + kFRowVar, kFSBO16, kFLayout16),
                  kmajor_desc_raw(cb + 2 * kFColVar, kFSBO16, kFLayout16), idesc_s, 1u);
        }
        mma_any = true;
        mma_commit(&s_full[buf]);
        return true;
      };
      for (int64_t it = blockIdx.x; it < wk.items && !*abort; it += gridDim.x, ++ni) {
        int64_t rt, s0, s1;
        int ch, sg;
        item_of(it, &rt, &ch, &sg, &s0, &s1);
        const int ab = (int)(ni & 1);
        if (!wait_or_abort(&a_full[ab], (uint32_t)((ni >> 1) & 1), status, abort)) break;
        if (!wait_or_abort(&acc_empty[ab], (uint32_t)(((ni >> 1) & 1) ^ 1), status, abort)) break;
        tc_fence_after();
        const uint32_t dacc = tmem_base + kFAccCol + (uint32_t)(ab * 2 * kFMaxN);
        bool ok = logits(g, ab);
        for (int64_t s = s0; ok && s < s1; ++s, ++g) {
          if (s + 1 < s1 && !logits(g + 1, ab)) {
            ok = false;
            break;
          }
          const int st = (int)(g % S), buf = (int)(g % kFBufs);
          if (!wait_or_abort(&p_full[buf], (uint32_t)((g / kFBufs) & 1), status, abort)) {
            ok = false;
            break;
          }
          tc_fence_after();
          const uint32_t xs = smem_u32(sStage + (size_t)st * sbytes);
          const uint32_t phi = tmem_base + (uint32_t)(buf * 128), plo = phi + 64u;
#pragma unroll
          for (int kk = 0; kk < kFSlab / 8; ++kk) {
            // X tile kk / 4, K step kk % 4 (32 bytes inside the swizzled row)
            const uint32_t xhi = xs + (uint32_t)((kk >> 2) * 256 * N) + (uint32_t)((kk & 3) * 32);
            const uint64_t bhi = kmajor_desc_raw(xhi, kFSBO32, kFLayout128);
            const uint32_t acc = (s > s0 || kk > 0) ? 1u : 0u;
            // D[:, 0:2N] += P_hi [X_hi | X_lo];  D[:, 0:N] += P_lo X_hi
            mma_tf32_ts(dacc, phi + 8u * kk, bhi, idesc_p2, acc);
            mma_tf32_ts(dacc, plo + 8u * kk, bhi, idesc_p, 1u);
          }
          mma_commit(&s_empty[buf]);
          mma_commit(&b_empty[st]);
          if (s + 1 == s1) mma_commit(&a_empty[ab]);
        }
        if (!ok) break;
        mma_commit(&acc_full[ab]);
      }
    }
  } else {
    // ---- epilogue (warps 0-15) ----------------------------------------------------
    const int q = warp & 3, ch2 = (warp >> 2) & 1, grp = warp >> 3;
    const uint32_t lane_off = (uint32_t)(q * 32) << 16;
    int64_t g = 0, ni = 0;
    bool dead = false;
    for (int64_t it = blockIdx.x; it < wk.items && !dead; it += gridDim.x, ++ni) {
      int64_t rt, s0, s1;
      int ch, sg;
      item_of(it, &rt, &ch, &sg, &s0, &s1);
      for (int64_t s = s0; s < s1; ++s, ++g) {
        if ((int)(g & 1) != grp) continue;  // the other group's slab
        const int buf = (int)(g % kFBufs);
        if (!warp_wait_or_abort(&s_full[buf], (uint32_t)((g / kFBufs) & 1), status, abort, lane)) {
          dead = true;
          break;
        }
        tc_fence_after();
        const uint32_t ts = tmem_base + lane_off + (uint32_t)(buf * 128 + ch2 * 32);
        float v[32];
        tmem_ld32(ts, v);
#pragma unroll
        for (int h = 0; h < 2; ++h) {
          uint32_t hi[16], lo[16];
#pragma unroll
          for (int u = 0; u < 16; ++u) {
            const float p = ex2_approx(v[16 * h + u]);
            // P_hi by truncation (an AND instead of a conversion), P_lo the
            // exact remainder rounded to TF32: |error| <= 2^-22 |p|
            hi[u] = __float_as_uint(p) & 0xffffe000u;
            lo[u] = to_tf32(p - __uint_as_float(hi[u]));
          }
          tmem_st16(ts + (uint32_t)(16 * h), hi);
          tmem_st16(ts + 64u + (uint32_t)(16 * h), lo);
        }
        tmem_st_wait();
        tc_fence_before();
        __syncwarp();
        if (lane == 0) mbar_arrive(&p_full[buf]);
      }
      if (dead) break;
      if (grp == 0 && ch2 == 0) {
        // the item's accumulators: rows of lane quadrant q; the output is the
        // sum of the two column halves
        const int ab = (int)(ni & 1);
        if (!warp_wait_or_abort(&acc_full[ab], (uint32_t)((ni >> 1) & 1), status, abort, lane)) {
          dead = true;
          break;
        }
        tc_fence_after();
        const int64_t r = rt * kFRows + q * 32 + lane;
        const uint32_t da = tmem_base + lane_off + kFAccCol + (uint32_t)(ab * 2 * kFMaxN);
        for (int c0 = 0; c0 < N; c0 += 16) {
          float o[16], o2[16];
          tmem_ld16x2(da + (uint32_t)c0, da + (uint32_t)(N + c0), o, o2);
          if (r < m) {
#pragma unroll
            for (int u = 0; u < 16; ++u) {
              const int col = ch * N + c0 + u;
              if (col < k) {
                const float val = o[u] + o2[u];
                if (wk.segs == 1)
                  Y[r * ldy + col] = val + (lam != 0.0f ? lam * X[r * ldx + col] : 0.0f);
                else
                  part[((int64_t)sg * m + r) * k + col] = val;
              }
            }
          }
        }
        tc_fence_before();
        __syncwarp();
        if (lane == 0) mbar_arrive(&acc_empty[ab]);
      }
    }
  }

  // ---- teardown: every role has left its loop ---------------------------------
  __syncthreads();
  if (*abort) {
    // bounded drains of the copies in flight and of the MMAs issued
    if (warp == kFCopyWarp && lane == 0) {
      for (int64_t gg = a_issued > 2 ? a_issued - 2 : 0; gg < a_issued; ++gg)
        mbar_wait_drain(&a_full[gg & 1], (uint32_t)((gg >> 1) & 1), status);
      for (int64_t gg = b_issued > S ? b_issued - S : 0; gg < b_issued; ++gg)
        mbar_wait_drain(&b_full[gg % S], (uint32_t)((gg / S) & 1), status);
    }
    if (warp == kFMmaWarp && lane == 0 && mma_any) {
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

// Right-hand sides per chunk: up to 32, a multiple of 16 (the MMA's N; the
// stacked P_hi [X_hi | X_lo] product is 2 N wide).
int k2f_chunk_cols(int k) { return (int)round_up(k < kFMaxN ? k : kFMaxN, 16); }

int k2f_stages(int N) {
  const int avail = 227 * 1024 - 1024 - 2 * (int)kFRowOps - 512;
  int S = avail / (int)k2f_stage_bytes(N);
  return S > kFMaxStages ? kFMaxStages : S;
}

size_t k2f_smem_bytes(int N, int S) {
  size_t b = 1024 + 2 * (size_t)kFRowOps + (size_t)S * k2f_stage_bytes(N) +
             (size_t)(4 + 2 * S + 3 * kFBufs + 4 + 1) * 8 + 16;
  if (b <= kTmemExclusiveSmem) b = kTmemExclusiveSmem + 1024;  // one TMEM owner per SM
  return b;
}

// Segments so that the items fill the SMs several times over (at least 8
// slabs each).
K2fWork k2f_work(int64_t m, int64_t n, int k, int N) {
  K2fWork w{};
  w.rtiles = ceil_div(m, kFRows);
  w.chunks = (int)ceil_div(k, N);
  w.nslabs = ceil_div(n, kFSlab);
  const int64_t base = w.rtiles * w.chunks;
  const int64_t want = 8 * (int64_t)sm_count();
  int64_t segs = base >= want ? 1 : ceil_div(want, base);
  const int64_t max_segs = w.nslabs / 8 > 1 ? w.nslabs / 8 : 1;
  if (segs > max_segs) segs = max_segs;
  if (segs > 64) segs = 64;
  w.sps = ceil_div(w.nslabs, segs);
  w.segs = (int)ceil_div(w.nslabs, w.sps);
  w.items = base * w.segs;
  return w;
}

struct K2fLayout {
  size_t x_off, x_bytes, part_off, part_bytes, rimg_off, cimg_off, total;
};

K2fLayout k2f_layout(int64_t m, int64_t n, int k, bool same_points) {
  const int N = k2f_chunk_cols(k);
  const K2fWork w = k2f_work(m, n, k, N);
  K2fLayout L{};
  L.x_off = 0;
  L.x_bytes = (size_t)round_up((int64_t)((size_t)w.chunks * (size_t)(2 * w.nslabs) * 256 * N), 1024);
  L.part_off = L.x_off + L.x_bytes;
  L.part_bytes = w.segs > 1 ? (size_t)round_up((int64_t)((size_t)w.segs * m * k * 4), 1024) : 0;
  L.rimg_off = L.part_off + L.part_bytes;
  L.cimg_off = same_points ? L.rimg_off : L.rimg_off + k1t_image_bytes(m);
  L.total = L.cimg_off + k1t_image_bytes(n);
  return L;
}

// Largest k that takes the flash kernel (LAKER_VARIANT_MULTI_FLASH_K; 0 off).
int k2f_max_k() { return variant_get(LAKER_VARIANT_MULTI_FLASH_K); }

}  // namespace

bool k2f_enabled(int k, int clamp) { return !clamp && k > 1 && k <= k2f_max_k(); }

size_t k2f_workspace_bytes(int64_t m, int64_t n, int k, bool same_points) {
  return k2f_layout(m, n, k, same_points).total;
}

cudaError_t launch_k2f(const float* rows32, int64_t m, const float* cols32, int64_t n, int d,
                       float lam, const float* X, int64_t ldx, int k, float* Y, int64_t ldy,
                       uint8_t* ws, int* status, cudaStream_t s, const int* gate) {
  if (m <= 0 || n <= 0 || k < 1) return cudaSuccess;
  const bool same = rows32 == cols32 && m == n;
  const int N = k2f_chunk_cols(k);
  const K2fWork wk = k2f_work(m, n, k, N);
  const K2fLayout L = k2f_layout(m, n, k, same);
  uint8_t* ximg = ws + L.x_off;
  float* part = wk.segs > 1 ? reinterpret_cast<float*>(ws + L.part_off) : nullptr;
  uint8_t* rimg = ws + L.rimg_off;
  uint8_t* cimg = ws + L.cimg_off;
  cudaError_t e = launch_pack_x32(X, n, ldx, k, N, 2 * wk.nslabs, ximg, gate, s);
  const int fmt = padded_dim(d) <= 10 ? kK1tF16x2 : kK1tF16;
  const int nv = fmt == kK1tF16x2 ? 2 : 3;
  if (e == cudaSuccess) e = launch_k1t_pack(rows32, m, d, rimg, round_up(m, 512), s, fmt);
  if (e == cudaSuccess && !same) e = launch_k1t_pack(cols32, n, d, cimg, round_up(n, 512), s, fmt);
  if (e != cudaSuccess) return e;
  const int S = k2f_stages(N);
  const size_t smem = k2f_smem_bytes(N, S);
  if (S < 2 || smem > 227 * 1024) return cudaErrorInvalidConfiguration;
  e = cudaFuncSetAttribute(k2f_matvec, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
  const int64_t grid = wk.items < (int64_t)sm_count() ? wk.items : (int64_t)sm_count();
  k2f_matvec<<<(unsigned)grid, kFThreads, smem, s>>>(rimg, m, cimg, ximg, N, S, wk, lam, X, ldx, k,
                                                     Y, ldy, part, nv, status, gate);
  e = cudaGetLastError();
  if (e != cudaSuccess || wk.segs == 1) return e;
  return launch_seg_reduce(part, wk.segs, m, k, lam, X, ldx, Y, ldy, gate, s);
}

cudaError_t set_wait_limit_flash(unsigned long long ns) { return set_wait_limit_this_unit(ns); }

}  // namespace laker
