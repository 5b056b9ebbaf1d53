// Symmetric FP32 fused matvec: y = lam x + exp(E E^T) x evaluating each
// off-diagonal kernel entry once.
//
// The points are cut into blocks of B = T*R.  Work items are the block pairs
// (a, b) with a <= b, enumerated row-major over the upper triangle; a
// persistent grid gives every CTA a contiguous, equal share of them.  For a
// pair, the CTA holds the R rows per thread of block a in registers (scaled by
// log2 e, duplicated per float2 half, plus their x values) and walks the
// columns of block b, staged by double-buffered TMA bulk copies: per column
// pair the logits are DP packed FMAs, the entries come from MUFU ex2, the row
// sums take one packed FMA (as in the plain kernel) and -- for a < b -- the
// column sums another one.  Column sums are reduced over the warp with
// shuffles and over the CTA in shared memory, then stored per pair; row sums
// are accumulated over the pair's column tiles and also stored per pair.  A
// fixed-order finish adds both partial sets, so the result is deterministic
// and does not depend on the grid, on the CTA that processed a pair or on the
// other instances of a batch.  Work per computed entry: d FMA + 2 FMA + 1 exp2,
// i.e. (d + 2) / 2 FMA and 1/2 exp2 per logical entry.
//
// The BATCHED instantiation runs many independent problems in one launch
// (BatchMap): the pair list is the concatenation of the running instances'
// pair lists (a block-diagonal operator), split evenly over the grid at run
// time, so the whole grid works on whatever is still running.
#include <cstdlib>

#include "sym.cuh"

namespace laker {
namespace {

// Position in a CTA's flat sequence of column tiles (pair p, tile t of block
// b).  p counts the pairs of the launch; the pair's partial sums live at slot
// gp0 + (p - pstart).
struct SymCursor {
  int64_t p, p_end;
  int j;  // index into the running-instance list (batched)
  int64_t a, b;
  int t;
  // metadata of the current instance
  int64_t nb, npts, seg, blk0, pstart, pend, gp0;
};

template <bool BATCHED>
__device__ __forceinline__ void cursor_load_inst(SymCursor& cu, const SymPlan& sp,
                                                 const BatchMap& bm, int64_t n) {
  if (BATCHED) {
    const SlotInfo& si = bm.slots[bm.act_inst[cu.j]];
    cu.nb = si.nblk;
    cu.npts = si.npts;
    cu.seg = si.seg;
    cu.blk0 = si.blk_start;
    cu.pstart = bm.act_ps[cu.j];
    cu.pend = bm.act_ps[cu.j + 1];
    cu.gp0 = si.pair_start;
  } else {
    cu.nb = sp.nb;
    cu.npts = n;
    cu.seg = 0;
    cu.blk0 = 0;
    cu.pstart = 0;
    cu.pend = sp.npairs;
    cu.gp0 = 0;
  }
}

// Place the cursor on tile 0 of pair p, moving to the instance that holds it.
// Returns false when the CTA's range is exhausted.
template <bool BATCHED>
__device__ __forceinline__ bool cursor_settle(SymCursor& cu, const SymPlan& sp, const BatchMap& bm,
                                              int64_t n) {
  if (cu.p >= cu.p_end) return false;
  if (BATCHED) {
    while (cu.p >= cu.pend) {  // ends: p < p_end <= act_ps[*act_count]
      ++cu.j;
      cursor_load_inst<BATCHED>(cu, sp, bm, n);
    }
  }
  sym_pair_coords(cu.p - cu.pstart, cu.nb, &cu.a, &cu.b);
  cu.t = 0;
  return true;
}

// Next tile that holds points (tiles starting at or past the instance's n are
// empty and skipped).
template <bool BATCHED, int B, int TC, int TPB>
__device__ __forceinline__ bool cursor_next(SymCursor& cu, const SymPlan& sp, const BatchMap& bm,
                                            int64_t n) {
  ++cu.t;
  if (cu.t < TPB && cu.b * B + (int64_t)cu.t * TC < cu.npts) return true;
  ++cu.p;
  if (cu.p >= cu.p_end) return false;
  if (cu.p < cu.pend) {
    if (++cu.b >= cu.nb) {
      ++cu.a;
      cu.b = cu.a;
    }
    cu.t = 0;
    return true;
  }
  return cursor_settle<BATCHED>(cu, sp, bm, n);
}

template <int DP, int R, int T, bool CLAMP, bool BATCHED>
__global__ void __launch_bounds__(T, 3)
    k1s_matvec_f32(const float* __restrict__ E, int64_t n, const float* __restrict__ x,
                   float* __restrict__ colpart, double* __restrict__ rowpart, SymPlan sp,
                   BatchMap bm, int* status, const int* gate) {
  if (gate && *gate == 0) return;
  constexpr int TC = kTileCols32;
  constexpr int TP = TC / 2;
  constexpr int TILE_FLOATS = TC * DP;
  constexpr int B = T * R;
  constexpr int TPB = B / TC;  // column tiles per block
  constexpr int NW = T / 32;
  static_assert(B % TC == 0, "block must be a whole number of column tiles");
  __shared__ __align__(128) float sE[2][TILE_FLOATS];
  __shared__ __align__(16) float sX[2][TC];
  __shared__ __align__(16) float sCol[NW][TC];
  __shared__ __align__(8) uint64_t bar[2];

  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int64_t c = blockIdx.x;
  int64_t p_begin, p_end;
  SymCursor cu;
  cu.j = 0;
  if (BATCHED) {
    // split the running instances' pairs evenly over the grid
    const int nact = *bm.act_count;
    if (nact <= 0) return;
    const int64_t total = bm.act_ps[nact];
    const int64_t q = total / gridDim.x, rem = total % gridDim.x;
    p_begin = c * q + (c < rem ? c : rem);
    p_end = p_begin + q + (c < rem ? 1 : 0);
    if (p_begin >= p_end) return;
    // running instance of the first pair: binary search of act_ps
    int lo = 0, hi = nact - 1;
    while (lo < hi) {
      const int mid = (lo + hi + 1) >> 1;
      if (bm.act_ps[mid] <= p_begin) lo = mid; else hi = mid - 1;
    }
    cu.j = lo;
  } else {
    p_begin = c * sp.q + (c < sp.rem ? c : sp.rem);
    p_end = p_begin + sp.q + (c < sp.rem ? 1 : 0);
    if (p_begin >= p_end) return;
  }
  cu.p = p_begin;
  cu.p_end = p_end;
  cursor_load_inst<BATCHED>(cu, sp, bm, n);
  if (!cursor_settle<BATCHED>(cu, sp, bm, n)) return;  // uniform: every thread sees the same

  if (tid == 0) {
    mbar_init(&bar[0], 1);
    mbar_init(&bar[1], 1);
    mbar_fence_init();
  }
  __syncthreads();

  auto col0_of = [&](const SymCursor& s) -> int64_t { return s.seg + s.b * B + (int64_t)s.t * TC; };
  auto issue = [&](int64_t col0, int buf) {
    mbar_arrive_expect_tx(&bar[buf], TILE_FLOATS * 4);
    bulk_g2s(sE[buf], E + (col0 >> 1) * (DP * 2), TILE_FLOATS * 4, &bar[buf]);
  };
  auto load_x = [&](const SymCursor& s, int buf) {
    const int64_t local0 = s.b * B + (int64_t)s.t * TC;
    for (int j = tid; j < TC; j += T) sX[buf][j] = (local0 + j < s.npts) ? x[s.seg + local0 + j] : 0.0f;
  };

  // rows of block a of the current instance in registers; row sums of the current pair
  float2 ev[R][DP];
  float2 xr[R];
  double acc[R];
#pragma unroll
  for (int r = 0; r < R; ++r) acc[r] = 0.0;
  auto load_rows = [&](const SymCursor& s) {
#pragma unroll
    for (int r = 0; r < R; ++r) {
      const int64_t li = s.a * B + r * T + tid;
      const bool ok = li < s.npts;
      const int64_t i = s.seg + li;
      const float* blk = E + (i >> 1) * (DP * 2) + (i & 1);
#pragma unroll
      for (int k = 0; k < DP; ++k) {
        const float v = ok ? blk[2 * k] * kLog2e : 0.0f;
        ev[r][k] = make_float2(v, v);
      }
      const float xi = ok ? x[i] : 0.0f;
      xr[r] = make_float2(xi, xi);
    }
  };
  // Row sums are stored per pair: the finish then adds an instance's pairs in
  // a fixed order that does not depend on which CTA processed them (the
  // result is the same alone or inside any batch).
  auto flush_rows = [&](int64_t pair) {
    double* dst = rowpart + pair * (int64_t)B;
#pragma unroll
    for (int r = 0; r < R; ++r) {
      dst[r * T + tid] = acc[r];
      acc[r] = 0.0;
    }
  };

  load_rows(cu);
  SymCursor nx = cu;
  if (tid == 0) issue(col0_of(nx), 0);
  load_x(nx, 0);
  bool have_nx = cursor_next<BATCHED, B, TC, TPB>(nx, sp, bm, n);
  __syncthreads();

  int k_tile = 0, issued = 1, consumed = 0;
  bool failed = false;
  for (;;) {
    const int buf = k_tile & 1;
    if (have_nx) {
      if (tid == 0) issue(col0_of(nx), buf ^ 1);
      load_x(nx, buf ^ 1);
      ++issued;
    }
    const int ok = __syncthreads_and(mbar_wait_bounded(&bar[buf], (k_tile >> 1) & 1, status) ? 1 : 0);
    if (!ok) {
      failed = true;
      break;
    }
    ++consumed;
    const bool offdiag = cu.a != cu.b;
    const float* Et = sE[buf];
    const float2* X2 = reinterpret_cast<const float2*>(sX[buf]);
    float2 tacc[R];
#pragma unroll
    for (int r = 0; r < R; ++r) tacc[r] = make_float2(0.0f, 0.0f);

    if (offdiag) {
      // 8 column pairs at a time: their column partials are reduced together
      // so the shuffle latency overlaps.
#pragma unroll 1
      for (int q0 = 0; q0 < TP; q0 += 8) {
        float2 cs[8];
#pragma unroll
        for (int u = 0; u < 8; ++u) {
          const int q = q0 + u;
          const float4* cp = reinterpret_cast<const float4*>(Et + q * (DP * 2));
          float2 cv[DP];
#pragma unroll
          for (int h = 0; h < DP / 2; ++h) {
            const float4 v = cp[h];
            cv[2 * h] = make_float2(v.x, v.y);
            cv[2 * h + 1] = make_float2(v.z, v.w);
          }
          const float2 xv = X2[q];
          float2 ca = make_float2(0.0f, 0.0f);
#pragma unroll
          for (int r = 0; r < R; ++r) {
            float2 s = __fmul2_rn(ev[r][0], cv[0]);
#pragma unroll
            for (int k = 1; k < DP; ++k) s = __ffma2_rn(ev[r][k], cv[k], s);
            if (CLAMP) {
              s.x = fminf(s.x, kClampLog2);
              s.y = fminf(s.y, kClampLog2);
            }
            float2 e;
            e.x = ex2_approx(s.x);
            e.y = ex2_approx(s.y);
            tacc[r] = __ffma2_rn(e, xv, tacc[r]);
            ca = __ffma2_rn(e, xr[r], ca);
          }
          cs[u] = ca;
        }
        // warp sums of the 16 column partials (columns 2 q0 .. 2 q0 + 15):
        // reduce-scatter, lane l ends with column 2 q0 + (l >> 1)
        float cv16[16];
#pragma unroll
        for (int u = 0; u < 8; ++u) {
          cv16[2 * u] = cs[u].x;
          cv16[2 * u + 1] = cs[u].y;
        }
        const float colsum = warp_reduce_scatter<16>(cv16, lane);
        if ((lane & 1) == 0) sCol[warp][2 * q0 + (lane >> 1)] = colsum;
      }
    } else {
#pragma unroll 2
      for (int q = 0; q < TP; ++q) {
        const float4* cp = reinterpret_cast<const float4*>(Et + q * (DP * 2));
        float2 cv[DP];
#pragma unroll
        for (int h = 0; h < DP / 2; ++h) {
          const float4 v = cp[h];
          cv[2 * h] = make_float2(v.x, v.y);
          cv[2 * h + 1] = make_float2(v.z, v.w);
        }
        const float2 xv = X2[q];
#pragma unroll
        for (int r = 0; r < R; ++r) {
          float2 s = __fmul2_rn(ev[r][0], cv[0]);
#pragma unroll
          for (int k = 1; k < DP; ++k) s = __ffma2_rn(ev[r][k], cv[k], s);
          if (CLAMP) {
            s.x = fminf(s.x, kClampLog2);
            s.y = fminf(s.y, kClampLog2);
          }
          float2 e;
          e.x = ex2_approx(s.x);
          e.y = ex2_approx(s.y);
          tacc[r] = __ffma2_rn(e, xv, tacc[r]);
        }
      }
    }
#pragma unroll
    for (int r = 0; r < R; ++r) acc[r] += (double)tacc[r].x + (double)tacc[r].y;
    __syncthreads();  // sE/sX[buf] are refilled next; sCol is complete
    if (offdiag) {
      // this tile's column sums (columns t*TC .. t*TC+TC-1 of block b)
      for (int j = tid; j < TC; j += T) {
        float s = 0.0f;
#pragma unroll
        for (int w = 0; w < NW; ++w) s += sCol[w][j];
        colpart[(cu.gp0 + cu.p - cu.pstart) * B + cu.t * TC + j] = s;
      }
    }
    __syncthreads();  // sCol is reused by the next tile

    // advance the consumer; store the row sums when the pair changes and
    // reload the rows when the row block changes
    const int64_t prev_p = cu.p, prev_slot = cu.gp0 + cu.p - cu.pstart;
    const int64_t prev_block = cu.blk0 + cu.a;
    const bool more = cursor_next<BATCHED, B, TC, TPB>(cu, sp, bm, n);
    ++k_tile;
    if (!more || cu.p != prev_p) flush_rows(prev_slot);
    if (more && cu.blk0 + cu.a != prev_block) load_rows(cu);
    if (!more) break;
    if (have_nx) have_nx = cursor_next<BATCHED, B, TC, TPB>(nx, sp, bm, n);
  }
  if (failed) {
    for (int k = consumed; k < issued; ++k) mbar_wait_drain(&bar[k & 1], (k >> 1) & 1, status);
  }
}

// FP64 twin of k1s_matvec_f32 (the accurate operator of the residual
// recomputation): the same blocks, pairs, cursors and per-pair partial sums,
// with FP64 logits, exp and accumulation.  Column tiles are packed64 rows
// (TC points of DP doubles, one TMA bulk copy each); R rows per thread.
// Two CTAs per SM (at most 128 registers a thread): twice the warps to hide
// the dependent FP64 chains (9.3 against 9.7 ms at n = 100k with one CTA).
template <int DP, int R, int T, bool CLAMP, bool BATCHED>
__global__ void __launch_bounds__(T, 2)
    k4s_matvec_f64(const double* __restrict__ E, int64_t n, const double* __restrict__ x,
                   double* __restrict__ colpart, double* __restrict__ rowpart, SymPlan sp,
                   BatchMap bm, int* status, const int* gate) {
  if (gate && *gate == 0) return;
  constexpr int TC = kTileCols64;
  constexpr int TILE = TC * DP;
  constexpr int B = T * R;
  constexpr int TPB = B / TC;
  constexpr int NW = T / 32;
  constexpr int CB = 8;  // columns whose partials are reduced together
  static_assert(B % TC == 0, "block must be a whole number of column tiles");
  __shared__ __align__(128) double sE[2][TILE];
  __shared__ __align__(16) double sX[2][TC];
  __shared__ double sCol[NW][TC];
  __shared__ double sExp[64];
  __shared__ __align__(8) uint64_t bar[2];

  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int64_t c = blockIdx.x;
  int64_t p_begin, p_end;
  SymCursor cu;
  cu.j = 0;
  if (BATCHED) {
    const int nact = *bm.act_count;
    if (nact <= 0) return;
    const int64_t total = bm.act_ps[nact];
    const int64_t q = total / gridDim.x, rem = total % gridDim.x;
    p_begin = c * q + (c < rem ? c : rem);
    p_end = p_begin + q + (c < rem ? 1 : 0);
    if (p_begin >= p_end) return;
    int lo = 0, hi = nact - 1;
    while (lo < hi) {
      const int mid = (lo + hi + 1) >> 1;
      if (bm.act_ps[mid] <= p_begin) lo = mid; else hi = mid - 1;
    }
    cu.j = lo;
  } else {
    p_begin = c * sp.q + (c < sp.rem ? c : sp.rem);
    p_end = p_begin + sp.q + (c < sp.rem ? 1 : 0);
    if (p_begin >= p_end) return;
  }
  cu.p = p_begin;
  cu.p_end = p_end;
  cursor_load_inst<BATCHED>(cu, sp, bm, n);
  if (!cursor_settle<BATCHED>(cu, sp, bm, n)) return;

  if (tid == 0) {
    mbar_init(&bar[0], 1);
    mbar_init(&bar[1], 1);
    mbar_fence_init();
  }
  exp_table_to_shared(sExp, tid, T);
  __syncthreads();

  auto col0_of = [&](const SymCursor& s) -> int64_t { return s.seg + s.b * B + (int64_t)s.t * TC; };
  auto issue = [&](int64_t col0, int buf) {
    mbar_arrive_expect_tx(&bar[buf], TILE * 8);
    bulk_g2s(sE[buf], E + col0 * DP, TILE * 8, &bar[buf]);
  };
  auto load_x = [&](const SymCursor& s, int buf) {
    const int64_t local0 = s.b * B + (int64_t)s.t * TC;
    for (int j = tid; j < TC; j += T) sX[buf][j] = (local0 + j < s.npts) ? x[s.seg + local0 + j] : 0.0;
  };

  double ev[R][DP], xr[R], acc[R];
#pragma unroll
  for (int r = 0; r < R; ++r) acc[r] = 0.0;
  auto load_rows = [&](const SymCursor& s) {
#pragma unroll
    for (int r = 0; r < R; ++r) {
      const int64_t li = s.a * B + r * T + tid;
      const bool ok = li < s.npts;
      const int64_t i = s.seg + li;
#pragma unroll
      for (int k = 0; k < DP; ++k) ev[r][k] = ok ? E[i * DP + k] : 0.0;
      xr[r] = ok ? x[i] : 0.0;
    }
  };
  auto flush_rows = [&](int64_t slot) {
    double* dst = rowpart + slot * (int64_t)B;
#pragma unroll
    for (int r = 0; r < R; ++r) {
      dst[r * T + tid] = acc[r];
      acc[r] = 0.0;
    }
  };
  auto entry = [&](const double* cp, int r) -> double {
    double s = ev[r][0] * cp[0];
#pragma unroll
    for (int k = 1; k < DP; ++k) s = fma(ev[r][k], cp[k], s);
    if (CLAMP) s = fmin(s, kClamp64);
    return exp_tab(s, sExp);
  };

  load_rows(cu);
  SymCursor nx = cu;
  if (tid == 0) issue(col0_of(nx), 0);
  load_x(nx, 0);
  bool have_nx = cursor_next<BATCHED, B, TC, TPB>(nx, sp, bm, n);
  __syncthreads();

  int k_tile = 0, issued = 1, consumed = 0;
  bool failed = false;
  for (;;) {
    const int buf = k_tile & 1;
    if (have_nx) {
      if (tid == 0) issue(col0_of(nx), buf ^ 1);
      load_x(nx, buf ^ 1);
      ++issued;
    }
    const int ok = __syncthreads_and(mbar_wait_bounded(&bar[buf], (k_tile >> 1) & 1, status) ? 1 : 0);
    if (!ok) {
      failed = true;
      break;
    }
    ++consumed;
    const bool offdiag = cu.a != cu.b;
    const double* Et = sE[buf];
    const double* Xt = sX[buf];
    if (offdiag) {
#pragma unroll 1
      for (int j0 = 0; j0 < TC; j0 += CB) {
        double cs[CB];
#pragma unroll
        for (int u = 0; u < CB; ++u) {
          const double* cp = Et + (j0 + u) * DP;
          const double xj = Xt[j0 + u];
          double ca = 0.0;
#pragma unroll
          for (int r = 0; r < R; ++r) {
            const double e = entry(cp, r);
            acc[r] = fma(e, xj, acc[r]);
            ca = fma(e, xr[r], ca);
          }
          cs[u] = ca;
        }
        // reduce-scatter: lane l ends with column j0 + l / (32 / CB)
        const double colsum = warp_reduce_scatter<CB>(cs, lane);
        if ((lane & (32 / CB - 1)) == 0) sCol[warp][j0 + lane / (32 / CB)] = colsum;
      }
    } else {
#pragma unroll 2
      for (int j = 0; j < TC; ++j) {
        const double* cp = Et + j * DP;
        const double xj = Xt[j];
#pragma unroll
        for (int r = 0; r < R; ++r) acc[r] = fma(entry(cp, r), xj, acc[r]);
      }
    }
    __syncthreads();  // sE/sX[buf] are refilled next; sCol is complete
    if (offdiag) {
      for (int j = tid; j < TC; j += T) {
        double s = 0.0;
#pragma unroll
        for (int w = 0; w < NW; ++w) s += sCol[w][j];
        colpart[(cu.gp0 + cu.p - cu.pstart) * B + cu.t * TC + j] = s;
      }
    }
    __syncthreads();

    const int64_t prev_p = cu.p, prev_slot = cu.gp0 + cu.p - cu.pstart;
    const int64_t prev_block = cu.blk0 + cu.a;
    const bool more = cursor_next<BATCHED, B, TC, TPB>(cu, sp, bm, n);
    ++k_tile;
    if (!more || cu.p != prev_p) flush_rows(prev_slot);
    if (more && cu.blk0 + cu.a != prev_block) load_rows(cu);
    if (!more) break;
    if (have_nx) have_nx = cursor_next<BATCHED, B, TC, TPB>(nx, sp, bm, n);
  }
  if (failed) {
    for (int k = consumed; k < issued; ++k) mbar_wait_drain(&bar[k & 1], (k >> 1) & 1, status);
  }
}

}  // namespace
}  // namespace laker

namespace laker {
namespace {

constexpr int kSymRows = 4;      // rows per thread
constexpr int kSymThreads = 128;  // threads per CTA -> B = 512 points per block

template <int DP, bool CLAMP, bool BATCHED>
cudaError_t launch_k1s_t(const float* E, int64_t n, const float* x, double* rowpart,
                         float* colpart, const SymPlan& sp, const BatchMap& bm, int* status,
                         const int* gate, cudaStream_t s) {
  k1s_matvec_f32<DP, kSymRows, kSymThreads, CLAMP, BATCHED>
      <<<sp.grid, kSymThreads, 0, s>>>(E, n, x, colpart, rowpart, sp, bm, status, gate);
  return cudaGetLastError();
}

int k1s_occupancy(int dp) {
  static int cache[9] = {};
  if (dp < 2 || dp > 16) return 2;
  int& c = cache[dp / 2];
  if (c > 0) return c;
  const void* fn = nullptr;
#define LAKER_K1S_FN(DPv)                                                                 \
  if (dp == DPv)                                                                          \
    fn = reinterpret_cast<const void*>(&k1s_matvec_f32<DPv, kSymRows, kSymThreads, false, false>);
  LAKER_K1S_FN(2) LAKER_K1S_FN(4) LAKER_K1S_FN(6) LAKER_K1S_FN(8) LAKER_K1S_FN(10) LAKER_K1S_FN(12)
  LAKER_K1S_FN(14) LAKER_K1S_FN(16)
#undef LAKER_K1S_FN
  int nb = 0;
  if (!fn || cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, fn, kSymThreads, 0) != cudaSuccess ||
      nb < 1) {
    cudaGetLastError();
    nb = 2;
  }
  c = nb;
  return c;
}

#define LAKER_DISPATCH_DPS(dp, CALL)                    \
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

constexpr int kSym64Rows = 2;      // rows per thread of the FP64 kernel
constexpr int kSym64Threads = 256;  // -> the same 512-point blocks
static_assert(kSym64Rows * kSym64Threads == kSymRows * kSymThreads,
              "FP32 and FP64 symmetric kernels share their blocks and pair slots");

template <int DP, bool CLAMP, bool BATCHED>
cudaError_t launch_k4s_t(const double* E, int64_t n, const double* x, double* rowpart,
                         double* colpart, const SymPlan& sp, const BatchMap& bm, int* status,
                         const int* gate, cudaStream_t s) {
  k4s_matvec_f64<DP, kSym64Rows, kSym64Threads, CLAMP, BATCHED>
      <<<sp.grid, kSym64Threads, 0, s>>>(E, n, x, colpart, rowpart, sp, bm, status, gate);
  return cudaGetLastError();
}

int k4s_occupancy(int dp) {
  static int cache[9] = {};
  if (dp < 2 || dp > 16) return 1;
  int& c = cache[dp / 2];
  if (c > 0) return c;
  const void* fn = nullptr;
#define LAKER_K4S_FN(DPv)                                                                 \
  if (dp == DPv)                                                                          \
    fn = reinterpret_cast<const void*>(&k4s_matvec_f64<DPv, kSym64Rows, kSym64Threads, false, false>);
  LAKER_K4S_FN(2) LAKER_K4S_FN(4) LAKER_K4S_FN(6) LAKER_K4S_FN(8) LAKER_K4S_FN(10) LAKER_K4S_FN(12)
  LAKER_K4S_FN(14) LAKER_K4S_FN(16)
#undef LAKER_K4S_FN
  int nb = 0;
  if (!fn || cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, fn, kSym64Threads, 0) != cudaSuccess ||
      nb < 1) {
    cudaGetLastError();
    nb = 1;
  }
  c = nb;
  return c;
}

__global__ void sym_finish_kernel(SymPlan sp, const double* __restrict__ rowpart,
                                  const float* __restrict__ colpart, int64_t n, float lam,
                                  const float* __restrict__ x, float* __restrict__ y, int64_t ldy,
                                  const int* status) {
  const bool failed = status_failed(status);
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x)
    y[i * ldy] = failed ? nan_f32()
                        : (float)((double)lam * (double)x[i] + sym_row_sum(sp, rowpart, colpart, i));
}

// y = [b -] (lam x + K64 x) from the FP64 kernel's partials.
__global__ void sym_finish64_kernel(SymPlan sp, const double* __restrict__ rowpart,
                                    const double* __restrict__ colpart, int64_t n, double lam,
                                    const double* __restrict__ x, const double* __restrict__ b,
                                    int64_t ldb, double* __restrict__ y, int64_t ldy,
                                    const int* status) {
  const bool failed = status_failed(status);
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x) {
    const double a = lam * x[i] + sym_row_sum(sp, rowpart, colpart, i);
    y[i * ldy] = failed ? nan_f64() : (b ? b[i * ldb] - a : a);
  }
}

}  // namespace

int sym_block_points() { return kSymRows * kSymThreads; }

SymPlan k1s_plan_pairs(int64_t nb, int64_t npairs, int d) {
  SymPlan sp{};
  sp.B = kSymRows * kSymThreads;
  sp.nb = nb;
  sp.npairs = npairs;
  const int64_t slots = (int64_t)sm_count() * k1s_occupancy(padded_dim(d));
  sp.grid = (int)(npairs < slots ? (npairs > 0 ? npairs : 1) : slots);
  sp.q = npairs / sp.grid;
  sp.rem = npairs % sp.grid;
  sp.cfg = 0;
  return sp;
}

SymPlan k1s_plan(int64_t n, int d) {
  const int B = kSymRows * kSymThreads;
  const int64_t nb = n > 0 ? ceil_div(n, B) : 1;
  return k1s_plan_pairs(nb, nb * (nb + 1) / 2, d);
}

cudaError_t launch_k1s(const float* E32, int64_t n, int d, int clamp, const float* x,
                       double* rowpart, float* colpart, const SymPlan& sp, int* status,
                       const int* gate, cudaStream_t s) {
  const int dp = padded_dim(d);
  const BatchMap none{};
  if (clamp) {
    LAKER_DISPATCH_DPS(dp, return (launch_k1s_t<DPv, true, false>(E32, n, x, rowpart, colpart, sp, none, status, gate, s)));
  } else {
    LAKER_DISPATCH_DPS(dp, return (launch_k1s_t<DPv, false, false>(E32, n, x, rowpart, colpart, sp, none, status, gate, s)));
  }
  return cudaErrorInvalidValue;
}

cudaError_t launch_k1s_batched(const float* E32, int d, int clamp, const float* x,
                               double* rowpart, float* colpart, const SymPlan& sp,
                               const BatchMap& bm, int* status, const int* gate, cudaStream_t s) {
  const int dp = padded_dim(d);
  if (clamp) {
    LAKER_DISPATCH_DPS(dp, return (launch_k1s_t<DPv, true, true>(E32, 0, x, rowpart, colpart, sp, bm, status, gate, s)));
  } else {
    LAKER_DISPATCH_DPS(dp, return (launch_k1s_t<DPv, false, true>(E32, 0, x, rowpart, colpart, sp, bm, status, gate, s)));
  }
  return cudaErrorInvalidValue;
}

cudaError_t launch_sym_finish(const SymPlan& sp, const double* rowpart, const float* colpart,
                              int64_t n, float lam, const float* x, float* y, int64_t ldy,
                              const int* status, cudaStream_t s) {
  int g = (int)ceil_div(n, 256);
  if (g > sm_count() * 8) g = sm_count() * 8;
  sym_finish_kernel<<<g, 256, 0, s>>>(sp, rowpart, colpart, n, lam, x, y, ldy, status);
  return cudaGetLastError();
}

SymPlan k4s_plan_pairs(int64_t nb, int64_t npairs, int d) {
  SymPlan sp{};
  sp.B = kSym64Rows * kSym64Threads;
  sp.nb = nb;
  sp.npairs = npairs;
  const int64_t slots = (int64_t)sm_count() * k4s_occupancy(padded_dim(d));
  sp.grid = (int)(npairs < slots ? (npairs > 0 ? npairs : 1) : slots);
  sp.q = npairs / sp.grid;
  sp.rem = npairs % sp.grid;
  sp.cfg = 0;
  return sp;
}

SymPlan k4s_plan(int64_t n, int d) {
  const int B = kSym64Rows * kSym64Threads;
  const int64_t nb = n > 0 ? ceil_div(n, B) : 1;
  return k4s_plan_pairs(nb, nb * (nb + 1) / 2, d);
}

cudaError_t launch_k4s(const double* E64, int64_t n, int d, int clamp, const double* x,
                       double* rowpart, double* colpart, const SymPlan& sp, int* status,
                       const int* gate, cudaStream_t s) {
  const int dp = padded_dim(d);
  const BatchMap none{};
  if (clamp) {
    LAKER_DISPATCH_DPS(dp, return (launch_k4s_t<DPv, true, false>(E64, n, x, rowpart, colpart, sp, none, status, gate, s)));
  } else {
    LAKER_DISPATCH_DPS(dp, return (launch_k4s_t<DPv, false, false>(E64, n, x, rowpart, colpart, sp, none, status, gate, s)));
  }
  return cudaErrorInvalidValue;
}

cudaError_t launch_k4s_batched(const double* E64, int d, int clamp, const double* x,
                               double* rowpart, double* colpart, const SymPlan& sp,
                               const BatchMap& bm, int* status, const int* gate, cudaStream_t s) {
  const int dp = padded_dim(d);
  if (clamp) {
    LAKER_DISPATCH_DPS(dp, return (launch_k4s_t<DPv, true, true>(E64, 0, x, rowpart, colpart, sp, bm, status, gate, s)));
  } else {
    LAKER_DISPATCH_DPS(dp, return (launch_k4s_t<DPv, false, true>(E64, 0, x, rowpart, colpart, sp, bm, status, gate, s)));
  }
  return cudaErrorInvalidValue;
}

cudaError_t launch_sym_finish64(const SymPlan& sp, const double* rowpart, const double* colpart,
                                int64_t n, double lam, const double* x, const double* b,
                                int64_t ldb, double* y, int64_t ldy, const int* status,
                                cudaStream_t s) {
  int g = (int)ceil_div(n, 256);
  if (g > sm_count() * 8) g = sm_count() * 8;
  sym_finish64_kernel<<<g, 256, 0, s>>>(sp, rowpart, colpart, n, lam, x, b, ldb, y, ldy, status);
  return cudaGetLastError();
}

cudaError_t set_wait_limit_sym(unsigned long long ns) { return set_wait_limit_this_unit(ns); }

// Square operators of at most LAKER_VARIANT_SYM_MIN_BLOCKS 512-point blocks
// (default 6: n <= 3072, at most 21 block pairs, so as many CTAs) run the
// plain fused kernel, which spreads the rows over the whole GPU.
bool k1_symmetric_for(int64_t n) {
  const int64_t min_blocks = variant_get(LAKER_VARIANT_SYM_MIN_BLOCKS);
  return k1_use_symmetric() && n > 0 && n > min_blocks * kSymRows * kSymThreads;
}

bool k1_use_symmetric() {
  static int v = -1;
  if (v < 0) {
    const char* e = getenv("LAKER_K1_SYMMETRIC");
    v = (e && e[0] == '0') ? 0 : 1;
  }
  return v == 1;
}

bool k4_use_symmetric() {
  static int v = -1;
  if (v < 0) {
    const char* e = getenv("LAKER_K4_SYMMETRIC");
    v = (e && e[0] == '0') ? 0 : 1;
  }
  return v == 1;
}

}  // namespace laker

using namespace laker;

extern "C" int laker_fp32_matvec_work(int64_t n, int d, double* entries, double* flops,
                                      double* exps) {
  if (n < 0 || d < 1 || d > 16) return LAKER_ERR_INVALID_ARG;
  const double nn = (double)n * (double)n;
  double e, f;
  if (k1_symmetric_for(n)) {
    // diagonal block pairs: every entry evaluated, used once (row sums);
    // off-diagonal pairs: evaluated once, used twice (row and column sums)
    const SymPlan sp = k1s_plan(n, d);
    const double B = (double)sp.B;
    const double last = (double)(n - (sp.nb - 1) * sp.B);
    const double diag = (double)(sp.nb - 1) * B * B + last * last;
    const double off = (nn - diag) * 0.5;
    e = diag + off;
    // tensor-core logits: the CUDA cores do only the accumulation FMAs
    f = k1t_enabled(d) ? 2.0 * (diag + 2.0 * off) : 2.0 * (diag * (d + 1) + off * (d + 2));
  } else {
    e = nn;
    f = 2.0 * nn * (d + 1);
  }
  if (entries) *entries = e;
  if (flops) *flops = f;
  if (exps) *exps = e;
  return LAKER_OK;
}

extern "C" int laker_fp32_operator_kernel(int64_t n, int d) {
  if (n < 0 || d < 1 || d > 16) return -1;
  if (!k1_symmetric_for(n)) return 0;
  return k1t_enabled(d) ? 2 : 1;
}
