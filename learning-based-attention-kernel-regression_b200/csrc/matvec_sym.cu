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
// (BatchMap): the pair list is the concatenation of the instances' pair
// lists, so the operator is block diagonal; converged instances are skipped.
#include <cstdlib>

#include "sym.cuh"

namespace laker {
namespace {

// Position in a CTA's flat sequence of column tiles (pair p, tile t of block b).
struct SymCursor {
  int64_t p, p_end;
  int inst;
  int64_t a, b;
  int t;
  // metadata of instance `inst`
  int64_t nb, npts, seg, blk0, pstart, pend;
};

template <bool BATCHED>
__device__ __forceinline__ void cursor_load_inst(SymCursor& cu, const SymPlan& sp,
                                                 const BatchMap& bm, int64_t n) {
  if (BATCHED) {
    cu.nb = bm.nblk[cu.inst];
    cu.npts = bm.npts[cu.inst];
    cu.seg = bm.seg[cu.inst];
    cu.blk0 = bm.blk_start[cu.inst];
    cu.pstart = bm.pair_start[cu.inst];
    cu.pend = bm.pair_start[cu.inst + 1];
  } else {
    cu.nb = sp.nb;
    cu.npts = n;
    cu.seg = 0;
    cu.blk0 = 0;
    cu.pstart = 0;
    cu.pend = sp.npairs;
  }
}

// Place the cursor on tile 0 of pair p, moving past finished instances.
// Returns false when the CTA's range is exhausted.
template <bool BATCHED>
__device__ __forceinline__ bool cursor_settle(SymCursor& cu, const SymPlan& sp, const BatchMap& bm,
                                              int64_t n) {
  for (;;) {
    if (cu.p >= cu.p_end) return false;
    if (BATCHED) {
      while (cu.p >= cu.pend) {
        ++cu.inst;
        cursor_load_inst<BATCHED>(cu, sp, bm, n);
      }
      if (bm.done && bm.done[cu.inst]) {
        cu.p = cu.pend;
        continue;
      }
    }
    sym_pair_coords(cu.p - cu.pstart, cu.nb, &cu.a, &cu.b);
    cu.t = 0;
    return true;
  }
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
                   float* __restrict__ colpart, float* __restrict__ rowpart, SymPlan sp,
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
  const int64_t p_begin = c * sp.q + (c < sp.rem ? c : sp.rem);
  const int64_t p_end = p_begin + sp.q + (c < sp.rem ? 1 : 0);
  if (p_begin >= p_end) return;

  // consumer cursor (cu) and prefetch cursor (nx) over the same tile sequence
  SymCursor cu;
  cu.p = p_begin;
  cu.p_end = p_end;
  cu.inst = 0;
  if (BATCHED) {
    // instance of the first pair: binary search of pair_start
    int lo = 0, hi = bm.count - 1;
    while (lo < hi) {
      const int mid = (lo + hi + 1) >> 1;
      if (bm.pair_start[mid] <= p_begin) lo = mid; else hi = mid - 1;
    }
    cu.inst = lo;
  }
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

  // rows of block (cu.inst, cu.a) in registers; row sums of the current pair
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
    float* dst = rowpart + pair * (int64_t)B;
#pragma unroll
    for (int r = 0; r < R; ++r) {
      dst[r * T + tid] = (float)acc[r];
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
        // warp reduction of the 16 column partials (fixed butterfly order)
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
#pragma unroll
          for (int u = 0; u < 8; ++u) {
            cs[u].x += __shfl_xor_sync(0xffffffffu, cs[u].x, o);
            cs[u].y += __shfl_xor_sync(0xffffffffu, cs[u].y, o);
          }
        }
        if (lane < 8) {
          // lane u stores column pair q0 + u (a register select per lane)
          float2 mine = cs[0];
#pragma unroll
          for (int u = 1; u < 8; ++u)
            if (lane == u) mine = cs[u];
          reinterpret_cast<float2*>(sCol[warp])[q0 + lane] = mine;
        }
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
        colpart[cu.p * (int64_t)B + cu.t * TC + j] = s;
      }
    }
    __syncthreads();  // sCol is reused by the next tile

    // advance the consumer; store the row sums when the pair changes and
    // reload the rows when the row block changes
    const int64_t prev_pair = cu.p, prev_block = cu.blk0 + cu.a;
    const bool more = cursor_next<BATCHED, B, TC, TPB>(cu, sp, bm, n);
    ++k_tile;
    if (!more || cu.p != prev_pair) flush_rows(prev_pair);
    if (more && cu.blk0 + cu.a != prev_block) load_rows(cu);
    if (!more) break;
    if (have_nx) have_nx = cursor_next<BATCHED, B, TC, TPB>(nx, sp, bm, n);
  }
  if (failed) {
    for (int k = consumed + 1; k < issued; ++k) mbar_wait_bounded(&bar[k & 1], (k >> 1) & 1, status);
  }
}

}  // namespace
}  // namespace laker

namespace laker {
namespace {

constexpr int kSymRows = 4;      // rows per thread
constexpr int kSymThreads = 128;  // threads per CTA -> B = 512 points per block

template <int DP, bool CLAMP, bool BATCHED>
cudaError_t launch_k1s_t(const float* E, int64_t n, const float* x, float* rowpart,
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

__global__ void sym_finish_kernel(SymPlan sp, const float* __restrict__ rowpart,
                                  const float* __restrict__ colpart, int64_t n, float lam,
                                  const float* __restrict__ x, float* __restrict__ y, int64_t ldy) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x)
    y[i * ldy] = (float)((double)lam * (double)x[i] + sym_row_sum(sp, rowpart, colpart, i));
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
                       float* rowpart, float* colpart, const SymPlan& sp, int* status,
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
                               float* rowpart, float* colpart, const SymPlan& sp,
                               const BatchMap& bm, int* status, const int* gate, cudaStream_t s) {
  const int dp = padded_dim(d);
  if (clamp) {
    LAKER_DISPATCH_DPS(dp, return (launch_k1s_t<DPv, true, true>(E32, 0, x, rowpart, colpart, sp, bm, status, gate, s)));
  } else {
    LAKER_DISPATCH_DPS(dp, return (launch_k1s_t<DPv, false, true>(E32, 0, x, rowpart, colpart, sp, bm, status, gate, s)));
  }
  return cudaErrorInvalidValue;
}

cudaError_t launch_sym_finish(const SymPlan& sp, const float* rowpart, const float* colpart,
                              int64_t n, float lam, const float* x, float* y, int64_t ldy,
                              cudaStream_t s) {
  int g = (int)ceil_div(n, 256);
  if (g > sm_count() * 8) g = sm_count() * 8;
  sym_finish_kernel<<<g, 256, 0, s>>>(sp, rowpart, colpart, n, lam, x, y, ldy);
  return cudaGetLastError();
}

bool k1_use_symmetric() {
  static int v = -1;
  if (v < 0) {
    const char* e = getenv("LAKER_K1_SYMMETRIC");
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
  if (k1_use_symmetric() && n > 0) {
    // diagonal block pairs: every entry evaluated, used once (row sums);
    // off-diagonal pairs: evaluated once, used twice (row and column sums)
    const SymPlan sp = k1s_plan(n, d);
    const double B = (double)sp.B;
    const double last = (double)(n - (sp.nb - 1) * sp.B);
    const double diag = (double)(sp.nb - 1) * B * B + last * last;
    const double off = (nn - diag) * 0.5;
    e = diag + off;
    f = 2.0 * (diag * (d + 1) + off * (d + 2));
  } else {
    e = nn;
    f = 2.0 * nn * (d + 1);
  }
  if (entries) *entries = e;
  if (flops) *flops = f;
  if (exps) *exps = e;
  return LAKER_OK;
}
