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
// are kept across the consecutive pairs of one row block and stored once per
// (CTA, row block) run.  A fixed-order finish adds both partial sets, so the
// result is deterministic.  Work per computed entry: d FMA + 2 FMA + 1 exp2,
// i.e. (d + 2) / 2 FMA and 1/2 exp2 per logical entry.
#include <cstdlib>

#include "sym.cuh"

namespace laker {
namespace {

template <int DP, int R, int T, bool CLAMP>
__global__ void __launch_bounds__(T, 3)
    k1s_matvec_f32(const float* __restrict__ E, int64_t n, const float* __restrict__ x,
                   float* __restrict__ colpart, double* __restrict__ rowpart, SymPlan sp,
                   int* status, const int* gate) {
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

  // ---- the CTA's flat tile sequence: (pair, tile-in-block), skipping tiles
  // that start at or beyond n (they hold no points).
  auto tile_col0 = [&](int64_t b, int t) -> int64_t { return b * B + (int64_t)t * TC; };
  int64_t a0, b0;
  sym_pair_coords(p_begin, sp.nb, &a0, &b0);

  if (tid == 0) {
    mbar_init(&bar[0], 1);
    mbar_init(&bar[1], 1);
    mbar_fence_init();
  }
  __syncthreads();

  auto issue = [&](int64_t col0, int buf) {
    mbar_arrive_expect_tx(&bar[buf], TILE_FLOATS * 4);
    bulk_g2s(sE[buf], E + (col0 >> 1) * (DP * 2), TILE_FLOATS * 4, &bar[buf]);
  };
  auto load_x = [&](int64_t col0, int buf) {
    for (int j = tid; j < TC; j += T) {
      const int64_t cc = col0 + j;
      sX[buf][j] = (cc < n) ? x[cc] : 0.0f;
    }
  };

  // iteration state: current pair (pa, pb), tile t within block pb
  int64_t pa = a0, pb = b0, p = p_begin;
  int t = 0;
  // next-tile cursor for prefetching
  int64_t na = a0, nbk = b0, np = p_begin;
  int nt = 0;
  auto advance = [&](int64_t& qa, int64_t& qb, int64_t& qp, int& qt) {
    // move to the next valid tile of the sequence
    for (;;) {
      if (++qt >= TPB || tile_col0(qb, qt) >= n) {
        qt = 0;
        ++qp;
        if (qp >= p_end) return;
        if (++qb >= sp.nb) {
          ++qa;
          qb = qa;
        }
      }
      if (tile_col0(qb, qt) < n) return;
    }
  };

  // rows of block pa in registers
  float2 ev[R][DP];
  float2 xr[R];
  double acc[R];
  auto load_rows = [&](int64_t a) {
#pragma unroll
    for (int r = 0; r < R; ++r) {
      const int64_t i = a * B + r * T + tid;
      const bool ok = i < n;
      const float* blk = E + (i >> 1) * (DP * 2) + (i & 1);
#pragma unroll
      for (int k = 0; k < DP; ++k) {
        const float v = ok ? blk[2 * k] * kLog2e : 0.0f;
        ev[r][k] = make_float2(v, v);
      }
      const float xi = ok ? x[i] : 0.0f;
      xr[r] = make_float2(xi, xi);
      acc[r] = 0.0;
    }
  };
  auto flush_rows = [&](int64_t a) {
    double* dst = rowpart + (c + a) * (int64_t)B;
#pragma unroll
    for (int r = 0; r < R; ++r) dst[r * T + tid] = acc[r];
  };

  load_rows(pa);
  // first tile
  if (tid == 0) issue(tile_col0(nbk, nt), 0);
  load_x(tile_col0(nbk, nt), 0);
  advance(na, nbk, np, nt);
  __syncthreads();

  int k_tile = 0, issued = 1, consumed = 0;
  bool failed = false;
  while (p < p_end) {
    const int buf = k_tile & 1;
    const bool have_next = np < p_end;
    if (have_next) {
      const int64_t col0 = tile_col0(nbk, nt);
      if (tid == 0) issue(col0, buf ^ 1);
      load_x(col0, buf ^ 1);
      ++issued;
    }
    const int ok = __syncthreads_and(mbar_wait_bounded(&bar[buf], (k_tile >> 1) & 1, status) ? 1 : 0);
    if (!ok) {
      failed = true;
      break;
    }
    ++consumed;
    const bool offdiag = pa != pb;
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
      // this tile's column sums (columns t*TC .. t*TC+TC-1 of block pb)
      for (int j = tid; j < TC; j += T) {
        float s = 0.0f;
#pragma unroll
        for (int w = 0; w < NW; ++w) s += sCol[w][j];
        colpart[sym_pair_index(pa, pb, sp.nb) * (int64_t)B + t * TC + j] = s;
      }
    }
    __syncthreads();  // sCol is reused by the next tile

    // advance the consumer cursor
    const int64_t prev_a = pa;
    ++k_tile;
    {
      int64_t qa = pa, qb = pb, qp = p;
      int qt = t;
      advance(qa, qb, qp, qt);
      pa = qa;
      pb = qb;
      p = qp;
      t = qt;
    }
    if (p >= p_end || pa != prev_a) {
      flush_rows(prev_a);
      if (p < p_end) load_rows(pa);
    }
    if (have_next) advance(na, nbk, np, nt);
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

template <int DP, bool CLAMP>
cudaError_t launch_k1s_t(const float* E, int64_t n, const float* x, double* rowpart,
                         float* colpart, const SymPlan& sp, int* status, const int* gate,
                         cudaStream_t s) {
  k1s_matvec_f32<DP, kSymRows, kSymThreads, CLAMP>
      <<<sp.grid, kSymThreads, 0, s>>>(E, n, x, colpart, rowpart, sp, status, gate);
  return cudaGetLastError();
}

int k1s_occupancy(int dp) {
  static int cache[9] = {};
  if (dp < 2 || dp > 16) return 2;
  int& c = cache[dp / 2];
  if (c > 0) return c;
  const void* fn = nullptr;
#define LAKER_K1S_FN(DPv) \
  if (dp == DPv) fn = reinterpret_cast<const void*>(&k1s_matvec_f32<DPv, kSymRows, kSymThreads, false>);
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

}  // namespace

SymPlan k1s_plan(int64_t n, int d) {
  SymPlan sp{};
  sp.B = kSymRows * kSymThreads;
  sp.nb = n > 0 ? ceil_div(n, sp.B) : 1;
  sp.npairs = sp.nb * (sp.nb + 1) / 2;
  const int64_t slots = (int64_t)sm_count() * k1s_occupancy(padded_dim(d));
  sp.grid = (int)(sp.npairs < slots ? sp.npairs : slots);
  sp.q = sp.npairs / sp.grid;
  sp.rem = sp.npairs % sp.grid;
  sp.cfg = 0;
  return sp;
}

cudaError_t launch_k1s(const float* E32, int64_t n, int d, int clamp, const float* x,
                       double* rowpart, float* colpart, const SymPlan& sp, int* status,
                       const int* gate, cudaStream_t s) {
  const int dp = padded_dim(d);
  if (clamp) {
    LAKER_DISPATCH_DPS(dp, return (launch_k1s_t<DPv, true>(E32, n, x, rowpart, colpart, sp, status, gate, s)));
  } else {
    LAKER_DISPATCH_DPS(dp, return (launch_k1s_t<DPv, false>(E32, n, x, rowpart, colpart, sp, status, gate, s)));
  }
  return cudaErrorInvalidValue;
}

}  // namespace laker

namespace laker {
namespace {

__global__ void sym_finish_kernel(SymPlan sp, const double* __restrict__ rowpart,
                                  const float* __restrict__ colpart, int64_t n, float lam,
                                  const float* __restrict__ x, float* __restrict__ y, int64_t ldy) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x)
    y[i * ldy] = (float)((double)lam * (double)x[i] + sym_row_sum(sp, rowpart, colpart, i));
}

}  // namespace

cudaError_t launch_sym_finish(const SymPlan& sp, const double* rowpart, const float* colpart,
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
