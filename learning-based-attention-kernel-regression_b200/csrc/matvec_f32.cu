// FP32 fused attention-kernel matvec (the operator applied inside the PCG
// loop) and the CUDA-core multi-RHS variant.
//
// Single RHS (K1).  Each CTA owns T*R rows and one column segment.  Column
// embeddings arrive in shared memory through 1-D TMA bulk copies of the packed
// pair layout (double-buffered, mbarrier-completed); x is staged with plain
// loads.  Every thread keeps its R rows (scaled by log2 e and duplicated into
// both halves of a float2) in registers and walks the staged columns two at a
// time: the logit of a column pair is 2*DP packed FMAs (FFMA2), the kernel
// entries come from MUFU ex2, and the accumulation is one more FFMA2.  Each
// CTA reduces its segment into FP64 row partials; nothing of size n^2 is ever
// stored.  Algorithmic work per entry: d FMA (logit) + 1 FMA (accumulate) +
// 1 exp2.
#include <cstdlib>

#include "internal.cuh"
#include "sym.cuh"

namespace laker {
namespace {

constexpr int kK1Threads = 256;
constexpr int kK1Rows = 2;  // rows per thread

template <int DP, int R, int T, bool CLAMP>
__global__ void __launch_bounds__(T, 2)
    k1_matvec_f32(const float* __restrict__ rows, int64_t m, const float* __restrict__ cols,
                  int64_t n, const float* __restrict__ x, double* __restrict__ part,
                  int64_t cols_per_seg, int* status, const int* gate) {
  if (gate && *gate == 0) return;
  constexpr int TC = kTileCols32;
  constexpr int TP = TC / 2;
  constexpr int TILE_FLOATS = TC * DP;
  __shared__ __align__(128) float sE[2][TILE_FLOATS];
  __shared__ __align__(16) float sX[2][TC];
  __shared__ __align__(8) uint64_t bar[2];

  const int tid = threadIdx.x;
  const int64_t row0 = (int64_t)blockIdx.x * (T * R);
  const int64_t c_begin = (int64_t)blockIdx.y * cols_per_seg;
  const int64_t c_end = min(n, c_begin + cols_per_seg);
  const int ntiles = c_begin < c_end ? (int)ceil_div(c_end - c_begin, TC) : 0;

  // Row embeddings in registers, log2(e) folded in, duplicated per half.
  float2 ev[R][DP];
#pragma unroll
  for (int r = 0; r < R; ++r) {
    const int64_t i = row0 + r * T + tid;
    const float* blk = rows + (i >> 1) * (DP * 2) + (i & 1);
#pragma unroll
    for (int k = 0; k < DP; ++k) {
      const float v = (i < m) ? blk[2 * k] * kLog2e : 0.0f;
      ev[r][k] = make_float2(v, v);
    }
  }
  double acc[R];
#pragma unroll
  for (int r = 0; r < R; ++r) acc[r] = 0.0;

  if (tid == 0) {
    mbar_init(&bar[0], 1);
    mbar_init(&bar[1], 1);
    mbar_fence_init();
  }
  __syncthreads();

  auto issue = [&](int t, int b) {
    const int64_t c0 = c_begin + (int64_t)t * TC;
    mbar_arrive_expect_tx(&bar[b], TILE_FLOATS * 4);
    bulk_g2s(sE[b], cols + (c0 >> 1) * (DP * 2), TILE_FLOATS * 4, &bar[b]);
  };
  auto load_x = [&](int t, int b) {
    const int64_t c0 = c_begin + (int64_t)t * TC;
    for (int j = tid; j < TC; j += T) {
      const int64_t c = c0 + j;
      sX[b][j] = (c < c_end) ? x[c] : 0.0f;
    }
  };

  if (ntiles > 0) {
    if (tid == 0) issue(0, 0);
    load_x(0, 0);
  }
  __syncthreads();

  int issued = ntiles > 0 ? 1 : 0, consumed = 0;
  for (int t = 0; t < ntiles; ++t) {
    const int b = t & 1;
    if (t + 1 < ntiles) {
      if (tid == 0) issue(t + 1, b ^ 1);
      load_x(t + 1, b ^ 1);
      ++issued;
    }
    const int ok = __syncthreads_and(mbar_wait_bounded(&bar[b], (t >> 1) & 1, status) ? 1 : 0);
    if (!ok) break;
    ++consumed;

    const float* E = sE[b];
    const float2* X2 = reinterpret_cast<const float2*>(sX[b]);
    float2 tacc[R];
#pragma unroll
    for (int r = 0; r < R; ++r) tacc[r] = make_float2(0.0f, 0.0f);
#pragma unroll 2
    for (int q = 0; q < TP; ++q) {
      const float4* cp = reinterpret_cast<const float4*>(E + q * (DP * 2));
      float2 c[DP];
#pragma unroll
      for (int h = 0; h < DP / 2; ++h) {
        const float4 v = cp[h];
        c[2 * h] = make_float2(v.x, v.y);
        c[2 * h + 1] = make_float2(v.z, v.w);
      }
      const float2 xv = X2[q];
#pragma unroll
      for (int r = 0; r < R; ++r) {
        float2 s = __fmul2_rn(ev[r][0], c[0]);
#pragma unroll
        for (int k = 1; k < DP; ++k) s = __ffma2_rn(ev[r][k], c[k], s);
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
#pragma unroll
    for (int r = 0; r < R; ++r) acc[r] += (double)tacc[r].x + (double)tacc[r].y;
    __syncthreads();  // buffer b is refilled by the next iteration's issue
  }

  if (consumed < ntiles) {
    // A wait expired: drain (bounded) any copy still in flight, then leave.
    for (int t = consumed; t < issued; ++t) mbar_wait_drain(&bar[t & 1], (t >> 1) & 1, status);
    return;
  }

#pragma unroll
  for (int r = 0; r < R; ++r) {
    const int64_t i = row0 + r * T + tid;
    if (i < m) part[(int64_t)blockIdx.y * m + i] = acc[r];
  }
}

// K1 variants: rows per thread x threads per CTA.  Variant 0 is compiled for
// every padded dimension; the others only for d = 9..10 (the LAKER default),
// where the tile-shape autotuner picks among them.
struct K1Variant {
  int rows, threads;
};
constexpr K1Variant kK1Variants[] = {{2, 256}, {4, 256}, {2, 128}, {4, 128}, {3, 256}};
constexpr int kK1NumVariants = sizeof(kK1Variants) / sizeof(kK1Variants[0]);

template <int DP, int R, int TT, bool CLAMP>
cudaError_t launch_k1_rt(const float* rows, int64_t m, const float* cols, int64_t n,
                         const float* x, double* part, const SegPlan& p, int* status,
                         const int* gate, cudaStream_t s) {
  dim3 grid((unsigned)ceil_div(m, TT * R), (unsigned)p.S);
  k1_matvec_f32<DP, R, TT, CLAMP>
      <<<grid, TT, 0, s>>>(rows, m, cols, n, x, part, p.cols_per_seg, status, gate);
  return cudaGetLastError();
}

template <int DP, bool CLAMP>
cudaError_t launch_k1_t(const float* rows, int64_t m, const float* cols, int64_t n,
                        const float* x, double* part, const SegPlan& p, int* status,
                        const int* gate, cudaStream_t s) {
  if constexpr (DP == 10) {
    switch (p.cfg) {
      case 1: return launch_k1_rt<DP, 4, 256, CLAMP>(rows, m, cols, n, x, part, p, status, gate, s);
      case 2: return launch_k1_rt<DP, 2, 128, CLAMP>(rows, m, cols, n, x, part, p, status, gate, s);
      case 3: return launch_k1_rt<DP, 4, 128, CLAMP>(rows, m, cols, n, x, part, p, status, gate, s);
      case 4: return launch_k1_rt<DP, 3, 256, CLAMP>(rows, m, cols, n, x, part, p, status, gate, s);
      default: break;
    }
  }
  return launch_k1_rt<DP, kK1Rows, kK1Threads, CLAMP>(rows, m, cols, n, x, part, p, status, gate, s);
}

// Resident CTAs per SM of a K1 variant (occupancy API; 2 when unavailable).
int k1_occupancy(int cfg, int dp) {
  static int cache[kK1NumVariants][9] = {};
  if (cfg < 0 || cfg >= kK1NumVariants || dp < 2 || dp > 16) return 2;
  int& c = cache[cfg][dp / 2];
  if (c > 0) return c;
  int nb = 0;
  cudaError_t e = cudaErrorInvalidValue;
  const void* fn = nullptr;
#define LAKER_K1_FN(DPv)                                                               \
  if (dp == DPv) fn = reinterpret_cast<const void*>(&k1_matvec_f32<DPv, kK1Rows, kK1Threads, false>);
  LAKER_K1_FN(2) LAKER_K1_FN(4) LAKER_K1_FN(6) LAKER_K1_FN(8) LAKER_K1_FN(12) LAKER_K1_FN(14)
  LAKER_K1_FN(16)
#undef LAKER_K1_FN
  if (dp == 10) {
    switch (cfg) {
      case 1: fn = reinterpret_cast<const void*>(&k1_matvec_f32<10, 4, 256, false>); break;
      case 2: fn = reinterpret_cast<const void*>(&k1_matvec_f32<10, 2, 128, false>); break;
      case 3: fn = reinterpret_cast<const void*>(&k1_matvec_f32<10, 4, 128, false>); break;
      case 4: fn = reinterpret_cast<const void*>(&k1_matvec_f32<10, 3, 256, false>); break;
      default: fn = reinterpret_cast<const void*>(&k1_matvec_f32<10, kK1Rows, kK1Threads, false>);
    }
  }
  const int threads = (dp == 10) ? kK1Variants[cfg].threads : kK1Threads;
  if (fn) e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, fn, threads, 0);
  if (e != cudaSuccess || nb < 1) {
    cudaGetLastError();
    nb = 2;
  }
  c = nb;
  return c;
}

// Variant choice: LAKER_K1_VARIANT overrides (tuning sweeps); otherwise the
// default variant.
int k1_variant(int dp) {
  if (dp != 10) return 0;
  static int v = -1;
  if (v < 0) {
    const char* s = getenv("LAKER_K1_VARIANT");
    v = s ? atoi(s) : 0;
    if (v < 0 || v >= kK1NumVariants) v = 0;
  }
  return v;
}

// ---------------------------------------------------------------------------
// Multi-RHS fused matvec on CUDA cores: Y = lam X + exp(Er Ec^T) X for
// X (n x k).  A CTA owns a 64-row x 64-RHS output tile; per 32-column step it
// evaluates the 64 x 32 block of kernel entries into shared memory (each
// thread keeps one row embedding in registers) and multiplies it into X with
// 4 x 4 register microtiles.  Row sums are flushed to FP64 every 256 columns.
// Real = float: exp2 on MUFU with log2 e folded into the rows; Real = double:
// FP64 logits and exp (the accurate operator, optionally as a residual).
// Narrow products (k <= 16, e.g. the FP64 residual of a variance solve with
// few queries) use 64 x 16 tiles of 64 threads instead, so that no
// accumulation FMA lands on an absent right-hand side (LAKER_MULTI_NARROW=0
// keeps the 64-wide tile for comparisons).
// ---------------------------------------------------------------------------
constexpr int kMBM = 64, kMBN = 64, kMBK = 32, kMThreads = 256;
constexpr int kMBNNarrow = 16;

bool multi_narrow_enabled() {
  static int v = -1;
  if (v < 0) {
    const char* e = getenv("LAKER_MULTI_NARROW");
    v = (e && e[0] == '0') ? 0 : 1;
  }
  return v == 1;
}

}  // namespace

template <typename Real, int DP, bool CLAMP, bool RESIDUAL, int BN = kMBN>
__global__ void __launch_bounds__((kMBM / 4) * (BN / 4))
    multi_matvec_kernel(const Real* __restrict__ rows, int64_t m, const Real* __restrict__ cols,
                        int64_t n, int col_layout_pairs, Real lam, const Real* __restrict__ X,
                        int k, int64_t ldx, const Real* __restrict__ B, int64_t ldb,
                        Real* __restrict__ Y, int64_t ldy, int row_layout_pairs,
                        const int* gate) {
  if (gate && *gate == 0) return;
  constexpr int T = (kMBM / 4) * (BN / 4);  // threads: one 4 x 4 microtile each
  static_assert(T % kMBM == 0 && (kMBM * kMBK) % T == 0, "tile / thread mapping");
  __shared__ __align__(16) Real sCol[kMBK][DP + 1];
  __shared__ __align__(16) Real sP[kMBK][kMBM];
  __shared__ __align__(16) Real sX[kMBK][BN];
  __shared__ double sExp[64];
  const int tid = threadIdx.x;
  if constexpr (sizeof(Real) == 8) exp_table_to_shared(sExp, tid, T);
  const int tx = tid % (BN / 4), ty = tid / (BN / 4);
  const int64_t i0 = (int64_t)blockIdx.x * kMBM;
  const int64_t c0 = (int64_t)blockIdx.y * BN;

  auto emb = [&](const Real* base, int pairs, int64_t i, int kk) -> Real {
    return pairs ? base[(i >> 1) * (DP * 2) + 2 * kk + (i & 1)] : base[i * DP + kk];
  };

  // The row this thread evaluates kernel entries for (fixed for the CTA).
  const int a = tid & (kMBM - 1);
  Real rv[DP];
  {
    const int64_t i = i0 + a;
#pragma unroll
    for (int kk = 0; kk < DP; ++kk) {
      Real v = (i < m) ? emb(rows, row_layout_pairs, i, kk) : Real(0);
      if (sizeof(Real) == 4) v *= (Real)kLog2e;
      rv[kk] = v;
    }
  }
  // FP32: FP32 microtile sums flushed to FP64 every 8 steps; FP64: the
  // microtile accumulates in FP64 directly
  constexpr bool kF64 = sizeof(Real) == 8;
  Real acc[4][4];
  double acc64[kF64 ? 1 : 4][kF64 ? 1 : 4];
#pragma unroll
  for (int u = 0; u < 4; ++u)
#pragma unroll
    for (int v = 0; v < 4; ++v) acc[u][v] = Real(0);
  if constexpr (!kF64) {
#pragma unroll
    for (int u = 0; u < 4; ++u)
#pragma unroll
      for (int v = 0; v < 4; ++v) acc64[u][v] = 0.0;
  }

  // The next step's column embeddings and X tile are loaded into registers
  // while this step computes, and stored into shared memory after it.
  constexpr int kPC = (kMBK * DP + T - 1) / T, kPX = (kMBK * BN) / T;
  static_assert((kMBK * BN) % T == 0, "X tile / thread mapping");
  Real pc[kPC], px[kPX];
  auto fetch = [&](int st) {
    const int64_t j0 = (int64_t)st * kMBK;
#pragma unroll
    for (int t = 0; t < kPC; ++t) {
      const int o = tid + t * T;
      const int jj = o / DP, kk = o - jj * DP;
      const int64_t j = j0 + jj;
      pc[t] = (o < kMBK * DP && j < n) ? emb(cols, col_layout_pairs, j, kk) : Real(0);
    }
#pragma unroll
    for (int t = 0; t < kPX; ++t) {
      const int o = tid + t * T;
      const int jj = o / BN, cc = o - jj * BN;
      const int64_t j = j0 + jj, c = c0 + cc;
      px[t] = (j < n && c < k) ? X[j * ldx + c] : Real(0);
    }
  };
  auto store = [&]() {
#pragma unroll
    for (int t = 0; t < kPC; ++t) {
      const int o = tid + t * T;
      if (o < kMBK * DP) sCol[o / DP][o % DP] = pc[t];
    }
#pragma unroll
    for (int t = 0; t < kPX; ++t) {
      const int o = tid + t * T;
      sX[o / BN][o % BN] = px[t];
    }
  };

  const int nsteps = (int)ceil_div(n, kMBK);
  if (nsteps > 0) {
    fetch(0);
    store();
  }
  for (int st = 0; st < nsteps; ++st) {
    __syncthreads();
    if (st + 1 < nsteps) fetch(st + 1);
#pragma unroll
    for (int q = 0; q < (kMBM * kMBK) / T; ++q) {
      const int jj = tid / kMBM + (T / kMBM) * q;
      Real s = rv[0] * sCol[jj][0];
#pragma unroll
      for (int kk = 1; kk < DP; ++kk) s = fma(rv[kk], sCol[jj][kk], s);
      Real e;
      if constexpr (sizeof(Real) == 4) {
        if (CLAMP) s = fminf(s, kClampLog2);
        e = ex2_approx(s);
      } else {
        if (CLAMP) s = fmin(s, kClamp64);
        e = exp_tab(s, sExp);
      }
      sP[jj][a] = e;
    }
    __syncthreads();
#pragma unroll 8
    for (int jj = 0; jj < kMBK; ++jj) {
      Real pa[4], xb[4];
#pragma unroll
      for (int u = 0; u < 4; ++u) pa[u] = sP[jj][ty * 4 + u], xb[u] = sX[jj][tx * 4 + u];
#pragma unroll
      for (int u = 0; u < 4; ++u)
#pragma unroll
        for (int v = 0; v < 4; ++v) acc[u][v] = fma(pa[u], xb[v], acc[u][v]);
    }
    if constexpr (!kF64) {
      if ((st & 7) == 7 || st == nsteps - 1) {
#pragma unroll
        for (int u = 0; u < 4; ++u)
#pragma unroll
          for (int v = 0; v < 4; ++v) acc64[u][v] += (double)acc[u][v], acc[u][v] = Real(0);
      }
    }
    __syncthreads();
    if (st + 1 < nsteps) store();
  }

  const bool square = (m == n);
#pragma unroll
  for (int u = 0; u < 4; ++u) {
    const int64_t i = i0 + ty * 4 + u;
    if (i >= m) continue;
#pragma unroll
    for (int v = 0; v < 4; ++v) {
      const int64_t c = c0 + tx * 4 + v;
      if (c >= k) continue;
      double y;
      if constexpr (kF64) y = acc[u][v];
      else y = acc64[u][v];
      if (square) y += (double)lam * (double)X[i * ldx + c];
      if (RESIDUAL) y = (double)B[i * ldb + c] - y;
      Y[i * ldy + c] = (Real)y;
    }
  }
}

namespace {

template <int DP, bool CLAMP>
cudaError_t launch_multi_f32_t(const float* rows, int64_t m, const float* cols, int64_t n, float lam,
                               const float* X, int k, int64_t ldx, float* Y, int64_t ldy,
                               cudaStream_t s, const int* gate) {
  if (k <= kMBNNarrow && multi_narrow_enabled()) {
    dim3 grid((unsigned)ceil_div(m, kMBM), 1);
    multi_matvec_kernel<float, DP, CLAMP, false, kMBNNarrow>
        <<<grid, (kMBM / 4) * (kMBNNarrow / 4), 0, s>>>(rows, m, cols, n, 1, lam, X, k, ldx, nullptr,
                                                        0, Y, ldy, 1, gate);
    return cudaGetLastError();
  }
  dim3 grid((unsigned)ceil_div(m, kMBM), (unsigned)ceil_div(k, kMBN));
  multi_matvec_kernel<float, DP, CLAMP, false><<<grid, kMThreads, 0, s>>>(
      rows, m, cols, n, 1, lam, X, k, ldx, nullptr, 0, Y, ldy, 1, gate);
  return cudaGetLastError();
}

template <int DP, bool CLAMP>
cudaError_t launch_multi_f64_t(const double* rows, int64_t m, const double* cols, int64_t n,
                               double lam, const double* X, int k, int64_t ldx, const double* B,
                               int64_t ldb, double* Y, int64_t ldy, cudaStream_t s,
                               const int* gate) {
  if (k <= kMBNNarrow && multi_narrow_enabled()) {
    dim3 grid((unsigned)ceil_div(m, kMBM), 1);
    constexpr int T = (kMBM / 4) * (kMBNNarrow / 4);
    if (B)
      multi_matvec_kernel<double, DP, CLAMP, true, kMBNNarrow><<<grid, T, 0, s>>>(
          rows, m, cols, n, 0, lam, X, k, ldx, B, ldb, Y, ldy, 0, gate);
    else
      multi_matvec_kernel<double, DP, CLAMP, false, kMBNNarrow><<<grid, T, 0, s>>>(
          rows, m, cols, n, 0, lam, X, k, ldx, nullptr, 0, Y, ldy, 0, gate);
    return cudaGetLastError();
  }
  dim3 grid((unsigned)ceil_div(m, kMBM), (unsigned)ceil_div(k, kMBN));
  if (B)
    multi_matvec_kernel<double, DP, CLAMP, true><<<grid, kMThreads, 0, s>>>(
        rows, m, cols, n, 0, lam, X, k, ldx, B, ldb, Y, ldy, 0, gate);
  else
    multi_matvec_kernel<double, DP, CLAMP, false><<<grid, kMThreads, 0, s>>>(
        rows, m, cols, n, 0, lam, X, k, ldx, nullptr, 0, Y, ldy, 0, gate);
  return cudaGetLastError();
}

// Dispatch on the padded embedding dimension (2, 4, ..., 16) and the clamp.
#define LAKER_DISPATCH_DP(dp, CALL)                     \
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

__global__ void finish_f32_kernel(const double* __restrict__ part, int S, int64_t m, float lam,
                                  const float* __restrict__ x, int64_t ldx, float* __restrict__ y,
                                  int64_t ldy, int square, const int* status) {
  const bool failed = status_failed(status);
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < m;
       i += (int64_t)gridDim.x * blockDim.x) {
    double acc = square ? (double)lam * (double)x[i * ldx] : 0.0;
    for (int s = 0; s < S; ++s) acc += part[(int64_t)s * m + i];
    y[i * ldy] = failed ? nan_f32() : (float)acc;
  }
}

__global__ void poison_on_status_kernel(const int* __restrict__ status, float* __restrict__ Y,
                                        int64_t m, int k, int64_t ldy) {
  if (!status_failed(status)) return;
  const int64_t total = m * (int64_t)k;
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < total;
       t += (int64_t)gridDim.x * blockDim.x)
    Y[(t / k) * ldy + t % k] = nan_f32();
}

}  // namespace

SegPlan k1_plan(int64_t m, int64_t n, int d) {
  const int dp = padded_dim(d);
  const int cfg = k1_variant(dp);
  const K1Variant v = kK1Variants[cfg];
  SegPlan p = plan_segments(m, n, v.rows * v.threads, k1_occupancy(cfg, dp), kTileCols32);
  p.cfg = cfg;
  return p;
}

cudaError_t launch_k1(const float* rows32, int64_t m, const float* cols32, int64_t n, int d,
                      int clamp, const float* x, double* part, const SegPlan& plan, int* status,
                      const int* gate, cudaStream_t s) {
  const int dp = padded_dim(d);
  if (clamp) {
    LAKER_DISPATCH_DP(dp, return (launch_k1_t<DPv, true>(rows32, m, cols32, n, x, part, plan, status, gate, s)));
  } else {
    LAKER_DISPATCH_DP(dp, return (launch_k1_t<DPv, false>(rows32, m, cols32, n, x, part, plan, status, gate, s)));
  }
  return cudaErrorInvalidValue;
}

cudaError_t launch_multi_f32(const float* rows32, int64_t m, const float* cols32, int64_t n, int d,
                             float lam, int clamp, const float* X, int k, int64_t ldx, float* Y,
                             int64_t ldy, cudaStream_t s, const int* gate) {
  if (ceil_div(k, kMBN) > 65535) return cudaErrorInvalidValue;
  const int dp = padded_dim(d);
  if (clamp) {
    LAKER_DISPATCH_DP(dp, return (launch_multi_f32_t<DPv, true>(rows32, m, cols32, n, lam, X, k, ldx, Y, ldy, s, gate)));
  } else {
    LAKER_DISPATCH_DP(dp, return (launch_multi_f32_t<DPv, false>(rows32, m, cols32, n, lam, X, k, ldx, Y, ldy, s, gate)));
  }
  return cudaErrorInvalidValue;
}

cudaError_t launch_multi_f64(const double* rows64, int64_t m, const double* cols64, int64_t n, int d,
                             double lam, int clamp, const double* X, int k, int64_t ldx,
                             const double* B, int64_t ldb, double* Y, int64_t ldy, cudaStream_t s,
                             const int* gate) {
  if (ceil_div(k, kMBN) > 65535) return cudaErrorInvalidValue;
  const int dp = padded_dim(d);
  if (clamp) {
    LAKER_DISPATCH_DP(dp, return (launch_multi_f64_t<DPv, true>(rows64, m, cols64, n, lam, X, k, ldx, B, ldb, Y, ldy, s, gate)));
  } else {
    LAKER_DISPATCH_DP(dp, return (launch_multi_f64_t<DPv, false>(rows64, m, cols64, n, lam, X, k, ldx, B, ldb, Y, ldy, s, gate)));
  }
  return cudaErrorInvalidValue;
}

cudaError_t set_wait_limit_f32(unsigned long long ns) { return set_wait_limit_this_unit(ns); }

cudaError_t launch_poison_on_status(const int* status, float* Y, int64_t m, int k, int64_t ldy,
                                    cudaStream_t s) {
  if (m <= 0 || k <= 0) return cudaSuccess;
  int g = (int)ceil_div(m * (int64_t)k, 256);
  if (g > sm_count() * 4) g = sm_count() * 4;
  poison_on_status_kernel<<<g, 256, 0, s>>>(status, Y, m, k, ldy);
  return cudaGetLastError();
}

}  // namespace laker

using namespace laker;

extern "C" size_t laker_matvec_workspace_bytes(int64_t m, int64_t n, int d, int k, int precision) {
  if (m < 0 || n < 0 || d < 1 || d > 16 || k < 1) return 0;
  if (k > 1) {
    // the tensor-core paths stage X as split, swizzled TF32 tiles (and the
    // flash-style kernel the split-FP16 operand images of the points)
    size_t b = k2_use_tensor_cores() && n > 0 ? (size_t)round_up((int64_t)k2_image_bytes(m, n, k), 256) : 0;
    const size_t f = n > 0 && m > 0 ? k2f_workspace_bytes(m, n, k, false) : 0;
    return kWsHeader + (b > f ? b : f);
  }
  const SegPlan p = precision == 64 ? k4_plan(m, n, d) : k1_plan(m, n, d);
  size_t bytes = (size_t)p.S * (size_t)m * sizeof(double);
  if (m == n && n > 0) {
    // a square product with the same embeddings may take the symmetric kernel
    size_t sym = precision == 64 ? sym_partial_bytes<double>(k4s_plan(n, d))
                                 : sym_partial_bytes<float>(k1s_plan(n, d));
    if (precision != 64 && k1t_enabled(d))  // + the tensor-core kernel's operand image
      sym = (size_t)round_up((int64_t)sym, 1024) + k1t_image_bytes(n);
    if (sym > bytes) bytes = sym;
  }
  return kWsHeader + bytes;
}

extern "C" int laker_attn_matvec_f32(const float* rows32, int64_t m, const float* cols32, int64_t n,
                                     int d, float lam, int clamp, const float* X, int k,
                                     int64_t ldx, float* Y, int64_t ldy, void* workspace,
                                     size_t workspace_bytes, void* stream) {
  if (m < 0 || n < 0 || d < 1 || d > 16 || k < 1 || ldx < k || ldy < k) return LAKER_ERR_INVALID_ARG;
  if (m == 0) return LAKER_OK;
  if (!rows32 || !cols32 || !Y || !workspace || (n > 0 && !X) || (m == n && !X))
    return LAKER_ERR_INVALID_ARG;
  if (workspace_bytes < laker_matvec_workspace_bytes(m, n, d, k, 32)) return LAKER_ERR_WORKSPACE;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  WsHeader* hdr = static_cast<WsHeader*>(workspace);
  cudaError_t e = cudaMemsetAsync(&hdr->status, 0, sizeof(int), s);
  if (e != cudaSuccess) return fail_cuda(e);
  if (k > 1) {
    if (n > 0 && k2f_enabled(k, clamp)) {
      uint8_t* img = reinterpret_cast<uint8_t*>(workspace) + kWsHeader;
      e = launch_k2f(rows32, m, cols32, n, d, (m == n) ? lam : 0.0f, X, ldx, k, Y, ldy, img,
                     &hdr->status, s);
      if (e == cudaSuccess) e = launch_poison_on_status(&hdr->status, Y, m, k, ldy, s);
    } else if (k2_use_tensor_cores() && n > 0) {
      uint8_t* img = reinterpret_cast<uint8_t*>(workspace) + kWsHeader;
      e = launch_k2(rows32, m, cols32, n, d, clamp, (m == n) ? lam : 0.0f, X, ldx, k, Y, ldy, img,
                    &hdr->status, s);
      if (e == cudaSuccess) e = launch_poison_on_status(&hdr->status, Y, m, k, ldy, s);
    } else {
      e = launch_multi_f32(rows32, m, cols32, n, d, (m == n) ? lam : 0.0f, clamp, X, k, ldx, Y, ldy, s);
    }
    return e == cudaSuccess ? LAKER_OK : fail_cuda(e);
  }
  // Single RHS: strided x is staged element-wise; a contiguous copy is not needed.
  if (ldx != 1) return LAKER_ERR_UNSUPPORTED;
  char* wbase = static_cast<char*>(workspace) + kWsHeader;
  if (rows32 == cols32 && m == n && k1_symmetric_for(n)) {
    // the operator itself: every off-diagonal entry evaluated once
    const bool tc = k1t_enabled(d);
    const SymPlan sp = tc ? k1t_plan(n) : k1s_plan(n, d);
    double* rowpart = reinterpret_cast<double*>(wbase);
    float* colpart = sym_colpart_ptr<float>(wbase, sp);
    if (tc) {
      uint8_t* img = reinterpret_cast<uint8_t*>(wbase) + round_up((int64_t)sym_partial_bytes<float>(sp), 1024);
      const int fmt = k1t_format(clamp, d);
      e = launch_k1t_pack(cols32, n, d, img, sp.nb * sym_block_points(), s, fmt);
      if (e == cudaSuccess)
        e = launch_k1t(img, n, clamp, X, rowpart, colpart, sp, &hdr->status, nullptr, s, fmt);
    } else {
      e = launch_k1s(cols32, n, d, clamp, X, rowpart, colpart, sp, &hdr->status, nullptr, s);
    }
    if (e == cudaSuccess)
      e = launch_sym_finish(sp, rowpart, colpart, n, lam, X, Y, ldy, &hdr->status, s);
    return e == cudaSuccess ? LAKER_OK : fail_cuda(e);
  }
  const SegPlan plan = k1_plan(m, n, d);
  double* part = reinterpret_cast<double*>(wbase);
  if (n > 0) {
    e = launch_k1(rows32, m, cols32, n, d, clamp, X, part, plan, &hdr->status, nullptr, s);
    if (e != cudaSuccess) return fail_cuda(e);
  }
  const int S = n > 0 ? plan.S : 0;
  int g = (int)ceil_div(m, 256);
  if (g > sm_count() * 8) g = sm_count() * 8;
  finish_f32_kernel<<<g, 256, 0, s>>>(part, S, m, lam, X, ldx, Y, ldy, (m == n) ? 1 : 0,
                                      &hdr->status);
  e = cudaGetLastError();
  return e == cudaSuccess ? LAKER_OK : fail_cuda(e);
}
