// FP64 fused attention-kernel matvec / residual (the accurate operator).
//
// Same tiling as the FP32 kernel: a CTA owns T*R rows and one column
// segment, column embeddings (packed64 rows) are staged by double-buffered
// TMA bulk copies, x by plain loads.  Logits, exp and accumulation are FP64,
// so the result carries the float64 reference operator's accuracy: the PCG
// loop uses it to recompute the true residual b - A x, and float64 operators
// and predictions use it directly.
#include "sym.cuh"

namespace laker {
namespace {

constexpr int kK4Threads = 256;
constexpr int kK4Rows = 2;

template <int DP, int R, int T, bool CLAMP>
__global__ void __launch_bounds__(T, 2)
    k4_matvec_f64(const double* __restrict__ rows, int64_t m, const double* __restrict__ cols,
                  int64_t n, const double* __restrict__ x, double* __restrict__ part,
                  int64_t cols_per_seg, int* status, const int* gate) {
  if (gate && *gate == 0) return;
  constexpr int TC = kTileCols64;
  constexpr int TILE = TC * DP;
  __shared__ __align__(128) double sE[2][TILE];
  __shared__ __align__(16) double sX[2][TC];
  __shared__ double sExp[64];
  __shared__ __align__(8) uint64_t bar[2];

  const int tid = threadIdx.x;
  const int64_t row0 = (int64_t)blockIdx.x * (T * R);
  const int64_t c_begin = (int64_t)blockIdx.y * cols_per_seg;
  const int64_t c_end = min(n, c_begin + cols_per_seg);
  const int ntiles = c_begin < c_end ? (int)ceil_div(c_end - c_begin, TC) : 0;

  double ev[R][DP];
#pragma unroll
  for (int r = 0; r < R; ++r) {
    const int64_t i = row0 + r * T + tid;
#pragma unroll
    for (int k = 0; k < DP; ++k) ev[r][k] = (i < m) ? rows[i * DP + k] : 0.0;
  }
  double acc[R];
#pragma unroll
  for (int r = 0; r < R; ++r) acc[r] = 0.0;

  if (tid == 0) {
    mbar_init(&bar[0], 1);
    mbar_init(&bar[1], 1);
    mbar_fence_init();
  }
  exp_table_to_shared(sExp, tid, T);
  __syncthreads();

  auto issue = [&](int t, int b) {
    const int64_t c0 = c_begin + (int64_t)t * TC;
    mbar_arrive_expect_tx(&bar[b], TILE * 8);
    bulk_g2s(sE[b], cols + c0 * DP, TILE * 8, &bar[b]);
  };
  auto load_x = [&](int t, int b) {
    const int64_t c0 = c_begin + (int64_t)t * TC;
    for (int j = tid; j < TC; j += T) {
      const int64_t c = c0 + j;
      sX[b][j] = (c < c_end) ? x[c] : 0.0;
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
    const double* E = sE[b];
#pragma unroll 2
    for (int j = 0; j < TC; ++j) {
      const double2* cp = reinterpret_cast<const double2*>(E + j * DP);
      double c[DP];
#pragma unroll
      for (int h = 0; h < DP / 2; ++h) {
        const double2 v = cp[h];
        c[2 * h] = v.x;
        c[2 * h + 1] = v.y;
      }
      const double xj = sX[b][j];
#pragma unroll
      for (int r = 0; r < R; ++r) {
        double s = ev[r][0] * c[0];
#pragma unroll
        for (int k = 1; k < DP; ++k) s = fma(ev[r][k], c[k], s);
        if (CLAMP) s = fmin(s, kClamp64);
        acc[r] = fma(exp_tab(s, sExp), xj, acc[r]);
      }
    }
    __syncthreads();
  }

  if (consumed < ntiles) {
    for (int t = consumed; t < issued; ++t) mbar_wait_drain(&bar[t & 1], (t >> 1) & 1, status);
    return;
  }
#pragma unroll
  for (int r = 0; r < R; ++r) {
    const int64_t i = row0 + r * T + tid;
    if (i < m) part[(int64_t)blockIdx.y * m + i] = acc[r];
  }
}

template <int DP, bool CLAMP>
cudaError_t launch_k4_t(const double* rows, int64_t m, const double* cols, int64_t n,
                        const double* x, double* part, const SegPlan& p, int* status,
                        const int* gate, cudaStream_t s) {
  dim3 grid((unsigned)ceil_div(m, kK4Threads * kK4Rows), (unsigned)p.S);
  k4_matvec_f64<DP, kK4Rows, kK4Threads, CLAMP>
      <<<grid, kK4Threads, 0, s>>>(rows, m, cols, n, x, part, p.cols_per_seg, status, gate);
  return cudaGetLastError();
}

#define LAKER_DISPATCH_DP64(dp, CALL)                   \
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

__global__ void finish_f64_kernel(const double* __restrict__ part, int S, int64_t m, double lam,
                                  const double* __restrict__ x, int64_t ldx,
                                  const double* __restrict__ b, int64_t ldb,
                                  double* __restrict__ y, int64_t ldy, int square,
                                  const int* status) {
  const bool failed = status_failed(status);
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < m;
       i += (int64_t)gridDim.x * blockDim.x) {
    double acc = square ? lam * x[i * ldx] : 0.0;
    for (int s = 0; s < S; ++s) acc += part[(int64_t)s * m + i];
    y[i * ldy] = failed ? nan_f64() : (b ? b[i * ldb] - acc : acc);
  }
}

}  // namespace

// Resident CTAs per SM of the FP64 kernel (occupancy API; 2 when unavailable).
int k4_occupancy(int dp) {
  static int cache[9] = {};
  if (dp < 2 || dp > 16) return 2;
  int& c = cache[dp / 2];
  if (c > 0) return c;
  const void* fn = nullptr;
#define LAKER_K4_FN(DPv) \
  if (dp == DPv) fn = reinterpret_cast<const void*>(&k4_matvec_f64<DPv, kK4Rows, kK4Threads, false>);
  LAKER_K4_FN(2) LAKER_K4_FN(4) LAKER_K4_FN(6) LAKER_K4_FN(8) LAKER_K4_FN(10) LAKER_K4_FN(12)
  LAKER_K4_FN(14) LAKER_K4_FN(16)
#undef LAKER_K4_FN
  int nb = 0;
  if (!fn || cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, fn, kK4Threads, 0) != cudaSuccess ||
      nb < 1) {
    cudaGetLastError();
    nb = 2;
  }
  c = nb;
  return c;
}

SegPlan k4_plan(int64_t m, int64_t n, int d) {
  return plan_segments(m, n, kK4Threads * kK4Rows, k4_occupancy(padded_dim(d)), kTileCols64);
}

cudaError_t launch_k4(const double* rows64, int64_t m, const double* cols64, int64_t n, int d,
                      int clamp, const double* x, double* part, const SegPlan& plan, int* status,
                      const int* gate, cudaStream_t s) {
  const int dp = padded_dim(d);
  if (clamp) {
    LAKER_DISPATCH_DP64(dp, return (launch_k4_t<DPv, true>(rows64, m, cols64, n, x, part, plan, status, gate, s)));
  } else {
    LAKER_DISPATCH_DP64(dp, return (launch_k4_t<DPv, false>(rows64, m, cols64, n, x, part, plan, status, gate, s)));
  }
  return cudaErrorInvalidValue;
}

cudaError_t set_wait_limit_f64(unsigned long long ns) { return set_wait_limit_this_unit(ns); }

}  // namespace laker

using namespace laker;

extern "C" int laker_attn_matvec_f64(const double* rows64, int64_t m, const double* cols64,
                                     int64_t n, int d, double lam, int clamp, const double* X,
                                     int k, int64_t ldx, const double* B, int64_t ldb, double* Y,
                                     int64_t ldy, void* workspace, size_t workspace_bytes,
                                     void* stream) {
  if (m < 0 || n < 0 || d < 1 || d > 16 || k < 1 || ldx < k || ldy < k || (B && ldb < k))
    return LAKER_ERR_INVALID_ARG;
  if (m == 0) return LAKER_OK;
  if (!rows64 || !cols64 || !Y || !workspace || (n > 0 && !X) || (m == n && !X))
    return LAKER_ERR_INVALID_ARG;
  if (workspace_bytes < laker_matvec_workspace_bytes(m, n, d, k, 64)) return LAKER_ERR_WORKSPACE;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  WsHeader* hdr = static_cast<WsHeader*>(workspace);
  cudaError_t e = cudaMemsetAsync(&hdr->status, 0, sizeof(int), s);
  if (e != cudaSuccess) return fail_cuda(e);
  if (k > 1) {
    e = launch_multi_f64(rows64, m, cols64, n, d, (m == n) ? lam : 0.0, clamp, X, k, ldx, B, ldb,
                         Y, ldy, s);
    return e == cudaSuccess ? LAKER_OK : fail_cuda(e);
  }
  char* wbase = static_cast<char*>(workspace) + kWsHeader;
  if (rows64 == cols64 && m == n && ldx == 1 && k4_use_symmetric()) {
    // the operator itself: every off-diagonal entry evaluated once
    const SymPlan sp = k4s_plan(n, d);
    double* rowpart = reinterpret_cast<double*>(wbase);
    double* colpart = sym_colpart_ptr<double>(wbase, sp);
    e = launch_k4s(rows64, n, d, clamp, X, rowpart, colpart, sp, &hdr->status, nullptr, s);
    if (e == cudaSuccess)
      e = launch_sym_finish64(sp, rowpart, colpart, n, lam, X, B, ldb, Y, ldy, &hdr->status, s);
    return e == cudaSuccess ? LAKER_OK : fail_cuda(e);
  }
  const SegPlan plan = k4_plan(m, n, d);
  double* part = reinterpret_cast<double*>(wbase);
  if (n > 0) {
    if (ldx != 1) return LAKER_ERR_UNSUPPORTED;
    e = launch_k4(rows64, m, cols64, n, d, clamp, X, part, plan, &hdr->status, nullptr, s);
    if (e != cudaSuccess) return fail_cuda(e);
  }
  int g = (int)ceil_div(m, 256);
  if (g > sm_count() * 8) g = sm_count() * 8;
  finish_f64_kernel<<<g, 256, 0, s>>>(part, n > 0 ? plan.S : 0, m, lam, X, ldx, B, ldb, Y, ldy,
                                      (m == n) ? 1 : 0, &hdr->status);
  e = cudaGetLastError();
  return e == cudaSuccess ? LAKER_OK : fail_cuda(e);
}
