// Embedding packing, operator diagonal, materialised kernel blocks and the
// predictive-variance epilogue.
#include "internal.cuh"

namespace laker {
namespace {

template <typename Tin>
__global__ void pack32_kernel(const Tin* __restrict__ E, int64_t n, int d, int64_t ld, int dp,
                              int64_t npairs, float* __restrict__ out) {
  const int64_t total = npairs * dp * 2;
  for (int64_t o = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; o < total;
       o += (int64_t)gridDim.x * blockDim.x) {
    const int64_t q = o / (dp * 2);
    const int rem = (int)(o - q * dp * 2);
    const int k = rem >> 1, s = rem & 1;
    const int64_t i = 2 * q + s;
    out[o] = (i < n && k < d) ? static_cast<float>(E[i * ld + k]) : 0.0f;
  }
}

template <typename Tin>
__global__ void pack64_kernel(const Tin* __restrict__ E, int64_t n, int d, int64_t ld, int dp,
                              int64_t rows, double* __restrict__ out) {
  const int64_t total = rows * dp;
  for (int64_t o = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; o < total;
       o += (int64_t)gridDim.x * blockDim.x) {
    const int64_t i = o / dp;
    const int k = (int)(o - i * dp);
    out[o] = (i < n && k < d) ? static_cast<double>(E[i * ld + k]) : 0.0;
  }
}

__global__ void diagonal_kernel(const double* __restrict__ e64, int64_t n, int dp, double lam,
                                double* __restrict__ out) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x) {
    double s = 0.0;
    for (int k = 0; k < dp; ++k) s = fma(e64[i * dp + k], e64[i * dp + k], s);
    out[i] = lam + exp(s);
  }
}

// exp(Er Ec^T) for a 32 x 32 output tile per 256-thread block; each thread
// produces 4 rows of one column.  Logits in FP64.
template <typename Tout>
__global__ void kernel_eval_kernel(const double* __restrict__ r64, int64_t m,
                                   const double* __restrict__ c64, int64_t p, int dp, int clamp,
                                   Tout* __restrict__ out, int64_t ldo) {
  __shared__ double sr[32][17];
  __shared__ double sc[32][17];
  const int tx = threadIdx.x & 31, ty = threadIdx.x >> 5;
  const int64_t i0 = (int64_t)blockIdx.y * 32, j0 = (int64_t)blockIdx.x * 32;
  for (int o = threadIdx.x; o < 32 * dp; o += blockDim.x) {
    const int a = o / dp, k = o - a * dp;
    sr[a][k] = (i0 + a < m) ? r64[(i0 + a) * dp + k] : 0.0;
    sc[a][k] = (j0 + a < p) ? c64[(j0 + a) * dp + k] : 0.0;
  }
  __syncthreads();
  const double cl = sizeof(Tout) == 8 ? kClamp64 : 80.0;
  const int64_t j = j0 + tx;
#pragma unroll
  for (int q = 0; q < 4; ++q) {
    const int a = ty * 4 + q;
    const int64_t i = i0 + a;
    double s = 0.0;
    for (int k = 0; k < dp; ++k) s = fma(sr[a][k], sc[tx][k], s);
    if (clamp) s = fmin(s, cl);
    if (i < m && j < p) out[i * ldo + j] = static_cast<Tout>(exp(s));
  }
}

// var_q = max(0, exp(||e_q||^2) - sum_i K[i,q] V[i,q]); one block of 32 x 32
// threads per 32 query columns, fixed-order reduction.
__global__ void variance_kernel(const double* __restrict__ q64, int64_t m, int dp,
                                const double* __restrict__ K, const double* __restrict__ V,
                                int64_t n, int64_t ld, double* __restrict__ var) {
  __shared__ double red[32][33];
  const int tx = threadIdx.x & 31, ty = threadIdx.x >> 5;
  const int64_t q = (int64_t)blockIdx.x * 32 + tx;
  double s = 0.0;
  if (q < m) {
    for (int64_t i = ty; i < n; i += 32) s = fma(K[i * ld + q], V[i * ld + q], s);
  }
  red[ty][tx] = s;
  __syncthreads();
  if (ty == 0 && q < m) {
    double t = 0.0;
    for (int r = 0; r < 32; ++r) t += red[r][tx];
    double nn = 0.0;
    for (int k = 0; k < dp; ++k) nn = fma(q64[q * dp + k], q64[q * dp + k], nn);
    const double v = exp(nn) - t;
    var[q] = v > 0.0 ? v : 0.0;
  }
}

inline int grid_for(int64_t work, int threads) {
  int64_t g = ceil_div(work, threads);
  const int64_t cap = (int64_t)sm_count() * 16;
  if (g > cap) g = cap;
  return (int)(g < 1 ? 1 : g);
}

}  // namespace
}  // namespace laker

using namespace laker;

extern "C" size_t laker_packed32_floats(int64_t n, int d) {
  if (n < 0 || d < 1 || d > 16) return 0;
  return (size_t)packed_pairs(n) * padded_dim(d) * 2;
}

extern "C" size_t laker_packed64_doubles(int64_t n, int d) {
  if (n < 0 || d < 1 || d > 16) return 0;
  return (size_t)packed_rows64(n) * padded_dim(d);
}

extern "C" int laker_pack_f32(const void* E, int e_is_f64, int64_t n, int d, int64_t ld,
                              float* packed32, void* stream) {
  if (!packed32 || n < 0 || d < 1 || d > 16 || ld < d || (n > 0 && !E)) return LAKER_ERR_INVALID_ARG;
  const int dp = padded_dim(d);
  const int64_t np = packed_pairs(n);
  const int g = grid_for(np * dp * 2, 256);
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  if (e_is_f64)
    pack32_kernel<double><<<g, 256, 0, s>>>(static_cast<const double*>(E), n, d, ld, dp, np, packed32);
  else
    pack32_kernel<float><<<g, 256, 0, s>>>(static_cast<const float*>(E), n, d, ld, dp, np, packed32);
  cudaError_t e = cudaGetLastError();
  return e == cudaSuccess ? LAKER_OK : fail_cuda(e);
}

extern "C" int laker_pack_f64(const void* E, int e_is_f64, int64_t n, int d, int64_t ld,
                              double* packed64, void* stream) {
  if (!packed64 || n < 0 || d < 1 || d > 16 || ld < d || (n > 0 && !E)) return LAKER_ERR_INVALID_ARG;
  const int dp = padded_dim(d);
  const int64_t rows = packed_rows64(n);
  const int g = grid_for(rows * dp, 256);
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  if (e_is_f64)
    pack64_kernel<double><<<g, 256, 0, s>>>(static_cast<const double*>(E), n, d, ld, dp, rows, packed64);
  else
    pack64_kernel<float><<<g, 256, 0, s>>>(static_cast<const float*>(E), n, d, ld, dp, rows, packed64);
  cudaError_t e = cudaGetLastError();
  return e == cudaSuccess ? LAKER_OK : fail_cuda(e);
}

extern "C" int laker_attn_diagonal(const double* packed64, int64_t n, int d, double lam, double* out,
                                   void* stream) {
  if (n < 0 || d < 1 || d > 16 || (n > 0 && (!packed64 || !out))) return LAKER_ERR_INVALID_ARG;
  if (n == 0) return LAKER_OK;
  diagonal_kernel<<<grid_for(n, 256), 256, 0, static_cast<cudaStream_t>(stream)>>>(
      packed64, n, padded_dim(d), lam, out);
  cudaError_t e = cudaGetLastError();
  return e == cudaSuccess ? LAKER_OK : fail_cuda(e);
}

extern "C" int laker_kernel_eval(const double* rows64, int64_t m, const double* cols64, int64_t p,
                                 int d, int clamp, void* out, int out_is_f64, int64_t ldo,
                                 void* stream) {
  if (m < 0 || p < 0 || d < 1 || d > 16 || ldo < p) return LAKER_ERR_INVALID_ARG;
  if (m == 0 || p == 0) return LAKER_OK;
  if (!rows64 || !cols64 || !out) return LAKER_ERR_INVALID_ARG;
  dim3 grid((unsigned)ceil_div(p, 32), (unsigned)ceil_div(m, 32));
  if (grid.y > 65535u) return LAKER_ERR_UNSUPPORTED;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  if (out_is_f64)
    kernel_eval_kernel<double><<<grid, 256, 0, s>>>(rows64, m, cols64, p, padded_dim(d), clamp,
                                                    static_cast<double*>(out), ldo);
  else
    kernel_eval_kernel<float><<<grid, 256, 0, s>>>(rows64, m, cols64, p, padded_dim(d), clamp,
                                                   static_cast<float*>(out), ldo);
  cudaError_t e = cudaGetLastError();
  return e == cudaSuccess ? LAKER_OK : fail_cuda(e);
}

extern "C" int laker_variance_finalize(const double* q64, int64_t m, int d, const double* Kxq,
                                       const double* V, int64_t n, int64_t ld, double* var,
                                       void* stream) {
  if (m < 0 || n < 0 || d < 1 || d > 16 || ld < m) return LAKER_ERR_INVALID_ARG;
  if (m == 0) return LAKER_OK;
  if (!q64 || !var || (n > 0 && (!Kxq || !V))) return LAKER_ERR_INVALID_ARG;
  variance_kernel<<<(unsigned)ceil_div(m, 32), 1024, 0, static_cast<cudaStream_t>(stream)>>>(
      q64, m, padded_dim(d), Kxq, V, n, ld, var);
  cudaError_t e = cudaGetLastError();
  return e == cudaSuccess ? LAKER_OK : fail_cuda(e);
}
