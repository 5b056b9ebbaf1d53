// Host-side launchers shared between the translation units of liblaker_b200.
#pragma once

#include "common.cuh"

namespace laker {

// Every caller-provided workspace starts with this header; `status` receives
// device-side failures (LAKER_ERR_TIMEOUT) of the kernels launched with it.
struct alignas(256) WsHeader {
  int status;
  int pad[63];
};
constexpr size_t kWsHeader = sizeof(WsHeader);

// Records a CUDA failure for laker_last_cuda_error() and returns LAKER_ERR_CUDA.
int fail_cuda(cudaError_t e);

// Streaming multiprocessor count of the current device (cached per device).
int sm_count();

// Split of the column range into S segments of cols_per_seg columns (a
// multiple of the staging tile) so that row blocks x segments fill whole
// waves of CTAs.
struct SegPlan {
  int S;
  int64_t cols_per_seg;
  int cfg = 0;  // kernel variant (rows per thread / threads per CTA)
};
SegPlan plan_segments(int64_t m, int64_t n, int rows_per_cta, int ctas_per_sm, int tile);

// ---- single-RHS fused matvecs: write per-segment FP64 row partials --------
// part[s * m + i] = sum_{j in segment s} exp(er_i . ec_j) x_j
SegPlan k1_plan(int64_t m, int64_t n, int d);
cudaError_t launch_k1(const float* rows32, int64_t m, const float* cols32, int64_t n, int d,
                      int clamp, const float* x, double* part, const SegPlan& plan, int* status,
                      const int* gate, cudaStream_t s);

SegPlan k4_plan(int64_t m, int64_t n, int d);
cudaError_t launch_k4(const double* rows64, int64_t m, const double* cols64, int64_t n, int d,
                      int clamp, const double* x, double* part, const SegPlan& plan, int* status,
                      const int* gate, cudaStream_t s);

// `gate` (nullable): the kernel does nothing when *gate == 0.

// ---- multi-RHS fused matvecs (CUDA cores) ----------------------------------
// Y[i, :] = lam * X[i, :] (if m == n) + sum_j exp(er_i . ec_j) X[j, :]
cudaError_t launch_multi_f32(const float* rows32, int64_t m, const float* cols32, int64_t n, int d,
                             float lam, int clamp, const float* X, int k, int64_t ldx, float* Y,
                             int64_t ldy, cudaStream_t s, const int* gate = nullptr);
// Y = B - (lam X + K X) when B != nullptr, else lam X + K X (FP64 throughout).
cudaError_t launch_multi_f64(const double* rows64, int64_t m, const double* cols64, int64_t n, int d,
                             double lam, int clamp, const double* X, int k, int64_t ldx,
                             const double* B, int64_t ldb, double* Y, int64_t ldy, cudaStream_t s,
                             const int* gate = nullptr);

// Tensor-core (tcgen05, split TF32) multi-RHS FP32 matvec (matvec_tc.cu).
int k2_chunk_cols(int k);
size_t k2_image_bytes(int64_t m, int64_t n, int k);
bool k2_use_tensor_cores();
cudaError_t launch_k2(const float* rows32, int64_t m, const float* cols32, int64_t n, int d,
                      int clamp, float lam, const float* X, int64_t ldx, int k, float* Y,
                      int64_t ldy, uint8_t* img, int* status, cudaStream_t s,
                      const int* gate = nullptr);

// Split, swizzled TF32 image of X (n x k) in 32-point tiles of N right-hand
// sides (the multi-RHS kernels' B operand): chunk c, tile t at
// (c * ntiles + t) * N * 256 bytes, [hi: N rows x 128 B][lo: N rows x 128 B]
// in the 128-byte-swizzled K-major layout; points past n are zero.
cudaError_t launch_pack_x32(const float* X, int64_t n, int64_t ldx, int k, int N, int64_t ntiles,
                            uint8_t* img, const int* gate, cudaStream_t s);
// Y = lam X + sum over `segs` segment partials (segs x m x k floats), in
// segment order.
cudaError_t launch_seg_reduce(const float* part, int segs, int64_t m, int k, float lam,
                              const float* X, int64_t ldx, float* Y, int64_t ldy, const int* gate,
                              cudaStream_t s);

// ---- flash-style multi-RHS FP32 matvec (matvec_flash.cu) --------------------
// Whether a product of k right-hand sides takes it (unclamped operators, k up
// to LAKER_VARIANT_MULTI_FLASH_K), and its workspace.
bool k2f_enabled(int k, int clamp);
size_t k2f_workspace_bytes(int64_t m, int64_t n, int k, bool same_points);
cudaError_t launch_k2f(const float* rows32, int64_t m, const float* cols32, int64_t n, int d,
                       float lam, const float* X, int64_t ldx, int k, float* Y, int64_t ldy,
                       uint8_t* ws, int* status, cudaStream_t s, const int* gate = nullptr);

// ---- multi-RHS solve and preconditioner apply (pcg_multi.cu) ----------------
size_t pcg_multi_workspace_bytes(int64_t n, int d, int nr, int k);
int pcg_solve_multi(const laker_operator* op, const laker_precond* pc, const double* B, int k,
                    double* X, const laker_pcg_params* prm, void* workspace, laker_pcg_result* res,
                    cudaStream_t s);
// Scratch of one multi-RHS apply Z = c^-1/2 R + Q W Q^T R (R, Z: n x k).
size_t precond_multi_scratch_bytes(int64_t n, int nr, int k);
template <typename ZT>
cudaError_t launch_precond_multi(const laker_precond* pc, const double* R, int k, ZT* Z,
                                 void* scratch, const int* gate, cudaStream_t s);

// Current kernel variant choice (variants.cu; LAKER_VARIANT_* in the header).
int variant_get(int which);

// Bounded-wait limit (ns) of the kernels of each translation unit that has
// pipeline waits, on the current device (LAKER_VARIANT_WAIT_LIMIT_US).
cudaError_t set_wait_limit_f32(unsigned long long ns);
cudaError_t set_wait_limit_f64(unsigned long long ns);
cudaError_t set_wait_limit_sym(unsigned long long ns);
cudaError_t set_wait_limit_symtc(unsigned long long ns);
cudaError_t set_wait_limit_tc(unsigned long long ns);
cudaError_t set_wait_limit_flash(unsigned long long ns);

// Y[i, c] = NaN for i < m, c < k when *status != 0: the outputs of a product
// whose kernel recorded a device-side failure (a bounded wait that expired)
// never look like a result.
cudaError_t launch_poison_on_status(const int* status, float* Y, int64_t m, int k, int64_t ldy,
                                    cudaStream_t s);

}  // namespace laker
