// Factored CCCP preconditioner apply: Z = c^-1/2 R + Q W Q^T R.
//
// Two streaming passes over Q (n x ldq, FP32, float4 rows): a projection
// u = Q^T r whose fixed-order FP64 total (and v = W u) is formed by the last
// block, then an expansion z = c^-1/2 r + Q v with one warp per row.
// HBM-bound: 2 * n * ldq * 4 bytes per apply.
#include <cstdint>

#include "pcg_state.cuh"

namespace laker {

int precond_grid() { return 2 * sm_count(); }

// Checks the factor descriptor: 1 <= nr <= ldq <= 1024, ldq % 4 == 0 and a
// 16-byte aligned Q (float4 rows).
bool precond_valid(const laker_precond* pc) {
  return pc && pc->n >= 0 && pc->nr >= 1 && pc->nr <= kMaxNr && pc->ldq >= pc->nr &&
         pc->ldq <= kMaxNr && (pc->ldq % 4) == 0 && pc->q_basis && pc->w_core &&
         (reinterpret_cast<uintptr_t>(pc->q_basis) % 16) == 0;
}

}  // namespace laker

using namespace laker;

extern "C" size_t laker_precond_workspace_bytes(int64_t n, int nr, int k) {
  if (n < 0 || nr < 1 || nr > kMaxNr || k < 1) return 0;
  if (k > 1) return kWsHeader + precond_multi_scratch_bytes(n, nr, k);
  const size_t G = (size_t)precond_grid();
  // header | counters | upart (G x 1024) | v (1024) | blockpart (G)
  return kWsHeader + 256 + round_up((int64_t)(G * kMaxNr * sizeof(double)), 256) +
         round_up((int64_t)(kMaxNr * sizeof(double)), 256) +
         round_up((int64_t)(G * sizeof(double)), 256);
}

extern "C" int laker_precond_apply(const laker_precond* pc, const double* R, int k, int64_t ldr,
                                   void* Z, int z_is_f64, int64_t ldz, void* workspace,
                                   size_t workspace_bytes, void* stream) {
  if (!pc || k < 1 || ldr < k || ldz < k) return LAKER_ERR_INVALID_ARG;
  if (pc->n == 0 && pc->nr >= 1) return LAKER_OK;
  if (!precond_valid(pc) || !R || !Z || !workspace) return LAKER_ERR_INVALID_ARG;
  if (workspace_bytes < laker_precond_workspace_bytes(pc->n, pc->nr, k)) return LAKER_ERR_WORKSPACE;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  if (k > 1) {
    // k right-hand sides: three tiled GEMMs over (n x k) row-major R and Z
    if (ldr != k || ldz != k) return LAKER_ERR_UNSUPPORTED;
    void* scratch = static_cast<char*>(workspace) + kWsHeader;
    const cudaError_t e = z_is_f64
        ? launch_precond_multi<double>(pc, R, k, static_cast<double*>(Z), scratch, nullptr, s)
        : launch_precond_multi<float>(pc, R, k, static_cast<float*>(Z), scratch, nullptr, s);
    return e == cudaSuccess ? LAKER_OK : fail_cuda(e);
  }
  if (ldr != 1 || ldz != 1) return LAKER_ERR_UNSUPPORTED;
  const int G = precond_grid();
  char* base = static_cast<char*>(workspace);
  WsHeader* hdr = reinterpret_cast<WsHeader*>(base);
  unsigned int* counters = reinterpret_cast<unsigned int*>(base + kWsHeader);
  double* upart = reinterpret_cast<double*>(base + kWsHeader + 256);
  double* v = reinterpret_cast<double*>(reinterpret_cast<char*>(upart) +
                                        round_up((int64_t)((size_t)G * kMaxNr * sizeof(double)), 256));
  double* blockpart = reinterpret_cast<double*>(reinterpret_cast<char*>(v) +
                                                round_up((int64_t)(kMaxNr * sizeof(double)), 256));
  cudaError_t e = cudaMemsetAsync(hdr, 0, kWsHeader + 256, s);
  if (e != cudaSuccess) return fail_cuda(e);
  const PcView view{pc->q_basis, pc->w_core, pc->n, pc->nr, pc->ldq, pc->inv_sqrt_iso};
  if (z_is_f64)
    launch_precond_apply<double>(view, G, R, upart, v, static_cast<double*>(Z), blockpart,
                                 counters + 0, counters + 1, nullptr, 0, nullptr, nullptr, s);
  else
    launch_precond_apply<float>(view, G, R, upart, v, static_cast<float*>(Z), blockpart,
                                counters + 0, counters + 1, nullptr, 0, nullptr, nullptr, s);
  e = cudaGetLastError();
  return e == cudaSuccess ? LAKER_OK : fail_cuda(e);
}
