// Factored CCCP preconditioner apply: Z = c^-1/2 R + Q W Q^T R.
//
// Two streaming passes over Q (n x nr, FP32): a projection u = Q^T r with
// per-block FP64 partials whose fixed-order total (and v = W u) is formed by
// the last block, then an expansion z = c^-1/2 r + Q v with one warp per row.
// HBM-bound: 2 * n * nr * 4 bytes per apply.
#include "pcg_state.cuh"

namespace laker {

int precond_grid() { return 2 * sm_count(); }

}  // namespace laker

using namespace laker;

extern "C" size_t laker_precond_workspace_bytes(int64_t n, int nr, int k) {
  if (n < 0 || nr < 1 || nr > kMaxNr || k < 1) return 0;
  const size_t G = (size_t)precond_grid();
  // header | counters | upart (G x nr) | v (nr) | blockpart (G)
  return kWsHeader + 256 + round_up((int64_t)(G * nr * sizeof(double)), 256) +
         round_up((int64_t)(nr * sizeof(double)), 256) + round_up((int64_t)(G * sizeof(double)), 256);
}

extern "C" int laker_precond_apply(const laker_precond* pc, const double* R, int k, int64_t ldr,
                                   void* Z, int z_is_f64, int64_t ldz, void* workspace,
                                   size_t workspace_bytes, void* stream) {
  if (!pc || k < 1 || ldr < k || ldz < k) return LAKER_ERR_INVALID_ARG;
  if (pc->n < 0 || pc->nr < 1 || pc->nr > kMaxNr) return LAKER_ERR_INVALID_ARG;
  if (pc->n == 0) return LAKER_OK;
  if (!pc->q_basis || !pc->w_core || !R || !Z || !workspace) return LAKER_ERR_INVALID_ARG;
  if (k != 1 || ldr != 1 || ldz != 1) return LAKER_ERR_UNSUPPORTED;
  if (workspace_bytes < laker_precond_workspace_bytes(pc->n, pc->nr, k)) return LAKER_ERR_WORKSPACE;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  const int G = precond_grid();
  char* base = static_cast<char*>(workspace);
  WsHeader* hdr = reinterpret_cast<WsHeader*>(base);
  unsigned int* counters = reinterpret_cast<unsigned int*>(base + kWsHeader);
  double* upart = reinterpret_cast<double*>(base + kWsHeader + 256);
  double* v = reinterpret_cast<double*>(reinterpret_cast<char*>(upart) +
                                        round_up((int64_t)((size_t)G * pc->nr * sizeof(double)), 256));
  double* blockpart = reinterpret_cast<double*>(reinterpret_cast<char*>(v) +
                                                round_up((int64_t)(pc->nr * sizeof(double)), 256));
  cudaError_t e = cudaMemsetAsync(hdr, 0, kWsHeader + 256, s);
  if (e != cudaSuccess) return fail_cuda(e);
  const PcView view{pc->q_basis, pc->w_core, pc->n, pc->nr, pc->inv_sqrt_iso};
  pc_project_kernel<kVecThreads><<<G, kVecThreads, 0, s>>>(view, R, upart, v, counters + 0, nullptr);
  if (z_is_f64)
    pc_expand_kernel<kVecThreads, double><<<G, kVecThreads, 0, s>>>(
        view, R, v, static_cast<double*>(Z), blockpart, counters + 1, nullptr, 0, nullptr, nullptr);
  else
    pc_expand_kernel<kVecThreads, float><<<G, kVecThreads, 0, s>>>(
        view, R, v, static_cast<float*>(Z), blockpart, counters + 1, nullptr, 0, nullptr, nullptr);
  e = cudaGetLastError();
  return e == cudaSuccess ? LAKER_OK : fail_cuda(e);
}
