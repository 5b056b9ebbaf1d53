// Device-resident state of one PCG solve and the single-RHS kernels that the
// preconditioner apply and the PCG loop share.
#pragma once

#include "internal.cuh"

namespace laker {

// Scalars of the mixed-precision PCG recurrence.  Lives in the caller's
// workspace; only the last block of each reduction writes it.
struct alignas(256) PcgState {
  double bnorm;       // ||b||
  double tol_abs;     // tol * ||b||
  double rz;          // r . z of the current residual
  double pAp;         // p . A p
  double alpha, beta;
  double rnorm;       // recurrence residual norm (after the last update)
  double rmax;        // residual norm at the last FP64 recomputation
  double true_rnorm;  // ||b - A x|| from the last FP64 recomputation
  double delta;       // reliable-update factor
  double eps;         // breakdown threshold
  double lam;         // lambda
  int iter;           // PCG iterations (FP32 operator applications)
  int n_accurate;     // FP64 residual recomputations
  int max_iter;
  int active;         // 1 while the solve runs (gate of the FP32 matvec)
  int need_update;    // 1 when this iteration ends with an FP64 recomputation
  int done;
  int status;
  int pad;
  unsigned int counters[8];
};

// Counter slots used by the last-block reductions.
enum { kCtrBnorm = 0, kCtrMatvec, kCtrUpdate, kCtrResid, kCtrProject, kCtrExpand };

constexpr int kMaxNr = 1024;  // largest probe count of the fused apply
constexpr int kVecThreads = 256;

struct PcView {
  const float* Q;  // (n x nr) row-major
  const float* W;  // (nr x nr) symmetric
  int64_t n;
  int nr;
  double cis;  // c^-1/2
};

// u = Q^T r (per-block FP64 partials, fixed-order total in the last block),
// then v = W u.  One pass over Q; thread t owns columns t, t+T, ...
template <int T>
__global__ void __launch_bounds__(T)
    pc_project_kernel(PcView pc, const double* __restrict__ r, double* __restrict__ upart,
                      double* __restrict__ v, unsigned int* counter, const int* gate) {
  if (gate && *gate == 0) return;
  constexpr int NQ = kMaxNr / T;
  __shared__ double s_r[T];
  __shared__ double s_u[kMaxNr];
  const int tid = threadIdx.x;
  const int nr = pc.nr;
  const int64_t per = ceil_div(pc.n, (int64_t)gridDim.x);
  const int64_t i_begin = (int64_t)blockIdx.x * per;
  const int64_t i_end = min(pc.n, i_begin + per);
  double acc[NQ];
#pragma unroll
  for (int q = 0; q < NQ; ++q) acc[q] = 0.0;
  for (int64_t i0 = i_begin; i0 < i_end; i0 += T) {
    const int cnt = (int)min((int64_t)T, i_end - i0);
    __syncthreads();
    if (tid < cnt) s_r[tid] = r[i0 + tid];
    __syncthreads();
    for (int ii = 0; ii < cnt; ++ii) {
      const double ri = s_r[ii];
      const float* qrow = pc.Q + (i0 + ii) * nr;
#pragma unroll
      for (int q = 0; q < NQ; ++q) {
        const int c = tid + q * T;
        if (c < nr) acc[q] = fma((double)qrow[c], ri, acc[q]);
      }
    }
  }
#pragma unroll
  for (int q = 0; q < NQ; ++q) {
    const int c = tid + q * T;
    if (c < nr) upart[(int64_t)blockIdx.x * nr + c] = acc[q];
  }
  if (!arrive_last_block(counter)) return;
  for (int c = tid; c < nr; c += T) {
    double u = 0.0;
    for (unsigned int b = 0; b < gridDim.x; ++b) u += __ldcg(upart + (int64_t)b * nr + c);
    s_u[c] = u;
  }
  __syncthreads();
  for (int c = tid; c < nr; c += T) {
    double acc2 = 0.0;
    for (int cc = 0; cc < nr; ++cc) acc2 = fma((double)pc.W[(int64_t)cc * nr + c], s_u[cc], acc2);
    v[c] = acc2;
  }
}

// z = c^-1/2 r + Q v (one warp per row) and the fixed-order total of r . z.
// With a PcgState the last block turns r . z into beta (or seeds rz when
// `init`); without one it stores the total in dot_out (if non-null).
template <int T, typename ZT>
__global__ void __launch_bounds__(T)
    pc_expand_kernel(PcView pc, const double* __restrict__ r, const double* __restrict__ v,
                     ZT* __restrict__ z, double* __restrict__ blockpart, unsigned int* counter,
                     PcgState* st, int init, double* dot_out, const int* gate) {
  if (gate && *gate == 0) return;
  __shared__ double s_v[kMaxNr];
  __shared__ double s_red[T / 32];
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int nr = pc.nr;
  for (int c = tid; c < nr; c += T) s_v[c] = v[c];
  __syncthreads();
  double dot = 0.0;
  const int64_t nwarps = (int64_t)gridDim.x * (T / 32);
  for (int64_t i = (int64_t)blockIdx.x * (T / 32) + warp; i < pc.n; i += nwarps) {
    const float* qrow = pc.Q + i * nr;
    double s = 0.0;
    for (int c = lane; c < nr; c += 32) s = fma((double)qrow[c], s_v[c], s);
    s = warp_sum(s);
    if (lane == 0) {
      const double ri = r[i];
      const ZT zi = (ZT)(pc.cis * ri + s);
      z[i] = zi;
      dot = fma(ri, (double)zi, dot);
    }
  }
  double vals[1] = {dot};
  block_sum<T, 1>(vals, s_red);
  if (tid == 0) blockpart[blockIdx.x] = vals[0];
  if (!arrive_last_block(counter)) return;
  if (warp == 0) {
    double t = 0.0;
    // fixed order: lane-strided partial sums, then a fixed shuffle tree
    for (unsigned int b = lane; b < gridDim.x; b += 32) t += __ldcg(blockpart + b);
    t = warp_sum(t);
    if (lane == 0) {
      if (st) {
        if (init) {
          st->rz = t;
          st->beta = 0.0;
        } else {
          st->beta = t / st->rz;
          st->rz = t;
        }
        if (!isfinite(t)) {
          st->status = LAKER_ERR_NONFINITE;
          st->done = 1;
          st->active = 0;
        }
      } else if (dot_out) {
        *dot_out = t;
      }
    }
  }
}

}  // namespace laker
