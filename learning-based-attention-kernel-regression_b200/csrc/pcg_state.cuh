// Device-resident state of one PCG solve and the single-RHS preconditioner
// kernels shared by the standalone apply and the PCG loop.
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
  double rmax;        // max recurrence residual norm since the last FP64 recomputation
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
constexpr int kPcChunkCols = 128;  // columns covered by one float4 per lane of a warp

struct PcView {
  const float* Q;  // (n x ldq) row-major, columns nr..ldq-1 zero, rows 16-byte aligned
  const float* W;  // (nr x nr) symmetric
  int64_t n;
  int nr;
  int ldq;     // multiple of 4
  double cis;  // c^-1/2
};

// Rows a warp keeps in flight so that every lane has ~8 float4 loads pending.
template <int NCH>
struct PcRows {
  static constexpr int value = NCH >= 8 ? 1 : 8 / NCH;
};

// u = Q^T r, then v = W u.  One pass over Q: each warp walks rows with float4
// loads (lane l covers columns 4l + 128 j), keeping several rows in flight;
// per-warp FP32 column sums are combined in FP64 per block, and the last block
// forms the fixed-order FP64 total and v = W u.  HBM-bound: n * ldq * 4 bytes.
template <int T, int NCH>
__global__ void __launch_bounds__(T)
    pc_project_kernel(PcView pc, const double* __restrict__ r, double* __restrict__ upart,
                      double* __restrict__ v, unsigned int* counter, const int* gate) {
  if (gate && *gate == 0) return;
  constexpr int RW = PcRows<NCH>::value;
  constexpr int NW = T / 32;
  __shared__ __align__(16) float s_w[NW][NCH * kPcChunkCols];
  __shared__ double s_u[kMaxNr];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int ldq4 = pc.ldq >> 2;
  const float4* Q4 = reinterpret_cast<const float4*>(pc.Q);
  float4 acc[NCH];
#pragma unroll
  for (int ch = 0; ch < NCH; ++ch) acc[ch] = make_float4(0.f, 0.f, 0.f, 0.f);
  const int64_t nwarps = (int64_t)gridDim.x * NW;
  const int64_t wid = (int64_t)blockIdx.x * NW + warp;
  for (int64_t i0 = wid; i0 < pc.n; i0 += nwarps * RW) {
    float rv[RW];
    float4 q[RW][NCH];
#pragma unroll
    for (int u = 0; u < RW; ++u) {
      const int64_t i = i0 + (int64_t)u * nwarps;
      const bool ok = i < pc.n;
      rv[u] = ok ? (float)r[i] : 0.0f;
#pragma unroll
      for (int ch = 0; ch < NCH; ++ch) {
        const int c4 = lane + 32 * ch;
        q[u][ch] = (ok && c4 < ldq4) ? __ldg(Q4 + i * ldq4 + c4) : make_float4(0.f, 0.f, 0.f, 0.f);
      }
    }
#pragma unroll
    for (int u = 0; u < RW; ++u)
#pragma unroll
      for (int ch = 0; ch < NCH; ++ch) {
        acc[ch].x = fmaf(q[u][ch].x, rv[u], acc[ch].x);
        acc[ch].y = fmaf(q[u][ch].y, rv[u], acc[ch].y);
        acc[ch].z = fmaf(q[u][ch].z, rv[u], acc[ch].z);
        acc[ch].w = fmaf(q[u][ch].w, rv[u], acc[ch].w);
      }
  }
#pragma unroll
  for (int ch = 0; ch < NCH; ++ch)
    reinterpret_cast<float4*>(s_w[warp])[lane + 32 * ch] = acc[ch];
  __syncthreads();
  for (int c = threadIdx.x; c < pc.ldq; c += T) {
    double s = 0.0;
#pragma unroll
    for (int w = 0; w < NW; ++w) s += (double)s_w[w][c];
    upart[(int64_t)blockIdx.x * pc.ldq + c] = s;
  }
  if (!arrive_last_block(counter)) return;
  const int nr = pc.nr;
  // both sums in one fixed order, with 16 loads issued ahead of their adds
  for (int c = threadIdx.x; c < nr; c += T) {
    double u = 0.0;
    unsigned int b = 0;
    for (; b + 16 <= gridDim.x; b += 16) {
      double t[16];
#pragma unroll
      for (int e = 0; e < 16; ++e) t[e] = __ldcg(upart + (int64_t)(b + e) * pc.ldq + c);
#pragma unroll
      for (int e = 0; e < 16; ++e) u += t[e];
    }
    for (; b < gridDim.x; ++b) u += __ldcg(upart + (int64_t)b * pc.ldq + c);
    s_u[c] = u;
  }
  __syncthreads();
  for (int c = threadIdx.x; c < nr; c += T) {
    double acc2 = 0.0;
    int cc = 0;
    for (; cc + 16 <= nr; cc += 16) {
      float t[16];
#pragma unroll
      for (int e = 0; e < 16; ++e) t[e] = __ldg(pc.W + (int64_t)(cc + e) * nr + c);
#pragma unroll
      for (int e = 0; e < 16; ++e) acc2 = fma((double)t[e], s_u[cc + e], acc2);
    }
    for (; cc < nr; ++cc) acc2 = fma((double)pc.W[(int64_t)cc * nr + c], s_u[cc], acc2);
    v[c] = acc2;
  }
}

// z = c^-1/2 r + Q v (one warp per row, float4 loads, several rows in flight)
// and the fixed-order total of r . z.  With a PcgState the last block turns
// r . z into beta (or seeds rz when `init`); without one it stores the total
// in dot_out (if non-null).  HBM-bound: n * ldq * 4 bytes.
template <int T, int NCH, typename ZT>
__global__ void __launch_bounds__(T)
    pc_expand_kernel(PcView pc, const double* __restrict__ r, const double* __restrict__ v,
                     ZT* __restrict__ z, double* __restrict__ blockpart, unsigned int* counter,
                     PcgState* st, int init, double* dot_out, const int* gate) {
  if (gate && *gate == 0) return;
  constexpr int RW = PcRows<NCH>::value;
  constexpr int NW = T / 32;
  __shared__ __align__(16) float s_v[NCH * kPcChunkCols];
  __shared__ double s_red[NW];
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  for (int c = tid; c < NCH * kPcChunkCols; c += T) s_v[c] = (c < pc.nr) ? (float)v[c] : 0.0f;
  __syncthreads();
  const int ldq4 = pc.ldq >> 2;
  const float4* Q4 = reinterpret_cast<const float4*>(pc.Q);
  const float4* V4 = reinterpret_cast<const float4*>(s_v);
  double dot = 0.0;
  const int64_t nwarps = (int64_t)gridDim.x * NW;
  for (int64_t i0 = (int64_t)blockIdx.x * NW + warp; i0 < pc.n; i0 += nwarps * RW) {
    float4 q[RW][NCH];
#pragma unroll
    for (int u = 0; u < RW; ++u) {
      const int64_t i = i0 + (int64_t)u * nwarps;
#pragma unroll
      for (int ch = 0; ch < NCH; ++ch) {
        const int c4 = lane + 32 * ch;
        q[u][ch] = (i < pc.n && c4 < ldq4) ? __ldg(Q4 + i * ldq4 + c4)
                                           : make_float4(0.f, 0.f, 0.f, 0.f);
      }
    }
#pragma unroll
    for (int u = 0; u < RW; ++u) {
      const int64_t i = i0 + (int64_t)u * nwarps;
      float s = 0.0f;
#pragma unroll
      for (int ch = 0; ch < NCH; ++ch) {
        const float4 vv = V4[lane + 32 * ch];
        s = fmaf(q[u][ch].x, vv.x, s);
        s = fmaf(q[u][ch].y, vv.y, s);
        s = fmaf(q[u][ch].z, vv.z, s);
        s = fmaf(q[u][ch].w, vv.w, s);
      }
      s = warp_sum(s);
      if (lane == 0 && i < pc.n) {
        const double ri = r[i];
        const ZT zi = (ZT)(pc.cis * ri + (double)s);
        z[i] = zi;
        dot = fma(ri, (double)zi, dot);
      }
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

// Number of 128-column chunks (float4 per lane) of a padded Q row.
inline int pc_chunks(int ldq) { return (ldq + kPcChunkCols - 1) / kPcChunkCols; }

#define LAKER_PC_DISPATCH(nch, ...)                          \
  switch (nch) {                                              \
    case 1: { constexpr int NC = 1; __VA_ARGS__; } break;     \
    case 2: { constexpr int NC = 2; __VA_ARGS__; } break;     \
    case 3: { constexpr int NC = 3; __VA_ARGS__; } break;     \
    case 4: { constexpr int NC = 4; __VA_ARGS__; } break;     \
    case 5: { constexpr int NC = 5; __VA_ARGS__; } break;     \
    case 6: { constexpr int NC = 6; __VA_ARGS__; } break;     \
    case 7: { constexpr int NC = 7; __VA_ARGS__; } break;     \
    default: { constexpr int NC = 8; __VA_ARGS__; } break;    \
  }

// The two-pass apply, z = P r: projection then expansion on stream s.
template <typename ZT>
inline void launch_precond_apply(const PcView& pc, int grid, const double* r, double* upart,
                                 double* v, ZT* z, double* blockpart, unsigned int* ctr_project,
                                 unsigned int* ctr_expand, PcgState* st, int init,
                                 double* dot_out, const int* gate, cudaStream_t s) {
  LAKER_PC_DISPATCH(pc_chunks(pc.ldq), {
    pc_project_kernel<kVecThreads, NC><<<grid, kVecThreads, 0, s>>>(pc, r, upart, v, ctr_project,
                                                                    gate);
    pc_expand_kernel<kVecThreads, NC, ZT><<<grid, kVecThreads, 0, s>>>(
        pc, r, v, z, blockpart, ctr_expand, st, init, dot_out, gate);
  });
}

}  // namespace laker
