// Batched mixed-precision PCG: many independent regressions in one device loop.
//
// The instances are laid end to end (instance k at points off[k] ..
// off[k] + n[k], off 256-aligned), so one launch of the symmetric FP32 matvec
// over the concatenated block-pair lists applies every instance's operator
// (a block-diagonal operator), skipping converged instances.  Every other step
// runs one CTA per instance, which owns the instance's vectors and scalars and
// so needs no grid-wide reduction:
//   after_matvec : Ap = lam p + partials; p.Ap -> alpha; x += alpha p;
//                  r -= alpha Ap; |r| -> reliable-update decision
//   residual     : r = b - A64 x for the instances that asked (FP64 kernel,
//                  one CTA per 512-row block)
//   after_resid  : |r| -> stop test, convergence mask
//   precond      : u = Q^T r, v = W u, z = c r + Q v, r.z -> beta, p = z + beta p
// The iteration (5 launches) is captured once into a CUDA graph; the host
// replays it and polls the number of running instances between replays.
#include <algorithm>
#include <vector>

#include "pcg_state.cuh"
#include "sym.cuh"

namespace laker {
int precond_grid();

namespace {

constexpr int BT = 256;           // threads of the per-instance kernels
constexpr int kBatchAlign = 256;  // instance segment alignment (points)

struct InstState {
  double bnorm, tol_abs, rz, pAp, alpha, beta, rnorm, rmax, true_rnorm;
  int iter, n_accurate, done, status, need_update, pad0, pad1, pad2;
};

struct BatchDev {
  int count;
  int has_pc;
  int max_iter;
  int d;
  double delta, eps, tol;
  const int64_t* off;       // [count + 1]
  const int64_t* npts;      // [count]
  const double* lam;        // [count]
  const uint64_t* q;        // [count] Q pointers
  const uint64_t* w;        // [count] W pointers
  const int* nr;            // [count]
  const int* ldq;           // [count]
  const double* cis;        // [count]
  InstState* st;            // [count]
  int* done;                // [count] mirror of st[k].done for the matvec
  int* active;              // number of running instances
};

__device__ __forceinline__ void finish_instance(const BatchDev& bd, int k, int status) {
  bd.st[k].status = status;
  bd.st[k].done = 1;
  bd.done[k] = 1;
  atomicSub(bd.active, 1);
}

// x = 0, r = b, |b| -> seeds the instance state (zero rhs: done at once).
__global__ void __launch_bounds__(BT)
    batch_init_kernel(BatchDev bd, const double* __restrict__ B, double* __restrict__ X,
                      double* __restrict__ r) {
  const int k = blockIdx.x;
  const int64_t seg = bd.off[k], n = bd.npts[k];
  __shared__ double s_red[BT / 32];
  double acc = 0.0;
  for (int64_t i = threadIdx.x; i < n; i += BT) {
    const double bi = B[seg + i];
    r[seg + i] = bi;
    X[seg + i] = 0.0;
    acc = fma(bi, bi, acc);
  }
  double v[1] = {acc};
  block_sum<BT, 1>(v, s_red);
  if (threadIdx.x == 0) {
    InstState s{};
    const double bn = sqrt(v[0]);
    s.bnorm = bn;
    s.tol_abs = bd.tol * bn;
    s.rnorm = s.rmax = s.true_rnorm = bn;
    bd.st[k] = s;
    bd.done[k] = 0;
    if (bn == 0.0) {
      finish_instance(bd, k, LAKER_OK);
    } else if (!isfinite(bn)) {
      finish_instance(bd, k, LAKER_ERR_NONFINITE);
    }
  }
}

// z = P r (or r without a preconditioner), r.z -> beta (rz seeded on init),
// p = z + beta p.
__global__ void __launch_bounds__(BT)
    batch_precond_kernel(BatchDev bd, const double* __restrict__ r, float* __restrict__ z,
                         float* __restrict__ p, int init) {
  const int k = blockIdx.x;
  if (bd.st[k].done) return;
  constexpr int NW = BT / 32;
  __shared__ __align__(16) float s_w[NW][kMaxNr];
  __shared__ double s_u[kMaxNr];
  __shared__ __align__(16) float s_v[kMaxNr];
  __shared__ double s_red[NW];
  __shared__ double s_beta;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int64_t seg = bd.off[k], n = bd.npts[k];
  double dot = 0.0;
  if (bd.has_pc) {
    const float4* Q4 = reinterpret_cast<const float4*>(bd.q[k]);
    const float* W = reinterpret_cast<const float*>(bd.w[k]);
    const int nr = bd.nr[k], ldq = bd.ldq[k], ldq4 = ldq >> 2;
    const int nch = (ldq + kPcChunkCols - 1) / kPcChunkCols;
    // project: per-warp column sums (lane owns float4 chunks lane + 32 ch)
    float4 acc[8];
#pragma unroll
    for (int ch = 0; ch < 8; ++ch) acc[ch] = make_float4(0.f, 0.f, 0.f, 0.f);
    for (int64_t i = warp; i < n; i += NW) {
      const float ri = (float)r[seg + i];
#pragma unroll
      for (int ch = 0; ch < 8; ++ch) {
        const int c4 = lane + 32 * ch;
        if (ch < nch && c4 < ldq4) {
          const float4 q = __ldg(Q4 + i * ldq4 + c4);
          acc[ch].x = fmaf(q.x, ri, acc[ch].x);
          acc[ch].y = fmaf(q.y, ri, acc[ch].y);
          acc[ch].z = fmaf(q.z, ri, acc[ch].z);
          acc[ch].w = fmaf(q.w, ri, acc[ch].w);
        }
      }
    }
#pragma unroll
    for (int ch = 0; ch < 8; ++ch) {
      const int c4 = lane + 32 * ch;
      if (ch < nch && c4 < ldq4) reinterpret_cast<float4*>(s_w[warp])[c4] = acc[ch];
    }
    __syncthreads();
    for (int c = tid; c < nr; c += BT) {
      double u = 0.0;
#pragma unroll
      for (int w2 = 0; w2 < NW; ++w2) u += (double)s_w[w2][c];
      s_u[c] = u;
    }
    __syncthreads();
    for (int c = tid; c < ldq; c += BT) {
      double a2 = 0.0;
      if (c < nr)
        for (int cc = 0; cc < nr; ++cc) a2 = fma((double)W[(int64_t)cc * nr + c], s_u[cc], a2);
      s_v[c] = (float)a2;
    }
    __syncthreads();
    // expand: one warp per row
    const float4* V4 = reinterpret_cast<const float4*>(s_v);
    const double cis = bd.cis[k];
    for (int64_t i = warp; i < n; i += NW) {
      float s = 0.0f;
#pragma unroll
      for (int ch = 0; ch < 8; ++ch) {
        const int c4 = lane + 32 * ch;
        if (ch < nch && c4 < ldq4) {
          const float4 q = __ldg(Q4 + i * ldq4 + c4);
          const float4 vv = V4[c4];
          s = fmaf(q.x, vv.x, s);
          s = fmaf(q.y, vv.y, s);
          s = fmaf(q.z, vv.z, s);
          s = fmaf(q.w, vv.w, s);
        }
      }
      s = warp_sum(s);
      if (lane == 0) {
        const double ri = r[seg + i];
        const float zi = (float)(cis * ri + (double)s);
        z[seg + i] = zi;
        dot = fma(ri, (double)zi, dot);
      }
    }
  } else {
    for (int64_t i = tid; i < n; i += BT) {
      const double ri = r[seg + i];
      const float zi = (float)ri;
      z[seg + i] = zi;
      dot = fma(ri, (double)zi, dot);
    }
  }
  double vals[1] = {dot};
  block_sum<BT, 1>(vals, s_red);
  if (tid == 0) {
    InstState& s = bd.st[k];
    if (init) {
      s.rz = vals[0];
      s.beta = 0.0;
    } else {
      s.beta = vals[0] / s.rz;
      s.rz = vals[0];
    }
    s_beta = s.beta;
    if (!isfinite(vals[0])) finish_instance(bd, k, LAKER_ERR_NONFINITE);
  }
  __syncthreads();
  if (bd.st[k].done) return;
  const float beta = (float)s_beta;
  for (int64_t i = tid; i < n; i += BT)
    p[seg + i] = init ? z[seg + i] : fmaf(beta, p[seg + i], z[seg + i]);
}

// Ap = lam p + (symmetric partials); alpha; x, r update; reliable-update test.
__global__ void __launch_bounds__(BT)
    batch_after_matvec_kernel(BatchDev bd, SymPlan sp, BatchMap bm,
                              const float* __restrict__ rowpart, const float* __restrict__ colpart,
                              const float* __restrict__ p, float* __restrict__ Ap,
                              double* __restrict__ X, double* __restrict__ r) {
  const int k = blockIdx.x;
  if (bd.st[k].done) return;
  __shared__ double s_red[3 * (BT / 32)];
  __shared__ double s_alpha;
  __shared__ int s_stop;
  const int64_t seg = bd.off[k], n = bd.npts[k];
  const double lam = bd.lam[k];
  double d0 = 0.0, d1 = 0.0, d2 = 0.0;
  for (int64_t i = threadIdx.x; i < n; i += BT) {
    const double pi = p[seg + i];
    const double a = lam * pi + sym_row_sum_batched(sp, bm, rowpart, colpart, k, i);
    const float af = (float)a;
    Ap[seg + i] = af;
    d0 = fma(pi, (double)af, d0);
    d1 = fma(pi, pi, d1);
    d2 = fma((double)af, (double)af, d2);
  }
  double v[3] = {d0, d1, d2};
  block_sum<BT, 3>(v, s_red);
  if (threadIdx.x == 0) {
    InstState& s = bd.st[k];
    s.pAp = v[0];
    s_stop = 0;
    if (!isfinite(v[0]) || !isfinite(v[1]) || !isfinite(v[2])) {
      finish_instance(bd, k, LAKER_ERR_NONFINITE);
      s_stop = 1;
    } else if (v[0] <= -bd.eps * sqrt(v[1]) * sqrt(v[2])) {
      finish_instance(bd, k, LAKER_ERR_BREAKDOWN);  // laker/solvers.py:232-246
      s_stop = 1;
    } else {
      s.alpha = s.rz / v[0];
    }
    s_alpha = s.alpha;
  }
  __syncthreads();
  if (s_stop) return;
  const double alpha = s_alpha;
  double rr = 0.0;
  for (int64_t i = threadIdx.x; i < n; i += BT) {
    X[seg + i] = fma(alpha, (double)p[seg + i], X[seg + i]);
    const double ri = fma(-alpha, (double)Ap[seg + i], r[seg + i]);
    r[seg + i] = ri;
    rr = fma(ri, ri, rr);
  }
  double w1[1] = {rr};
  block_sum<BT, 1>(w1, s_red);
  if (threadIdx.x == 0) {
    InstState& s = bd.st[k];
    const double rn = sqrt(w1[0]);
    s.rnorm = rn;
    s.iter += 1;
    if (rn > s.rmax) s.rmax = rn;
    s.need_update =
        (rn <= bd.delta * s.rmax || rn <= s.tol_abs || s.iter >= bd.max_iter || !isfinite(rn)) ? 1 : 0;
  }
}

// r = b - (lam x + K64 x) for the instances whose need_update is set; one CTA
// per 512-row block of an instance, FP64 logits / exp / accumulation, column
// tiles staged in shared memory.
template <int DP>
__global__ void __launch_bounds__(BT)
    batch_residual_kernel(BatchDev bd, BatchMap bm, const double* __restrict__ E64,
                          const double* __restrict__ B, const double* __restrict__ X,
                          double* __restrict__ r, int clamp) {
  constexpr int R = 2, TCc = 64;
  const int64_t g = blockIdx.x;
  // instance of global block g
  int lo = 0, hi = bd.count - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (bm.blk_start[mid] <= g) lo = mid; else hi = mid - 1;
  }
  const int k = lo;
  if (bd.st[k].done || !bd.st[k].need_update) return;
  __shared__ __align__(16) double sE[TCc * DP];
  __shared__ double sX[TCc];
  const int64_t seg = bd.off[k], n = bd.npts[k];
  const int64_t a = g - bm.blk_start[k];
  double ev[R][DP], acc[R];
#pragma unroll
  for (int q = 0; q < R; ++q) {
    const int64_t li = a * (BT * R) + q * BT + threadIdx.x;
#pragma unroll
    for (int kk = 0; kk < DP; ++kk) ev[q][kk] = (li < n) ? E64[(seg + li) * DP + kk] : 0.0;
    acc[q] = 0.0;
  }
  for (int64_t j0 = 0; j0 < n; j0 += TCc) {
    __syncthreads();
    for (int o = threadIdx.x; o < TCc * DP; o += BT) {
      const int jj = o / DP;
      sE[o] = (j0 + jj < n) ? E64[(seg + j0) * DP + o] : 0.0;
    }
    for (int jj = threadIdx.x; jj < TCc; jj += BT) sX[jj] = (j0 + jj < n) ? X[seg + j0 + jj] : 0.0;
    __syncthreads();
#pragma unroll 2
    for (int jj = 0; jj < TCc; ++jj) {
      const double xj = sX[jj];
#pragma unroll
      for (int q = 0; q < R; ++q) {
        double s = ev[q][0] * sE[jj * DP];
#pragma unroll
        for (int kk = 1; kk < DP; ++kk) s = fma(ev[q][kk], sE[jj * DP + kk], s);
        if (clamp) s = fmin(s, kClamp64);
        acc[q] = fma(exp(s), xj, acc[q]);
      }
    }
  }
  const double lam = bd.lam[k];
#pragma unroll
  for (int q = 0; q < R; ++q) {
    const int64_t li = a * (BT * R) + q * BT + threadIdx.x;
    if (li < n) r[seg + li] = B[seg + li] - (lam * X[seg + li] + acc[q]);
  }
}

// |r| after an FP64 recomputation -> stop test.
__global__ void __launch_bounds__(BT) batch_after_residual_kernel(BatchDev bd, const double* __restrict__ r) {
  const int k = blockIdx.x;
  if (bd.st[k].done || !bd.st[k].need_update) return;
  __shared__ double s_red[BT / 32];
  const int64_t seg = bd.off[k], n = bd.npts[k];
  double rr = 0.0;
  for (int64_t i = threadIdx.x; i < n; i += BT) rr = fma(r[seg + i], r[seg + i], rr);
  double v[1] = {rr};
  block_sum<BT, 1>(v, s_red);
  if (threadIdx.x == 0) {
    InstState& s = bd.st[k];
    const double rn = sqrt(v[0]);
    s.rnorm = s.true_rnorm = s.rmax = rn;
    s.n_accurate += 1;
    s.need_update = 0;
    if (!isfinite(rn)) finish_instance(bd, k, LAKER_ERR_NONFINITE);
    else if (rn <= s.tol_abs) finish_instance(bd, k, LAKER_OK);
    else if (s.iter >= bd.max_iter) finish_instance(bd, k, LAKER_ERR_NOT_CONVERGED);
  }
}

// Host-side description of one batch solve (sizes and workspace carve-up).
struct BatchLayout {
  int count = 0;
  int64_t total = 0;        // padded points
  int64_t total_blocks = 0;
  int64_t total_pairs = 0;
  std::vector<int64_t> off, nblk, pair_start, blk_start;
  SymPlan sp{};
  size_t bytes = 0;
  // byte offsets into the workspace
  size_t o_hdr, o_off, o_npts, o_nblk, o_ps, o_bs, o_lam, o_q, o_w, o_nr, o_ldq, o_cis, o_st,
      o_done, o_active, o_r, o_z, o_p, o_ap, o_rowpart, o_colpart;
};

BatchLayout make_layout(int count, const int64_t* n, int d) {
  BatchLayout L;
  L.count = count;
  const int B = sym_block_points();
  L.off.resize(count + 1);
  L.nblk.resize(count);
  L.pair_start.resize(count + 1);
  L.blk_start.resize(count + 1);
  L.off[0] = L.pair_start[0] = L.blk_start[0] = 0;
  for (int k = 0; k < count; ++k) {
    const int64_t nk = n[k] > 0 ? n[k] : 0;
    L.off[k + 1] = L.off[k] + round_up(nk > 0 ? nk : 1, kBatchAlign);
    L.nblk[k] = nk > 0 ? ceil_div(nk, B) : 0;
    L.blk_start[k + 1] = L.blk_start[k] + L.nblk[k];
    L.pair_start[k + 1] = L.pair_start[k] + L.nblk[k] * (L.nblk[k] + 1) / 2;
  }
  L.total = L.off[count];
  L.total_blocks = L.blk_start[count];
  L.total_pairs = L.pair_start[count];
  L.sp = k1s_plan_pairs(L.total_blocks > 0 ? L.total_blocks : 1, L.total_pairs > 0 ? L.total_pairs : 1, d);
  size_t o = 0;
  auto take = [&](size_t b) {
    const size_t at = o;
    o += (size_t)round_up((int64_t)(b ? b : 1), 256);
    return at;
  };
  const size_t c = (size_t)count;
  L.o_hdr = take(kWsHeader);
  L.o_off = take((c + 1) * 8);
  L.o_npts = take(c * 8);
  L.o_nblk = take(c * 8);
  L.o_ps = take((c + 1) * 8);
  L.o_bs = take((c + 1) * 8);
  L.o_lam = take(c * 8);
  L.o_q = take(c * 8);
  L.o_w = take(c * 8);
  L.o_nr = take(c * 4);
  L.o_ldq = take(c * 4);
  L.o_cis = take(c * 8);
  L.o_st = take(c * sizeof(InstState));
  L.o_done = take(c * 4);
  L.o_active = take(256);
  L.o_r = take((size_t)L.total * 8);
  L.o_z = take((size_t)L.total * 4);
  L.o_p = take((size_t)L.total * 4);
  L.o_ap = take((size_t)L.total * 4);
  L.o_rowpart = take(sym_rowpart_elems(L.sp) * 4);
  L.o_colpart = take(sym_colpart_elems(L.sp) * 4);
  L.bytes = o;
  return L;
}

#define LAKER_DISPATCH_DPB(dp, CALL)                    \
  switch (dp) {                                         \
    case 2: { constexpr int DPv = 2; CALL; } break;     \
    case 4: { constexpr int DPv = 4; CALL; } break;     \
    case 6: { constexpr int DPv = 6; CALL; } break;     \
    case 8: { constexpr int DPv = 8; CALL; } break;     \
    case 10: { constexpr int DPv = 10; CALL; } break;   \
    case 12: { constexpr int DPv = 12; CALL; } break;   \
    case 14: { constexpr int DPv = 14; CALL; } break;   \
    case 16: { constexpr int DPv = 16; CALL; } break;   \
    default: break;                                     \
  }

}  // namespace
}  // namespace laker

using namespace laker;

extern "C" int64_t laker_batch_layout(int count, const int64_t* n, int64_t* offsets) {
  if (count < 0 || (count > 0 && !n)) return -1;
  int64_t o = 0;
  for (int k = 0; k < count; ++k) {
    if (offsets) offsets[k] = o;
    o += round_up(n[k] > 0 ? n[k] : 1, kBatchAlign);
  }
  if (offsets) offsets[count] = o;
  return o;
}

extern "C" size_t laker_pcg_batched_workspace_bytes(int count, const int64_t* n, int d) {
  if (count < 1 || !n || d < 1 || d > 16) return 0;
  for (int k = 0; k < count; ++k)
    if (n[k] < 1) return 0;
  return make_layout(count, n, d).bytes;
}

extern "C" int laker_pcg_solve_batched(const laker_batch* batch, const double* B, double* X,
                                       const laker_pcg_params* prm, void* workspace,
                                       size_t workspace_bytes, laker_pcg_result* results,
                                       void* stream) {
  if (!batch || !prm || !B || !X || !workspace || !results) return LAKER_ERR_INVALID_ARG;
  const int count = batch->count, d = batch->d;
  if (count < 1 || d < 1 || d > 16 || !batch->n || !batch->lambda_reg || !batch->packed32 ||
      !batch->packed64)
    return LAKER_ERR_INVALID_ARG;
  if (prm->max_iter < 0 || !(prm->tol >= 0.0) || !(prm->reliable_delta > 0.0) || prm->has_x0)
    return LAKER_ERR_INVALID_ARG;  // warm starts are not supported in batched mode
  for (int k = 0; k < count; ++k) {
    if (batch->n[k] < 1) return LAKER_ERR_INVALID_ARG;
    if (batch->precond) {
      const laker_precond& pc = batch->precond[k];
      if (pc.n != batch->n[k] || pc.nr < 1 || pc.nr > kMaxNr || pc.ldq < pc.nr || pc.ldq > kMaxNr ||
          (pc.ldq % 4) || !pc.q_basis || !pc.w_core || (reinterpret_cast<uintptr_t>(pc.q_basis) % 16))
        return LAKER_ERR_INVALID_ARG;
    }
  }
  const BatchLayout L = make_layout(count, batch->n, d);
  if (workspace_bytes < L.bytes) return LAKER_ERR_WORKSPACE;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  char* base = static_cast<char*>(workspace);
  auto at = [&](size_t o) { return static_cast<void*>(base + o); };

  // ---- device tables ----------------------------------------------------------
  std::vector<int64_t> npts(count);
  std::vector<double> lam(count), cis(count, 1.0);
  std::vector<uint64_t> qp(count, 0), wp(count, 0);
  std::vector<int> nr(count, 0), ldq(count, 4);
  for (int k = 0; k < count; ++k) {
    npts[k] = batch->n[k];
    lam[k] = batch->lambda_reg[k];
    if (batch->precond) {
      const laker_precond& pc = batch->precond[k];
      qp[k] = reinterpret_cast<uint64_t>(pc.q_basis);
      wp[k] = reinterpret_cast<uint64_t>(pc.w_core);
      nr[k] = pc.nr;
      ldq[k] = pc.ldq;
      cis[k] = pc.inv_sqrt_iso;
    }
  }
  cudaError_t e = cudaMemsetAsync(at(L.o_hdr), 0, kWsHeader, s);
  auto h2d = [&](size_t o, const void* src, size_t bytes) {
    if (e == cudaSuccess) e = cudaMemcpyAsync(at(o), src, bytes, cudaMemcpyHostToDevice, s);
  };
  h2d(L.o_off, L.off.data(), (count + 1) * 8);
  h2d(L.o_npts, npts.data(), count * 8);
  h2d(L.o_nblk, L.nblk.data(), count * 8);
  h2d(L.o_ps, L.pair_start.data(), (count + 1) * 8);
  h2d(L.o_bs, L.blk_start.data(), (count + 1) * 8);
  h2d(L.o_lam, lam.data(), count * 8);
  h2d(L.o_q, qp.data(), count * 8);
  h2d(L.o_w, wp.data(), count * 8);
  h2d(L.o_nr, nr.data(), count * 4);
  h2d(L.o_ldq, ldq.data(), count * 4);
  h2d(L.o_cis, cis.data(), count * 8);
  int active_init = count;
  h2d(L.o_active, &active_init, 4);
  if (e != cudaSuccess) return fail_cuda(e);

  BatchDev bd{};
  bd.count = count;
  bd.has_pc = batch->precond ? 1 : 0;
  bd.max_iter = prm->max_iter;
  bd.d = d;
  bd.delta = prm->reliable_delta;
  bd.eps = prm->breakdown_eps;
  bd.tol = prm->tol;
  bd.off = static_cast<const int64_t*>(at(L.o_off));
  bd.npts = static_cast<const int64_t*>(at(L.o_npts));
  bd.lam = static_cast<const double*>(at(L.o_lam));
  bd.q = static_cast<const uint64_t*>(at(L.o_q));
  bd.w = static_cast<const uint64_t*>(at(L.o_w));
  bd.nr = static_cast<const int*>(at(L.o_nr));
  bd.ldq = static_cast<const int*>(at(L.o_ldq));
  bd.cis = static_cast<const double*>(at(L.o_cis));
  bd.st = static_cast<InstState*>(at(L.o_st));
  bd.done = static_cast<int*>(at(L.o_done));
  bd.active = static_cast<int*>(at(L.o_active));

  BatchMap bm{};
  bm.count = count;
  bm.pair_start = static_cast<const int64_t*>(at(L.o_ps));
  bm.nblk = static_cast<const int64_t*>(at(L.o_nblk));
  bm.npts = bd.npts;
  bm.seg = bd.off;
  bm.blk_start = static_cast<const int64_t*>(at(L.o_bs));
  bm.done = bd.done;

  double* r = static_cast<double*>(at(L.o_r));
  float* z = static_cast<float*>(at(L.o_z));
  float* p = static_cast<float*>(at(L.o_p));
  float* Ap = static_cast<float*>(at(L.o_ap));
  float* rowpart = static_cast<float*>(at(L.o_rowpart));
  float* colpart = static_cast<float*>(at(L.o_colpart));
  int* dstatus = &static_cast<WsHeader*>(at(L.o_hdr))->status;
  const int dp = padded_dim(d);
  const unsigned nblocks = (unsigned)(L.total_blocks > 0 ? L.total_blocks : 1);

  int launches = 0;
  // ---- initialisation (plain launches on the caller's stream) ----------------
  batch_init_kernel<<<count, BT, 0, s>>>(bd, B, X, r);
  batch_precond_kernel<<<count, BT, 0, s>>>(bd, r, z, p, 1);
  launches += 2;
  e = cudaGetLastError();
  if (e != cudaSuccess) return fail_cuda(e);

  // ---- one iteration, captured once as a graph --------------------------------
  auto iteration = [&](cudaStream_t cs) -> cudaError_t {
    cudaError_t ee = launch_k1s_batched(batch->packed32, d, batch->clamp, p, rowpart, colpart, L.sp,
                                        bm, dstatus, bd.active, cs);
    if (ee != cudaSuccess) return ee;
    batch_after_matvec_kernel<<<count, BT, 0, cs>>>(bd, L.sp, bm, rowpart, colpart, p, Ap, X, r);
    LAKER_DISPATCH_DPB(dp, (batch_residual_kernel<DPv><<<nblocks, BT, 0, cs>>>(
                               bd, bm, batch->packed64, B, X, r, batch->clamp)));
    batch_after_residual_kernel<<<count, BT, 0, cs>>>(bd, r);
    batch_precond_kernel<<<count, BT, 0, cs>>>(bd, r, z, p, 0);
    return cudaGetLastError();
  };
  constexpr int kLaunchesPerIter = 5;
  int chunk = prm->check_every > 0 ? prm->check_every : 8;
  if (chunk > prm->max_iter && prm->max_iter > 0) chunk = prm->max_iter;

  cudaStream_t cs = nullptr;
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  e = cudaStreamCreateWithFlags(&cs, cudaStreamNonBlocking);
  if (e == cudaSuccess) e = cudaStreamBeginCapture(cs, cudaStreamCaptureModeThreadLocal);
  if (e == cudaSuccess) {
    cudaError_t ce = cudaSuccess;
    for (int it = 0; it < chunk && ce == cudaSuccess; ++it) ce = iteration(cs);
    e = cudaStreamEndCapture(cs, &graph);
    if (e == cudaSuccess) e = ce;
  }
  if (e == cudaSuccess) e = cudaGraphInstantiate(&exec, graph, 0);
  int iters_launched = 0, active = count;
  while (e == cudaSuccess && iters_launched < prm->max_iter) {
    e = cudaGraphLaunch(exec, s);
    if (e != cudaSuccess) break;
    iters_launched += chunk;
    launches += chunk * kLaunchesPerIter;
    e = cudaMemcpyAsync(&active, bd.active, 4, cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess || active <= 0) break;
  }
  if (exec) cudaGraphExecDestroy(exec);
  if (graph) cudaGraphDestroy(graph);
  if (cs) cudaStreamDestroy(cs);
  if (e != cudaSuccess) return fail_cuda(e);

  // ---- results ------------------------------------------------------------------
  std::vector<InstState> hs(count);
  int dev_status = 0;
  e = cudaMemcpyAsync(hs.data(), bd.st, count * sizeof(InstState), cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess) e = cudaMemcpyAsync(&dev_status, dstatus, 4, cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  if (e != cudaSuccess) return fail_cuda(e);
  for (int k = 0; k < count; ++k) {
    laker_pcg_result& o = results[k];
    o = laker_pcg_result{};
    o.status = hs[k].done ? hs[k].status : LAKER_ERR_NOT_CONVERGED;
    o.iterations = hs[k].iter;
    o.accurate_matvecs = hs[k].n_accurate;
    o.residual_norm = hs[k].bnorm == 0.0 ? 0.0 : hs[k].true_rnorm;
    o.rhs_norm = hs[k].bnorm;
    o.recurrence_norm = hs[k].rnorm;
    o.kernel_launches = launches;
  }
  return dev_status ? dev_status : LAKER_OK;
}
