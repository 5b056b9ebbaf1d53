// Batched mixed-precision PCG: many independent regressions in one device loop.
//
// Layout: instance k sits at points off[k] .. off[k] + n[k] of every batched
// vector (off 256-aligned, zero padding between instances); its rows are cut
// into 512-point blocks, global blocks blk_start[k] .. blk_start[k+1]-1 (the
// blocks of the symmetric matvec).  One iteration, captured once as a CUDA
// graph and replayed by the host until no instance is running:
//   matvec     part = K32 p over the block pairs of the running instances
//              (list compacted on the device, split evenly over the grid)
//   after_mv   [block] Ap = lam p + partial sums; p.Ap, p.p, Ap.Ap
//              [last block of the instance] alpha, or breakdown
//   update_xr  [block] x += alpha p; r -= alpha Ap; |r|^2; Q_blk^T r
//              [last] reliable-update decision; v = W Q^T r unless a residual follows
//   residual   K64 x over the block pairs of the instances that asked (FP64
//              symmetric kernel, list compacted on the device), then
//              [block] r = b - lam x - partial sums; |r|^2; Q_blk^T r
//              [last] stop test; v = W Q^T r
//   expand     [block] z = c r + Q_blk v; r.z        [last] beta
//   update_p   [block] p = z + beta p
//   compact    running-instance list and pair prefix sums for the next matvec
// The recurrence is the one of laker_pcg_solve (laker/solvers.py:189-295 with
// FP64 residual replacement).  Block partials are added by the instance's last
// block in block order, and the matvec's partial sums are per block pair, so
// an instance's arithmetic is the same alone or in any batch.
#include <algorithm>
#include <vector>

#include "pcg_state.cuh"
#include "sym.cuh"

namespace laker {
namespace {

constexpr int BT = 256;             // threads of the block kernels
constexpr int NW = BT / 32;
constexpr int RB = 512;             // rows per block (the symmetric matvec's blocks)
constexpr int kBatchAlign = 256;    // instance segment alignment (points)
constexpr int kCompactThreads = 1024;
static_assert(RB == 2 * BT, "two rows per thread in the block kernels");

struct InstState {
  double bnorm, tol_abs, rz, alpha, beta, rnorm, rmax, true_rnorm;
  int iter, n_accurate, done, status, need_update, pad0;
};

struct BatchDev {
  int count;
  int has_pc;
  int max_iter;
  int ustride;              // floats per projection vector (>= every ldq)
  double delta, eps, tol;
  const int64_t* off;       // [count + 1]
  const int64_t* npts;      // [count]
  const int64_t* nblk;      // [count]
  const int64_t* blk_start; // [count + 1]
  const int* blk_inst;      // [total blocks]
  const double* lam;        // [count]
  const uint64_t* q;        // [count] Q pointers (n x ldq FP32)
  const uint64_t* w;        // [count] W pointers (nr x nr FP32)
  const int* nr;            // [count]
  const int* ldq;           // [count]
  const double* cis;        // [count] c^-1/2
  InstState* st;            // [count]
  int* done;                // [count]
  int* active;              // running instances (host poll, matvec gate)
  unsigned int* ctr;        // [count] block arrival counters
  double* bpart;            // [total blocks * 4] block partial scalars
  float* upart;             // [total blocks * ustride] block partials of Q^T r
  float* vvec;              // [count * ustride] v = W Q^T r
};

struct BlockCtx {
  int64_t g;      // global block
  int k;          // instance
  unsigned nblk;  // blocks of the instance
  int64_t seg, n, row0, row1;
};

__device__ __forceinline__ BlockCtx block_ctx(const BatchDev& bd) {
  BlockCtx c;
  c.g = blockIdx.x;
  c.k = bd.blk_inst[c.g];
  const int64_t b0 = bd.blk_start[c.k];
  c.nblk = (unsigned)(bd.blk_start[c.k + 1] - b0);
  c.seg = bd.off[c.k];
  c.n = bd.npts[c.k];
  c.row0 = (c.g - b0) * RB;
  c.row1 = c.row0 + RB < c.n ? c.row0 + RB : c.n;
  return c;
}

__device__ __forceinline__ void finish_instance(const BatchDev& bd, int k, int status) {
  bd.st[k].status = status;
  bd.st[k].done = 1;
  bd.done[k] = 1;
}

// Sum of slot j of the instance's block partials, in block order.
__device__ __forceinline__ double sum_blocks(const BatchDev& bd, const BlockCtx& c, int j) {
  const int64_t b0 = bd.blk_start[c.k];
  double t = 0.0;
  for (unsigned b = 0; b < c.nblk; ++b) t += __ldcg(bd.bpart + (b0 + b) * 4 + j);
  return t;
}

// upart[g][col] = sum over the block's rows i of Q[i][col] * r_i.  Warps take
// rows; lane l holds the float4 column chunks l + 32 ch.  Caller has
// synchronised after writing r.
__device__ void project_block(const BatchDev& bd, const BlockCtx& c, const double* __restrict__ r,
                              float (*s_w)[kMaxNr]) {
  const float4* Q4 = reinterpret_cast<const float4*>(bd.q[c.k]);
  const int ldq = bd.ldq[c.k], ldq4 = ldq >> 2;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  float4 acc[8];
#pragma unroll
  for (int ch = 0; ch < 8; ++ch) acc[ch] = make_float4(0.f, 0.f, 0.f, 0.f);
  for (int64_t i = c.row0 + warp; i < c.row1; i += NW) {
    const float ri = (float)r[c.seg + i];
#pragma unroll
    for (int ch = 0; ch < 8; ++ch) {
      const int c4 = lane + 32 * ch;
      if (c4 < ldq4) {
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
    if (c4 < ldq4) reinterpret_cast<float4*>(s_w[warp])[c4] = acc[ch];
  }
  __syncthreads();
  float* dst = bd.upart + c.g * bd.ustride;
  for (int col = threadIdx.x; col < ldq; col += BT) {
    float s = 0.0f;
#pragma unroll
    for (int w2 = 0; w2 < NW; ++w2) s += s_w[w2][col];
    dst[col] = s;
  }
}

// Last block of an instance: u = sum of the block projections (block order),
// v = W u -> vvec[k].  s_u may alias the projection scratch (the arrival
// barrier separates the two uses).
__device__ void w_multiply(const BatchDev& bd, const BlockCtx& c, double* s_u) {
  const int nr = bd.nr[c.k], ldq = bd.ldq[c.k];
  const float* W = reinterpret_cast<const float*>(bd.w[c.k]);
  const int64_t b0 = bd.blk_start[c.k];
  for (int col = threadIdx.x; col < nr; col += BT) {
    double u = 0.0;
    for (unsigned b = 0; b < c.nblk; ++b) u += (double)__ldcg(bd.upart + (b0 + b) * bd.ustride + col);
    s_u[col] = u;
  }
  __syncthreads();
  float* v = bd.vvec + (int64_t)c.k * bd.ustride;
  for (int col = threadIdx.x; col < ldq; col += BT) {
    double a = 0.0;
    if (col < nr)
      for (int cc = 0; cc < nr; ++cc) a = fma((double)W[(int64_t)cc * nr + col], s_u[cc], a);
    v[col] = (float)a;
  }
}

// x = 0, r = b, |b|^2 and Q^T b -> instance state (zero rhs: done at once).
__global__ void __launch_bounds__(BT)
    batch_init_kernel(BatchDev bd, const double* __restrict__ B, double* __restrict__ X,
                      double* __restrict__ r) {
  __shared__ __align__(16) float s_w[NW][kMaxNr];
  __shared__ double s_red[BT / 32];
  __shared__ int s_go;
  const BlockCtx c = block_ctx(bd);
  double acc = 0.0;
  for (int64_t i = c.row0 + threadIdx.x; i < c.row1; i += BT) {
    const double bi = B[c.seg + i];
    r[c.seg + i] = bi;
    X[c.seg + i] = 0.0;
    acc = fma(bi, bi, acc);
  }
  double v[1] = {acc};
  block_sum<BT, 1>(v, s_red);
  if (threadIdx.x == 0) bd.bpart[c.g * 4] = v[0];
  if (bd.has_pc) project_block(bd, c, r, s_w);
  if (!arrive_last_of(&bd.ctr[c.k], c.nblk)) return;
  if (threadIdx.x == 0) {
    InstState s{};
    const double bn = sqrt(sum_blocks(bd, c, 0));
    s.bnorm = bn;
    s.tol_abs = bd.tol * bn;
    s.rnorm = s.rmax = s.true_rnorm = bn;
    bd.st[c.k] = s;
    s_go = 1;
    if (bn == 0.0) {
      finish_instance(bd, c.k, LAKER_OK);
      s_go = 0;
    } else if (!isfinite(bn)) {
      finish_instance(bd, c.k, LAKER_ERR_NONFINITE);
      s_go = 0;
    }
  }
  __syncthreads();
  if (s_go && bd.has_pc) w_multiply(bd, c, reinterpret_cast<double*>(&s_w[0][0]));
}

// z = c^-1/2 r + Q v (or r), r.z -> beta (rz seeded on init).
__global__ void __launch_bounds__(BT)
    batch_expand_kernel(BatchDev bd, const double* __restrict__ r, float* __restrict__ z, int init) {
  const BlockCtx c = block_ctx(bd);
  if (bd.st[c.k].done) return;
  __shared__ __align__(16) float s_v[kMaxNr];
  __shared__ double s_red[BT / 32];
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  double dot = 0.0;
  if (bd.has_pc) {
    const int ldq = bd.ldq[c.k], ldq4 = ldq >> 2;
    const float4* Q4 = reinterpret_cast<const float4*>(bd.q[c.k]);
    const float* vsrc = bd.vvec + (int64_t)c.k * bd.ustride;
    for (int col = tid; col < ldq; col += BT) s_v[col] = vsrc[col];
    __syncthreads();
    const float4* V4 = reinterpret_cast<const float4*>(s_v);
    const double cis = bd.cis[c.k];
    for (int64_t i = c.row0 + warp; i < c.row1; i += NW) {
      float s = 0.0f;
#pragma unroll
      for (int ch = 0; ch < 8; ++ch) {
        const int c4 = lane + 32 * ch;
        if (c4 < ldq4) {
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
        const double ri = r[c.seg + i];
        const float zi = (float)(cis * ri + (double)s);
        z[c.seg + i] = zi;
        dot = fma(ri, (double)zi, dot);
      }
    }
  } else {
    for (int64_t i = c.row0 + tid; i < c.row1; i += BT) {
      const double ri = r[c.seg + i];
      const float zi = (float)ri;
      z[c.seg + i] = zi;
      dot = fma(ri, (double)zi, dot);
    }
  }
  double v[1] = {dot};
  block_sum<BT, 1>(v, s_red);
  if (tid == 0) bd.bpart[c.g * 4] = v[0];
  if (!arrive_last_of(&bd.ctr[c.k], c.nblk)) return;
  if (tid == 0) {
    InstState& s = bd.st[c.k];
    const double rz = sum_blocks(bd, c, 0);
    if (init) {
      s.beta = 0.0;
    } else {
      s.beta = rz / s.rz;
    }
    s.rz = rz;
    if (!isfinite(rz)) finish_instance(bd, c.k, LAKER_ERR_NONFINITE);
  }
}

// p = z + beta p (p = z on init).
__global__ void __launch_bounds__(BT)
    batch_update_p_kernel(BatchDev bd, const float* __restrict__ z, float* __restrict__ p, int init) {
  const BlockCtx c = block_ctx(bd);
  if (bd.st[c.k].done) return;
  const float beta = (float)bd.st[c.k].beta;
  for (int64_t i = c.row0 + threadIdx.x; i < c.row1; i += BT) {
    const int64_t gi = c.seg + i;
    p[gi] = init ? z[gi] : fmaf(beta, p[gi], z[gi]);
  }
}

// Ap = lam p + (symmetric partials); p.Ap, p.p, Ap.Ap -> alpha or breakdown.
__global__ void __launch_bounds__(BT)
    batch_after_matvec_kernel(BatchDev bd, SymPlan sp, BatchMap bm,
                              const double* __restrict__ rowpart, const float* __restrict__ colpart,
                              const float* __restrict__ p, float* __restrict__ Ap) {
  const BlockCtx c = block_ctx(bd);
  if (bd.st[c.k].done) return;
  __shared__ double s_red[3 * (BT / 32)];
  const double lam = bd.lam[c.k];
  double d0 = 0.0, d1 = 0.0, d2 = 0.0;
  for (int64_t i = c.row0 + threadIdx.x; i < c.row1; i += BT) {
    const double pi = p[c.seg + i];
    const double a = lam * pi + sym_row_sum_batched(sp, bm, rowpart, colpart, c.k, i);
    const float af = (float)a;
    Ap[c.seg + i] = af;
    d0 = fma(pi, (double)af, d0);
    d1 = fma(pi, pi, d1);
    d2 = fma((double)af, (double)af, d2);
  }
  double v[3] = {d0, d1, d2};
  block_sum<BT, 3>(v, s_red);
  if (threadIdx.x == 0) {
    bd.bpart[c.g * 4 + 0] = v[0];
    bd.bpart[c.g * 4 + 1] = v[1];
    bd.bpart[c.g * 4 + 2] = v[2];
  }
  if (!arrive_last_of(&bd.ctr[c.k], c.nblk)) return;
  if (threadIdx.x == 0) {
    InstState& s = bd.st[c.k];
    const double pap = sum_blocks(bd, c, 0), pp = sum_blocks(bd, c, 1), aa = sum_blocks(bd, c, 2);
    if (!isfinite(pap) || !isfinite(pp) || !isfinite(aa)) {
      finish_instance(bd, c.k, LAKER_ERR_NONFINITE);
    } else if (pap <= -bd.eps * sqrt(pp) * sqrt(aa)) {
      finish_instance(bd, c.k, LAKER_ERR_BREAKDOWN);  // laker/solvers.py:232-246
    } else {
      s.alpha = s.rz / pap;
    }
  }
}

// x += alpha p; r -= alpha Ap; |r| -> reliable-update decision; Q^T r.
__global__ void __launch_bounds__(BT)
    batch_update_xr_kernel(BatchDev bd, const float* __restrict__ p, const float* __restrict__ Ap,
                           double* __restrict__ X, double* __restrict__ r) {
  const BlockCtx c = block_ctx(bd);
  if (bd.st[c.k].done) return;
  __shared__ __align__(16) float s_w[NW][kMaxNr];
  __shared__ double s_red[BT / 32];
  __shared__ int s_proj;
  const double alpha = bd.st[c.k].alpha;
  double rr = 0.0;
  for (int64_t i = c.row0 + threadIdx.x; i < c.row1; i += BT) {
    const int64_t gi = c.seg + i;
    X[gi] = fma(alpha, (double)p[gi], X[gi]);
    const double ri = fma(-alpha, (double)Ap[gi], r[gi]);
    r[gi] = ri;
    rr = fma(ri, ri, rr);
  }
  double v[1] = {rr};
  block_sum<BT, 1>(v, s_red);
  if (threadIdx.x == 0) bd.bpart[c.g * 4] = v[0];
  if (bd.has_pc) project_block(bd, c, r, s_w);
  if (!arrive_last_of(&bd.ctr[c.k], c.nblk)) return;
  if (threadIdx.x == 0) {
    InstState& s = bd.st[c.k];
    const double rn = sqrt(sum_blocks(bd, c, 0));
    s.rnorm = rn;
    s.iter += 1;
    // replace the residual once the recurrence has fallen by delta from its
    // peak since the last replacement (see laker_pcg_solve)
    if (rn > s.rmax) s.rmax = rn;
    s.need_update =
        (rn <= bd.delta * s.rmax || rn <= s.tol_abs || s.iter >= bd.max_iter || !isfinite(rn)) ? 1 : 0;
    s_proj = !s.need_update;
  }
  __syncthreads();
  if (s_proj && bd.has_pc) w_multiply(bd, c, reinterpret_cast<double*>(&s_w[0][0]));
}

// r = b - (lam x + K64 x) from the FP64 symmetric kernel's per-pair partial
// sums, for the blocks of instances whose need_update is set; then |r|^2,
// Q^T r and the stop test.
__global__ void __launch_bounds__(BT)
    batch_after_residual_kernel(BatchDev bd, SymPlan sp, BatchMap bm,
                                const double* __restrict__ rowpart, const double* __restrict__ colpart,
                                const double* __restrict__ B, const double* __restrict__ X,
                                double* __restrict__ r) {
  const BlockCtx c = block_ctx(bd);
  if (bd.st[c.k].done || !bd.st[c.k].need_update) return;
  __shared__ __align__(16) float s_w[NW][kMaxNr];
  __shared__ double s_red[BT / 32];
  __shared__ int s_go;
  const double lam = bd.lam[c.k];
  double rr = 0.0;
  for (int64_t i = c.row0 + threadIdx.x; i < c.row1; i += BT) {
    const int64_t gi = c.seg + i;
    const double ri = B[gi] - (lam * X[gi] + sym_row_sum_batched(sp, bm, rowpart, colpart, c.k, i));
    r[gi] = ri;
    rr = fma(ri, ri, rr);
  }
  double v[1] = {rr};
  block_sum<BT, 1>(v, s_red);
  if (threadIdx.x == 0) bd.bpart[c.g * 4] = v[0];
  if (bd.has_pc) project_block(bd, c, r, s_w);
  if (!arrive_last_of(&bd.ctr[c.k], c.nblk)) return;
  if (threadIdx.x == 0) {
    InstState& s = bd.st[c.k];
    const double rn = sqrt(sum_blocks(bd, c, 0));
    s.rnorm = s.true_rnorm = s.rmax = rn;
    s.n_accurate += 1;
    s.need_update = 0;
    s_go = 0;
    if (!isfinite(rn)) finish_instance(bd, c.k, LAKER_ERR_NONFINITE);
    else if (rn <= s.tol_abs) finish_instance(bd, c.k, LAKER_OK);
    else if (s.iter >= bd.max_iter) finish_instance(bd, c.k, LAKER_ERR_NOT_CONVERGED);
    else s_go = 1;
  }
  __syncthreads();
  if (s_go && bd.has_pc) w_multiply(bd, c, reinterpret_cast<double*>(&s_w[0][0]));
}

// Instance list for a batched matvec launch, in instance order: the running
// instances (need = 0; also refreshes the running count) or the running
// instances that asked for an FP64 residual (need = 1).  act_ps holds the
// exclusive prefix sums of their pair counts.  One CTA.
__global__ void __launch_bounds__(kCompactThreads)
    batch_compact_kernel(BatchDev bd, int need, int* __restrict__ act_inst,
                         int64_t* __restrict__ act_ps, int* __restrict__ act_count) {
  __shared__ long long s_p[kCompactThreads];
  __shared__ int s_c[kCompactThreads];
  const int tid = threadIdx.x;
  long long base_p = 0;
  int base_c = 0;
  for (int c0 = 0; c0 < bd.count; c0 += kCompactThreads) {
    const int k = c0 + tid;
    const bool act = k < bd.count && !bd.done[k] && (!need || bd.st[k].need_update);
    const long long np = act ? (long long)bd.nblk[k] * (bd.nblk[k] + 1) / 2 : 0;
    s_p[tid] = np;
    s_c[tid] = act ? 1 : 0;
    __syncthreads();
    for (int o = 1; o < kCompactThreads; o <<= 1) {  // inclusive scan
      const long long tp = tid >= o ? s_p[tid - o] : 0;
      const int tc = tid >= o ? s_c[tid - o] : 0;
      __syncthreads();
      s_p[tid] += tp;
      s_c[tid] += tc;
      __syncthreads();
    }
    if (act) {
      const int j = base_c + s_c[tid] - 1;
      act_inst[j] = k;
      act_ps[j] = base_p + s_p[tid] - np;
    }
    base_p += s_p[kCompactThreads - 1];
    base_c += s_c[kCompactThreads - 1];
    __syncthreads();
  }
  if (tid == 0) {
    act_ps[base_c] = base_p;
    *act_count = base_c;
    if (!need) *bd.active = base_c;
  }
}

// Host-side description of one batch solve (sizes and workspace carve-up).
struct BatchLayout {
  int count = 0;
  int ustride = 4;
  int64_t total = 0;  // padded points
  int64_t total_blocks = 0;
  int64_t total_pairs = 0;
  std::vector<int64_t> off, nblk, pair_start, blk_start;
  std::vector<int> blk_inst;
  SymPlan sp{}, sp64{};
  size_t bytes = 0;
  // byte offsets into the workspace
  size_t o_hdr, o_off, o_npts, o_nblk, o_ps, o_bs, o_binst, o_lam, o_q, o_w, o_nr, o_ldq, o_cis,
      o_st, o_done, o_active, o_ctr, o_actn, o_acti, o_actp, o_needn, o_needi, o_needp, o_bpart,
      o_upart, o_vvec, o_r, o_z, o_p, o_ap, o_rowpart, o_colpart, o_row64, o_col64;
};

BatchLayout make_layout(int count, const int64_t* n, int d, int max_ldq) {
  BatchLayout L;
  L.count = count;
  L.ustride = max_ldq > 4 ? (int)round_up(max_ldq, 4) : 4;
  const int B = sym_block_points();
  L.off.resize(count + 1);
  L.nblk.resize(count);
  L.pair_start.resize(count + 1);
  L.blk_start.resize(count + 1);
  L.off[0] = L.pair_start[0] = L.blk_start[0] = 0;
  for (int k = 0; k < count; ++k) {
    const int64_t nk = n[k] > 0 ? n[k] : 1;
    L.off[k + 1] = L.off[k] + round_up(nk, kBatchAlign);
    L.nblk[k] = ceil_div(nk, B);
    L.blk_start[k + 1] = L.blk_start[k] + L.nblk[k];
    L.pair_start[k + 1] = L.pair_start[k] + L.nblk[k] * (L.nblk[k] + 1) / 2;
  }
  L.total = L.off[count];
  L.total_blocks = L.blk_start[count];
  L.total_pairs = L.pair_start[count];
  L.blk_inst.resize(L.total_blocks);
  for (int k = 0; k < count; ++k)
    for (int64_t g = L.blk_start[k]; g < L.blk_start[k + 1]; ++g) L.blk_inst[g] = k;
  L.sp = k1s_plan_pairs(L.total_blocks, L.total_pairs, d);
  L.sp64 = k4s_plan_pairs(L.total_blocks, L.total_pairs, d);
  size_t o = 0;
  auto take = [&](size_t b) {
    const size_t at = o;
    o += (size_t)round_up((int64_t)(b ? b : 1), 256);
    return at;
  };
  const size_t c = (size_t)count, nbk = (size_t)L.total_blocks;
  L.o_hdr = take(kWsHeader);
  L.o_off = take((c + 1) * 8);
  L.o_npts = take(c * 8);
  L.o_nblk = take(c * 8);
  L.o_ps = take((c + 1) * 8);
  L.o_bs = take((c + 1) * 8);
  L.o_binst = take(nbk * 4);
  L.o_lam = take(c * 8);
  L.o_q = take(c * 8);
  L.o_w = take(c * 8);
  L.o_nr = take(c * 4);
  L.o_ldq = take(c * 4);
  L.o_cis = take(c * 8);
  L.o_st = take(c * sizeof(InstState));
  L.o_done = take(c * 4);
  L.o_active = take(4);
  L.o_ctr = take(c * 4);
  L.o_actn = take(4);
  L.o_acti = take(c * 4);
  L.o_actp = take((c + 1) * 8);
  L.o_needn = take(4);
  L.o_needi = take(c * 4);
  L.o_needp = take((c + 1) * 8);
  L.o_bpart = take(nbk * 4 * 8);
  L.o_upart = take(nbk * (size_t)L.ustride * 4);
  L.o_vvec = take(c * (size_t)L.ustride * 4);
  L.o_r = take((size_t)L.total * 8);
  L.o_z = take((size_t)L.total * 4);
  L.o_p = take((size_t)L.total * 4);
  L.o_ap = take((size_t)L.total * 4);
  L.o_rowpart = take(sym_rowpart_elems(L.sp) * 8);
  L.o_colpart = take(sym_colpart_elems(L.sp) * 4);
  L.o_row64 = take(sym_rowpart_elems(L.sp64) * 8);
  L.o_col64 = take(sym_colpart_elems(L.sp64) * 8);
  L.bytes = o;
  return L;
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

extern "C" size_t laker_pcg_batched_workspace_bytes(int count, const int64_t* n, int d, int max_nr) {
  if (count < 1 || !n || d < 1 || d > 16 || max_nr < 0 || max_nr > kMaxNr) return 0;
  for (int k = 0; k < count; ++k)
    if (n[k] < 1) return 0;
  return make_layout(count, n, d, max_nr).bytes;
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
  int max_ldq = 0;
  for (int k = 0; k < count; ++k) {
    if (batch->n[k] < 1) return LAKER_ERR_INVALID_ARG;
    if (batch->precond) {
      const laker_precond& pc = batch->precond[k];
      if (pc.n != batch->n[k] || pc.nr < 1 || pc.nr > kMaxNr || pc.ldq < pc.nr || pc.ldq > kMaxNr ||
          (pc.ldq % 4) || !pc.q_basis || !pc.w_core || (reinterpret_cast<uintptr_t>(pc.q_basis) % 16))
        return LAKER_ERR_INVALID_ARG;
      max_ldq = std::max(max_ldq, pc.ldq);
    }
  }
  const BatchLayout L = make_layout(count, batch->n, d, max_ldq);
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
  if (e == cudaSuccess) e = cudaMemsetAsync(at(L.o_done), 0, (size_t)count * 4, s);
  if (e == cudaSuccess) e = cudaMemsetAsync(at(L.o_ctr), 0, (size_t)count * 4, s);
  auto h2d = [&](size_t o, const void* src, size_t bytes) {
    if (e == cudaSuccess) e = cudaMemcpyAsync(at(o), src, bytes, cudaMemcpyHostToDevice, s);
  };
  h2d(L.o_off, L.off.data(), (count + 1) * 8);
  h2d(L.o_npts, npts.data(), count * 8);
  h2d(L.o_nblk, L.nblk.data(), count * 8);
  h2d(L.o_ps, L.pair_start.data(), (count + 1) * 8);
  h2d(L.o_bs, L.blk_start.data(), (count + 1) * 8);
  h2d(L.o_binst, L.blk_inst.data(), (size_t)L.total_blocks * 4);
  h2d(L.o_lam, lam.data(), count * 8);
  h2d(L.o_q, qp.data(), count * 8);
  h2d(L.o_w, wp.data(), count * 8);
  h2d(L.o_nr, nr.data(), count * 4);
  h2d(L.o_ldq, ldq.data(), count * 4);
  h2d(L.o_cis, cis.data(), count * 8);
  // the host vectors are pageable: finish the copies before they go out of scope
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  if (e != cudaSuccess) return fail_cuda(e);

  BatchDev bd{};
  bd.count = count;
  bd.has_pc = batch->precond ? 1 : 0;
  bd.max_iter = prm->max_iter;
  bd.ustride = L.ustride;
  bd.delta = prm->reliable_delta;
  bd.eps = prm->breakdown_eps;
  bd.tol = prm->tol;
  bd.off = static_cast<const int64_t*>(at(L.o_off));
  bd.npts = static_cast<const int64_t*>(at(L.o_npts));
  bd.nblk = static_cast<const int64_t*>(at(L.o_nblk));
  bd.blk_start = static_cast<const int64_t*>(at(L.o_bs));
  bd.blk_inst = static_cast<const int*>(at(L.o_binst));
  bd.lam = static_cast<const double*>(at(L.o_lam));
  bd.q = static_cast<const uint64_t*>(at(L.o_q));
  bd.w = static_cast<const uint64_t*>(at(L.o_w));
  bd.nr = static_cast<const int*>(at(L.o_nr));
  bd.ldq = static_cast<const int*>(at(L.o_ldq));
  bd.cis = static_cast<const double*>(at(L.o_cis));
  bd.st = static_cast<InstState*>(at(L.o_st));
  bd.done = static_cast<int*>(at(L.o_done));
  bd.active = static_cast<int*>(at(L.o_active));
  bd.ctr = static_cast<unsigned int*>(at(L.o_ctr));
  bd.bpart = static_cast<double*>(at(L.o_bpart));
  bd.upart = static_cast<float*>(at(L.o_upart));
  bd.vvec = static_cast<float*>(at(L.o_vvec));

  int* act_count = static_cast<int*>(at(L.o_actn));
  int* act_inst = static_cast<int*>(at(L.o_acti));
  int64_t* act_ps = static_cast<int64_t*>(at(L.o_actp));
  BatchMap bm{};
  bm.count = count;
  bm.pair_start = static_cast<const int64_t*>(at(L.o_ps));
  bm.nblk = bd.nblk;
  bm.npts = bd.npts;
  bm.seg = bd.off;
  bm.blk_start = bd.blk_start;
  bm.act_count = act_count;
  bm.act_inst = act_inst;
  bm.act_ps = act_ps;
  int* need_count = static_cast<int*>(at(L.o_needn));
  int* need_inst = static_cast<int*>(at(L.o_needi));
  int64_t* need_ps = static_cast<int64_t*>(at(L.o_needp));
  BatchMap bm64 = bm;
  bm64.act_count = need_count;
  bm64.act_inst = need_inst;
  bm64.act_ps = need_ps;
  double* row64 = static_cast<double*>(at(L.o_row64));
  double* col64 = static_cast<double*>(at(L.o_col64));

  double* r = static_cast<double*>(at(L.o_r));
  float* z = static_cast<float*>(at(L.o_z));
  float* p = static_cast<float*>(at(L.o_p));
  float* Ap = static_cast<float*>(at(L.o_ap));
  double* rowpart = static_cast<double*>(at(L.o_rowpart));
  float* colpart = static_cast<float*>(at(L.o_colpart));
  int* dstatus = &static_cast<WsHeader*>(at(L.o_hdr))->status;
  const unsigned nblocks = (unsigned)L.total_blocks;

  int launches = 0;
  // ---- initialisation (plain launches on the caller's stream) ----------------
  batch_init_kernel<<<nblocks, BT, 0, s>>>(bd, B, X, r);
  batch_expand_kernel<<<nblocks, BT, 0, s>>>(bd, r, z, 1);
  batch_update_p_kernel<<<nblocks, BT, 0, s>>>(bd, z, p, 1);
  batch_compact_kernel<<<1, kCompactThreads, 0, s>>>(bd, 0, act_inst, act_ps, act_count);
  launches += 4;
  e = cudaGetLastError();
  if (e != cudaSuccess) return fail_cuda(e);

  // ---- one iteration, captured once as a graph --------------------------------
  auto iteration = [&](cudaStream_t cs) -> cudaError_t {
    cudaError_t ee = launch_k1s_batched(batch->packed32, d, batch->clamp, p, rowpart, colpart, L.sp,
                                        bm, dstatus, bd.active, cs);
    if (ee != cudaSuccess) return ee;
    batch_after_matvec_kernel<<<nblocks, BT, 0, cs>>>(bd, L.sp, bm, rowpart, colpart, p, Ap);
    batch_update_xr_kernel<<<nblocks, BT, 0, cs>>>(bd, p, Ap, X, r);
    batch_compact_kernel<<<1, kCompactThreads, 0, cs>>>(bd, 1, need_inst, need_ps, need_count);
    ee = launch_k4s_batched(batch->packed64, d, batch->clamp, X, row64, col64, L.sp64, bm64,
                            dstatus, need_count, cs);
    if (ee != cudaSuccess) return ee;
    batch_after_residual_kernel<<<nblocks, BT, 0, cs>>>(bd, L.sp64, bm, row64, col64, B, X, r);
    batch_expand_kernel<<<nblocks, BT, 0, cs>>>(bd, r, z, 0);
    batch_update_p_kernel<<<nblocks, BT, 0, cs>>>(bd, z, p, 0);
    batch_compact_kernel<<<1, kCompactThreads, 0, cs>>>(bd, 0, act_inst, act_ps, act_count);
    return cudaGetLastError();
  };
  constexpr int kLaunchesPerIter = 9;
  int chunk = prm->check_every > 0 ? prm->check_every : 8;
  if (chunk > prm->max_iter && prm->max_iter > 0) chunk = prm->max_iter;

  cudaStream_t cs = nullptr;
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  int active = count;
  if (prm->max_iter > 0) {
    e = cudaStreamCreateWithFlags(&cs, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaStreamBeginCapture(cs, cudaStreamCaptureModeThreadLocal);
    if (e == cudaSuccess) {
      cudaError_t ce = cudaSuccess;
      for (int it = 0; it < chunk && ce == cudaSuccess; ++it) ce = iteration(cs);
      e = cudaStreamEndCapture(cs, &graph);
      if (e == cudaSuccess) e = ce;
    }
    if (e == cudaSuccess) e = cudaGraphInstantiate(&exec, graph, 0);
  }
  int iters_launched = 0;
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
