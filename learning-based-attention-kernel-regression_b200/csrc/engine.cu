// Solve engine: many independent mixed-precision PCG solves in one device loop,
// with instances admitted and collected between graph replays.
//
// Layout.  The workspace holds capacity-sized arenas: points (packed
// embeddings, b, x, r, z, p, Ap), 512-point blocks (one per 512 points), block
// pairs (the partial sums of the symmetric matvecs) and slots (per-instance
// record, state and lists).  Slot k's instance occupies points [seg, seg +
// round_up(n, 512)), blocks blk_start .. + nblk - 1 and pairs pair_start .. +
// nblk (nblk + 1) / 2 - 1 (SlotInfo); blk_inst maps a block to its slot (-1:
// free).  Space is handed out from the bottom of each arena; when a new
// instance does not fit above the top, the resident ones are moved down
// (points arrays only: the block and pair scratch is rewritten every
// iteration).
//
// One iteration, captured once as a CUDA graph and replayed by the host:
//   matvec     part = K32 p over the block pairs of the running instances
//              (list compacted on the device, split evenly over the grid)
//   after_mv   [block] Ap = lam p + partial sums; p.Ap, p.p, Ap.Ap
//              [last block of the instance] alpha, or breakdown
//   update_xr  [block] x += alpha p; r -= alpha Ap; |r|^2; Q_blk^T r
//              [last] reliable-update decision; v = W Q^T r unless a residual follows
//   need list  the running instances that asked for an FP64 residual
//   residual   K64 x over their block pairs (FP64 symmetric kernel), then
//              [block] r = b - lam x - partial sums; |r|^2; Q_blk^T r
//              [last] stop test; v = W Q^T r
//   expand     [block] z = c r + Q_blk v; r.z        [last] beta
//   update_p   [block] p = z + beta p
//   run list   running-instance list and pair prefix sums for the next matvec
// The block kernels are persistent: a fixed grid walks the blocks in use.
// The recurrence is the one of laker_pcg_solve (laker/solvers.py:189-295 with
// FP64 residual replacement).  Block partials are added by the instance's last
// block in block order and the matvecs' partial sums are per block pair, so an
// instance's arithmetic does not depend on where it sits or on the other
// instances: the same bits alone or in any mix.
#include <algorithm>
#include <type_traits>
#include <cstring>
#include <vector>

#include "pcg_state.cuh"
#include "sym.cuh"

namespace laker {
namespace {

constexpr int BT = 256;           // threads of the block kernels
constexpr int NW = BT / 32;
constexpr int RB = 512;           // points per block (the symmetric matvecs' blocks)
constexpr int kCompactThreads = 1024;
constexpr uint64_t kEngineMagic = 0x4c414b4552454e47ull;  // "LAKERENG"
static_assert(RB == 2 * BT, "two rows per thread in the block kernels");

struct InstState {
  double bnorm, tol_abs, rz, alpha, beta, rnorm, rmax, true_rnorm;
  int iter, n_accurate, done, status, need_update, pad0;
};

struct EngineDev {
  int max_slots;
  int max_iter;
  int ustride;              // floats per projection vector (>= every ldq)
  double delta, eps, tol;
  const SlotInfo* slots;    // [max_slots]
  const int* blk_inst;      // [blocks] slot of a block, -1: free
  const int64_t* nb_used;   // blocks in use (the persistent kernels' range)
  InstState* st;            // [max_slots]
  int* done;                // [max_slots] 1: not iterating (stopped or free)
  int* active;              // running instances (host poll, matvec gate)
  unsigned int* ctr;        // [max_slots] block arrival counters
  double* bpart;            // [blocks * 4] block partial scalars
  float* upart;             // [blocks * ustride] block partials of Q^T r
  float* vvec;              // [max_slots * ustride] v = W Q^T r
};

struct BlockCtx {
  int64_t g;      // block
  int k;          // slot
  unsigned nblk;  // blocks of the instance
  int64_t b0, seg, n, row0, row1;
};

__device__ __forceinline__ BlockCtx block_ctx(const EngineDev& ed, int64_t g, int k) {
  const SlotInfo& si = ed.slots[k];
  BlockCtx c;
  c.g = g;
  c.k = k;
  c.b0 = si.blk_start;
  c.nblk = (unsigned)si.nblk;
  c.seg = si.seg;
  c.n = si.npts;
  c.row0 = (g - c.b0) * RB;
  c.row1 = c.row0 + RB < c.n ? c.row0 + RB : c.n;
  return c;
}

// Range of blocks a persistent block kernel walks: [g_begin, g_end), or up to
// the blocks in use when g_end < 0.
__device__ __forceinline__ int64_t range_end(const EngineDev& ed, int64_t g_end) {
  return g_end >= 0 ? g_end : *ed.nb_used;
}

__device__ __forceinline__ void finish_instance(const EngineDev& ed, int k, int status) {
  ed.st[k].status = status;
  ed.st[k].done = 1;
  ed.done[k] = 1;
}

// Sum of slot j of the instance's block partials, in block order.
__device__ __forceinline__ double sum_blocks(const EngineDev& ed, const BlockCtx& c, int j) {
  double t = 0.0;
  for (unsigned b = 0; b < c.nblk; ++b) t += __ldcg(ed.bpart + (c.b0 + b) * 4 + j);
  return t;
}

// upart[g][col] = sum over the block's rows i of Q[i][col] * r_i.  Warps take
// rows; lane l holds the float4 column chunks l + 32 ch.  Caller has
// synchronised after writing r.
__device__ void project_block(const EngineDev& ed, const BlockCtx& c, const double* __restrict__ r,
                              float (*s_w)[kMaxNr]) {
  const SlotInfo& si = ed.slots[c.k];
  const float4* Q4 = reinterpret_cast<const float4*>(si.q);
  const int ldq = si.ldq, ldq4 = ldq >> 2;
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
  float* dst = ed.upart + c.g * ed.ustride;
  for (int col = threadIdx.x; col < ldq; col += BT) {
    float s = 0.0f;
#pragma unroll
    for (int w2 = 0; w2 < NW; ++w2) s += s_w[w2][col];
    dst[col] = s;
  }
}

// Last block of an instance: u = sum of the block projections, v = W u ->
// vvec[k].  Both sums run as four interleaved partial sums (index mod 4)
// combined in a fixed order, so that four loads are in flight per thread
// instead of one dependent chain; the result depends only on the instance.
// s_u may alias the projection scratch (the arrival barrier separates the two
// uses).
__device__ void w_multiply(const EngineDev& ed, const BlockCtx& c, double* s_u) {
  const SlotInfo& si = ed.slots[c.k];
  const int nr = si.nr, ldq = si.ldq;
  const float* W = reinterpret_cast<const float*>(si.w);
  for (int col = threadIdx.x; col < nr; col += BT) {
    const float* up = ed.upart + c.b0 * ed.ustride + col;
    double u0 = 0.0, u1 = 0.0, u2 = 0.0, u3 = 0.0;
    unsigned b = 0;
    // 16 loads issued before their adds (same partial sums, same order)
    for (; b + 16 <= c.nblk; b += 16) {
      float t[16];
#pragma unroll
      for (int e = 0; e < 16; ++e) t[e] = __ldcg(up + (int64_t)(b + e) * ed.ustride);
#pragma unroll
      for (int e = 0; e < 16; e += 4) {
        u0 += (double)t[e];
        u1 += (double)t[e + 1];
        u2 += (double)t[e + 2];
        u3 += (double)t[e + 3];
      }
    }
    for (; b + 4 <= c.nblk; b += 4) {
      u0 += (double)__ldcg(up + (int64_t)b * ed.ustride);
      u1 += (double)__ldcg(up + (int64_t)(b + 1) * ed.ustride);
      u2 += (double)__ldcg(up + (int64_t)(b + 2) * ed.ustride);
      u3 += (double)__ldcg(up + (int64_t)(b + 3) * ed.ustride);
    }
    for (; b < c.nblk; ++b) u0 += (double)__ldcg(up + (int64_t)b * ed.ustride);
    s_u[col] = (u0 + u1) + (u2 + u3);
  }
  __syncthreads();
  float* v = ed.vvec + (int64_t)c.k * ed.ustride;
  for (int col = threadIdx.x; col < ldq; col += BT) {
    double a0 = 0.0, a1 = 0.0, a2 = 0.0, a3 = 0.0;
    if (col < nr) {
      const float* wc = W + col;
      int cc = 0;
      // 16 loads of W issued before their FMAs (same partial sums, same order)
      for (; cc + 16 <= nr; cc += 16) {
        float t[16];
#pragma unroll
        for (int e = 0; e < 16; ++e) t[e] = __ldg(wc + (int64_t)(cc + e) * nr);
#pragma unroll
        for (int e = 0; e < 16; e += 4) {
          a0 = fma((double)t[e], s_u[cc + e], a0);
          a1 = fma((double)t[e + 1], s_u[cc + e + 1], a1);
          a2 = fma((double)t[e + 2], s_u[cc + e + 2], a2);
          a3 = fma((double)t[e + 3], s_u[cc + e + 3], a3);
        }
      }
      for (; cc + 4 <= nr; cc += 4) {
        a0 = fma((double)wc[(int64_t)cc * nr], s_u[cc], a0);
        a1 = fma((double)wc[(int64_t)(cc + 1) * nr], s_u[cc + 1], a1);
        a2 = fma((double)wc[(int64_t)(cc + 2) * nr], s_u[cc + 2], a2);
        a3 = fma((double)wc[(int64_t)(cc + 3) * nr], s_u[cc + 3], a3);
      }
      for (; cc < nr; ++cc) a0 = fma((double)wc[(int64_t)cc * nr], s_u[cc], a0);
    }
    v[col] = (float)((a0 + a1) + (a2 + a3));
  }
}

// Places slot k (record, blocks in use); `reset` also clears its state for a
// new instance.  One thread.
__global__ void eng_place_kernel(EngineDev ed, SlotInfo* slots, int64_t* nb_used, int k,
                                 SlotInfo info, int64_t new_nb_used, int reset) {
  slots[k] = info;
  *nb_used = new_nb_used;
  if (reset) {
    ed.st[k] = InstState{};
    ed.done[k] = 0;
    ed.ctr[k] = 0;
  }
}

__global__ void eng_fill_int_kernel(int* __restrict__ a, int64_t begin, int64_t end, int v) {
  for (int64_t i = begin + blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < end;
       i += (int64_t)gridDim.x * blockDim.x)
    a[i] = v;
}

__global__ void eng_set_i64_kernel(int64_t* p, int64_t v) { *p = v; }

// x = 0, r = b, |b|^2 and Q^T b -> instance state (zero rhs: done at once).
__global__ void __launch_bounds__(BT)
    eng_init_kernel(EngineDev ed, int64_t g_begin, int64_t g_end, const double* __restrict__ B,
                    double* __restrict__ X, double* __restrict__ r) {
  __shared__ __align__(16) float s_w[NW][kMaxNr];
  __shared__ double s_red[BT / 32];
  __shared__ int s_go;
  const int64_t ge = range_end(ed, g_end);
  for (int64_t g = g_begin + blockIdx.x; g < ge; g += gridDim.x) {
    const int k = ed.blk_inst[g];
    if (k < 0) continue;
    const BlockCtx c = block_ctx(ed, g, k);
    const bool hp = ed.slots[k].q != 0;
    double acc = 0.0;
    for (int64_t i = c.row0 + threadIdx.x; i < c.row1; i += BT) {
      const double bi = B[c.seg + i];
      r[c.seg + i] = bi;
      X[c.seg + i] = 0.0;
      acc = fma(bi, bi, acc);
    }
    double v[1] = {acc};
    block_sum<BT, 1>(v, s_red);
    if (threadIdx.x == 0) ed.bpart[c.g * 4] = v[0];
    if (hp) project_block(ed, c, r, s_w);
    if (arrive_last_of(&ed.ctr[c.k], c.nblk)) {
      if (threadIdx.x == 0) {
        InstState s{};
        const double bn = sqrt(sum_blocks(ed, c, 0));
        s.bnorm = bn;
        s.tol_abs = ed.tol * bn;
        s.rnorm = s.rmax = s.true_rnorm = bn;
        ed.st[c.k] = s;
        s_go = 1;
        if (bn == 0.0) {
          finish_instance(ed, c.k, LAKER_OK);
          s_go = 0;
        } else if (!isfinite(bn)) {
          finish_instance(ed, c.k, LAKER_ERR_NONFINITE);
          s_go = 0;
        }
      }
      __syncthreads();
      if (s_go && hp) w_multiply(ed, c, reinterpret_cast<double*>(&s_w[0][0]));
    }
    __syncthreads();  // shared scratch is reused by the next block
  }
}

// z = c^-1/2 r + Q v (or r), r.z -> beta (rz seeded on init).
__global__ void __launch_bounds__(BT)
    eng_expand_kernel(EngineDev ed, int64_t g_begin, int64_t g_end, const double* __restrict__ r,
                      float* __restrict__ z, int init) {
  __shared__ __align__(16) float s_v[kMaxNr];
  __shared__ double s_red[BT / 32];
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int64_t ge = range_end(ed, g_end);
  for (int64_t g = g_begin + blockIdx.x; g < ge; g += gridDim.x) {
    const int k = ed.blk_inst[g];
    if (k < 0 || ed.st[k].done) continue;
    const BlockCtx c = block_ctx(ed, g, k);
    const SlotInfo& si = ed.slots[k];
    double dot = 0.0;
    if (si.q != 0) {
      const int ldq = si.ldq, ldq4 = ldq >> 2;
      const float4* Q4 = reinterpret_cast<const float4*>(si.q);
      const float* vsrc = ed.vvec + (int64_t)k * ed.ustride;
      for (int col = tid; col < ldq; col += BT) s_v[col] = vsrc[col];
      __syncthreads();
      const float4* V4 = reinterpret_cast<const float4*>(s_v);
      const double cis = si.cis;
      // rows of Q in groups of LPR lanes (8, 16 or 32 by the row's width):
      // a warp takes 32 / LPR rows at a time and reduces within the group
      auto rows = [&](auto lpr_tag) {
        constexpr int LPR = decltype(lpr_tag)::value;
        constexpr int RPW = 32 / LPR;
        const int sub = lane / LPR, sl = lane % LPR;
        for (int64_t i0 = c.row0 + (int64_t)warp * RPW; i0 < c.row1; i0 += (int64_t)NW * RPW) {
          const int64_t i = i0 + sub;
          float s = 0.0f;
          if (i < c.row1) {
            for (int c4 = sl; c4 < ldq4; c4 += LPR) {
              const float4 q = __ldg(Q4 + i * ldq4 + c4);
              const float4 vv = V4[c4];
              s = fmaf(q.x, vv.x, s);
              s = fmaf(q.y, vv.y, s);
              s = fmaf(q.z, vv.z, s);
              s = fmaf(q.w, vv.w, s);
            }
          }
#pragma unroll
          for (int o = LPR / 2; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
          if (sl == 0 && i < c.row1) {
            const double ri = r[c.seg + i];
            const float zi = (float)(cis * ri + (double)s);
            z[c.seg + i] = zi;
            dot = fma(ri, (double)zi, dot);
          }
        }
      };
      if (ldq4 <= 64)
        rows(std::integral_constant<int, 8>{});
      else if (ldq4 <= 128)
        rows(std::integral_constant<int, 16>{});
      else
        rows(std::integral_constant<int, 32>{});
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
    if (tid == 0) ed.bpart[c.g * 4] = v[0];
    if (arrive_last_of(&ed.ctr[c.k], c.nblk) && tid == 0) {
      InstState& s = ed.st[c.k];
      const double rz = sum_blocks(ed, c, 0);
      s.beta = init ? 0.0 : rz / s.rz;
      s.rz = rz;
      if (!isfinite(rz)) finish_instance(ed, c.k, LAKER_ERR_NONFINITE);
    }
    __syncthreads();
  }
}

// p = z + beta p (p = z on init).
__global__ void __launch_bounds__(BT)
    eng_update_p_kernel(EngineDev ed, int64_t g_begin, int64_t g_end, const float* __restrict__ z,
                        float* __restrict__ p, int init) {
  const int64_t ge = range_end(ed, g_end);
  for (int64_t g = g_begin + blockIdx.x; g < ge; g += gridDim.x) {
    const int k = ed.blk_inst[g];
    if (k < 0 || ed.st[k].done) continue;
    const BlockCtx c = block_ctx(ed, g, k);
    const float beta = (float)ed.st[k].beta;
    for (int64_t i = c.row0 + threadIdx.x; i < c.row1; i += BT) {
      const int64_t gi = c.seg + i;
      p[gi] = init ? z[gi] : fmaf(beta, p[gi], z[gi]);
    }
  }
}

// Ap = lam p + (symmetric partials); p.Ap, p.p, Ap.Ap -> alpha or breakdown.
__global__ void __launch_bounds__(BT)
    eng_after_matvec_kernel(EngineDev ed, SymPlan sp, BatchMap bm,
                            const double* __restrict__ rowpart, const float* __restrict__ colpart,
                            const float* __restrict__ p, float* __restrict__ Ap) {
  __shared__ double s_red[3 * (BT / 32)];
  const int64_t ge = *ed.nb_used;
  for (int64_t g = blockIdx.x; g < ge; g += gridDim.x) {
    const int k = ed.blk_inst[g];
    if (k < 0 || ed.st[k].done) continue;
    const BlockCtx c = block_ctx(ed, g, k);
    const double lam = ed.slots[k].lam;
    double d0 = 0.0, d1 = 0.0, d2 = 0.0;
    for (int64_t i = c.row0 + threadIdx.x; i < c.row1; i += BT) {
      const double pi = p[c.seg + i];
      const double a = lam * pi + sym_row_sum_batched(sp, bm, rowpart, colpart, k, i);
      const float af = (float)a;
      Ap[c.seg + i] = af;
      d0 = fma(pi, (double)af, d0);
      d1 = fma(pi, pi, d1);
      d2 = fma((double)af, (double)af, d2);
    }
    double v[3] = {d0, d1, d2};
    block_sum<BT, 3>(v, s_red);
    if (threadIdx.x == 0) {
      ed.bpart[c.g * 4 + 0] = v[0];
      ed.bpart[c.g * 4 + 1] = v[1];
      ed.bpart[c.g * 4 + 2] = v[2];
    }
    if (arrive_last_of(&ed.ctr[c.k], c.nblk) && threadIdx.x == 0) {
      InstState& s = ed.st[c.k];
      const double pap = sum_blocks(ed, c, 0), pp = sum_blocks(ed, c, 1), aa = sum_blocks(ed, c, 2);
      if (!isfinite(pap) || !isfinite(pp) || !isfinite(aa)) {
        finish_instance(ed, c.k, LAKER_ERR_NONFINITE);
      } else if (pap <= -ed.eps * sqrt(pp) * sqrt(aa)) {
        finish_instance(ed, c.k, LAKER_ERR_BREAKDOWN);  // laker/solvers.py:232-246
      } else {
        s.alpha = s.rz / pap;
      }
    }
    __syncthreads();
  }
}

// x += alpha p; r -= alpha Ap; |r| -> reliable-update decision; Q^T r.
__global__ void __launch_bounds__(BT)
    eng_update_xr_kernel(EngineDev ed, const float* __restrict__ p, const float* __restrict__ Ap,
                         double* __restrict__ X, double* __restrict__ r) {
  __shared__ __align__(16) float s_w[NW][kMaxNr];
  __shared__ double s_red[BT / 32];
  __shared__ int s_proj;
  const int64_t ge = *ed.nb_used;
  for (int64_t g = blockIdx.x; g < ge; g += gridDim.x) {
    const int k = ed.blk_inst[g];
    if (k < 0 || ed.st[k].done) continue;
    const BlockCtx c = block_ctx(ed, g, k);
    const bool hp = ed.slots[k].q != 0;
    const double alpha = ed.st[k].alpha;
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
    if (threadIdx.x == 0) ed.bpart[c.g * 4] = v[0];
    if (hp) project_block(ed, c, r, s_w);
    if (arrive_last_of(&ed.ctr[c.k], c.nblk)) {
      if (threadIdx.x == 0) {
        InstState& s = ed.st[c.k];
        const double rn = sqrt(sum_blocks(ed, c, 0));
        s.rnorm = rn;
        s.iter += 1;
        // replace the residual once the recurrence has fallen by delta from
        // its peak since the last replacement (see laker_pcg_solve)
        if (rn > s.rmax) s.rmax = rn;
        s.need_update =
            (rn <= ed.delta * s.rmax || rn <= s.tol_abs || s.iter >= ed.max_iter || !isfinite(rn)) ? 1 : 0;
        s_proj = !s.need_update;
      }
      __syncthreads();
      if (s_proj && hp) w_multiply(ed, c, reinterpret_cast<double*>(&s_w[0][0]));
    }
    __syncthreads();
  }
}

// r = b - (lam x + K64 x) from the FP64 symmetric kernel's per-pair partial
// sums, for the blocks of instances whose need_update is set; then |r|^2,
// Q^T r and the stop test.
__global__ void __launch_bounds__(BT)
    eng_after_residual_kernel(EngineDev ed, SymPlan sp, BatchMap bm,
                              const double* __restrict__ rowpart, const double* __restrict__ colpart,
                              const double* __restrict__ B, const double* __restrict__ X,
                              double* __restrict__ r) {
  __shared__ __align__(16) float s_w[NW][kMaxNr];
  __shared__ double s_red[BT / 32];
  __shared__ int s_go;
  const int64_t ge = *ed.nb_used;
  for (int64_t g = blockIdx.x; g < ge; g += gridDim.x) {
    const int k = ed.blk_inst[g];
    if (k < 0 || ed.st[k].done || !ed.st[k].need_update) continue;
    const BlockCtx c = block_ctx(ed, g, k);
    const bool hp = ed.slots[k].q != 0;
    const double lam = ed.slots[k].lam;
    double rr = 0.0;
    for (int64_t i = c.row0 + threadIdx.x; i < c.row1; i += BT) {
      const int64_t gi = c.seg + i;
      const double ri = B[gi] - (lam * X[gi] + sym_row_sum_batched(sp, bm, rowpart, colpart, k, i));
      r[gi] = ri;
      rr = fma(ri, ri, rr);
    }
    double v[1] = {rr};
    block_sum<BT, 1>(v, s_red);
    if (threadIdx.x == 0) ed.bpart[c.g * 4] = v[0];
    if (hp) project_block(ed, c, r, s_w);
    if (arrive_last_of(&ed.ctr[c.k], c.nblk)) {
      if (threadIdx.x == 0) {
        InstState& s = ed.st[c.k];
        const double rn = sqrt(sum_blocks(ed, c, 0));
        s.rnorm = s.true_rnorm = s.rmax = rn;
        s.n_accurate += 1;
        s.need_update = 0;
        s_go = 0;
        if (!isfinite(rn)) finish_instance(ed, c.k, LAKER_ERR_NONFINITE);
        else if (rn <= s.tol_abs) finish_instance(ed, c.k, LAKER_OK);
        else if (s.iter >= ed.max_iter) finish_instance(ed, c.k, LAKER_ERR_NOT_CONVERGED);
        else s_go = 1;
      }
      __syncthreads();
      if (s_go && hp) w_multiply(ed, c, reinterpret_cast<double*>(&s_w[0][0]));
    }
    __syncthreads();
  }
}

// Instance list for a batched matvec launch, in slot order: the running
// instances (need = 0; also refreshes the running count) or the running
// instances that asked for an FP64 residual (need = 1).  act_ps holds the
// exclusive prefix sums of their pair counts.  One CTA.
__global__ void __launch_bounds__(kCompactThreads)
    eng_compact_kernel(EngineDev ed, int need, int* __restrict__ act_inst,
                       int64_t* __restrict__ act_ps, int* __restrict__ act_count) {
  __shared__ long long s_p[kCompactThreads];
  __shared__ int s_c[kCompactThreads];
  const int tid = threadIdx.x;
  long long base_p = 0;
  int base_c = 0;
  for (int c0 = 0; c0 < ed.max_slots; c0 += kCompactThreads) {
    const int k = c0 + tid;
    const bool act = k < ed.max_slots && !ed.done[k] && (!need || ed.st[k].need_update);
    const long long nb = act ? (long long)ed.slots[k].nblk : 0;
    const long long np = nb * (nb + 1) / 2;
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
    if (!need) *ed.active = base_c;
  }
}

// ---- host side ------------------------------------------------------------------
struct EngineLayout {
  int64_t cap_points = 0, cap_blocks = 0, cap_pairs = 0;
  int slots = 0, ustride = 4, dp = 2;
  bool tc = false;  // FP32 operator on the tensor cores (operand image arena)
  int fmt = 0;      // its image format (k1t_format at init), for every pack and launch
  size_t bytes = 0;
  size_t o_img = 0;
  size_t o_hdr, o_slots, o_st, o_done, o_ctr, o_scal, o_acti, o_actp, o_needi, o_needp, o_vvec,
      o_binst, o_bpart, o_upart, o_p32, o_p64, o_b, o_x, o_r, o_z, o_p, o_ap, o_row32, o_col32,
      o_row64, o_col64;
};

EngineLayout engine_layout(const laker_engine_config& cfg) {
  EngineLayout L;
  L.slots = cfg.max_slots;
  L.cap_points = round_up(cfg.max_points, RB);
  L.cap_blocks = L.cap_points / RB;
  L.cap_pairs = cfg.max_pairs;
  L.ustride = cfg.max_nr > 4 ? (int)round_up(cfg.max_nr, 4) : 4;
  L.dp = padded_dim(cfg.d);
  size_t o = 0;
  auto take = [&](size_t b) {
    const size_t at = o;
    o += (size_t)round_up((int64_t)(b ? b : 1), 256);
    return at;
  };
  const size_t S = (size_t)L.slots, CB = (size_t)L.cap_blocks, CP = (size_t)L.cap_points,
               PP = (size_t)L.cap_pairs * RB;
  L.o_hdr = take(kWsHeader);
  L.o_slots = take(S * sizeof(SlotInfo));
  L.o_st = take(S * sizeof(InstState));
  L.o_done = take(S * 4);
  L.o_ctr = take(S * 4);
  L.o_scal = take(64);  // active, act_count, need_count, nb_used
  L.o_acti = take(S * 4);
  L.o_actp = take((S + 1) * 8);
  L.o_needi = take(S * 4);
  L.o_needp = take((S + 1) * 8);
  L.o_vvec = take(S * (size_t)L.ustride * 4);
  L.o_binst = take(CB * 4);
  L.o_bpart = take(CB * 4 * 8);
  L.o_upart = take(CB * (size_t)L.ustride * 4);
  L.o_p32 = take(CP * L.dp * 4);
  L.o_p64 = take(CP * L.dp * 8);
  L.o_b = take(CP * 8);
  L.o_x = take(CP * 8);
  L.o_r = take(CP * 8);
  L.o_z = take(CP * 4);
  L.o_p = take(CP * 4);
  L.o_ap = take(CP * 4);
  L.o_row32 = take(PP * 8);
  L.o_col32 = take(PP * 4);
  L.o_row64 = take(PP * 8);
  L.o_col64 = take(PP * 8);
  L.tc = k1t_enabled(cfg.d);
  L.fmt = k1t_format(cfg.clamp, cfg.d);
  if (L.tc) L.o_img = take(k1t_image_bytes(L.cap_points));
  L.bytes = o;
  return L;
}

enum SlotState { kFree = 0, kRunning = 1, kStopped = 2 };

struct SlotHost {
  int state;
  SlotInfo info;
};

struct EngineHost {
  uint64_t magic;
  laker_engine_config cfg;
  laker_pcg_params prm;
  EngineLayout L;
  char* base;  // device workspace
  cudaStream_t stream, cap;
  cudaGraph_t graph;
  cudaGraphExec_t exec;
  SymPlan sp32, sp64;
  int block_grid;
  int running;
  int launched;      // a replay is in flight (laker_engine_launch)
  int readback[2];   // running count, device status of the last replay
  int64_t nb_used, pairs_used;
  SlotHost* slots;  // [max_slots], in the host buffer after this struct
  int* done_h;      // [max_slots]
  EngineDev ed;
  BatchMap bm32, bm64;

  template <typename T>
  T* at(size_t o) const {
    return reinterpret_cast<T*>(base + o);
  }
};

size_t host_bytes_for(int slots) {
  return (size_t)round_up((int64_t)sizeof(EngineHost), 64) +
         (size_t)slots * (sizeof(SlotHost) + sizeof(int)) + 64;
}

bool config_valid(const laker_engine_config* cfg) {
  return cfg && cfg->max_slots >= 1 && cfg->max_points >= 1 && cfg->max_pairs >= 1 && cfg->d >= 1 &&
         cfg->d <= 16 && cfg->max_nr >= 0 && cfg->max_nr <= kMaxNr && cfg->chunk >= 1;
}

EngineHost* engine_of(void* host) {
  EngineHost* e = static_cast<EngineHost*>(host);
  return (e && e->magic == kEngineMagic) ? e : nullptr;
}

// One iteration of every running instance (the graph body).
cudaError_t engine_iteration(EngineHost* e, cudaStream_t cs) {
  const EngineLayout& L = e->L;
  const EngineDev& ed = e->ed;
  const int d = e->cfg.d, clamp = e->cfg.clamp, G = e->block_grid;
  float* p = e->at<float>(L.o_p);
  float* Ap = e->at<float>(L.o_ap);
  float* z = e->at<float>(L.o_z);
  double* X = e->at<double>(L.o_x);
  double* r = e->at<double>(L.o_r);
  const double* B = e->at<double>(L.o_b);
  double* row32 = e->at<double>(L.o_row32);
  float* col32 = e->at<float>(L.o_col32);
  double* row64 = e->at<double>(L.o_row64);
  double* col64 = e->at<double>(L.o_col64);
  int* status = &e->at<WsHeader>(L.o_hdr)->status;
  int* scal = e->at<int>(L.o_scal);
  cudaError_t err =
      L.tc ? launch_k1t_batched(e->at<uint8_t>(L.o_img), clamp, p, row32, col32, e->sp32, e->bm32,
                                status, ed.active, cs, L.fmt)
           : launch_k1s_batched(e->at<float>(L.o_p32), d, clamp, p, row32, col32, e->sp32, e->bm32,
                                status, ed.active, cs);
  if (err != cudaSuccess) return err;
  eng_after_matvec_kernel<<<G, BT, 0, cs>>>(ed, e->sp32, e->bm32, row32, col32, p, Ap);
  eng_update_xr_kernel<<<G, BT, 0, cs>>>(ed, p, Ap, X, r);
  eng_compact_kernel<<<1, kCompactThreads, 0, cs>>>(ed, 1, e->at<int>(L.o_needi),
                                                    e->at<int64_t>(L.o_needp), scal + 2);
  err = launch_k4s_batched(e->at<double>(L.o_p64), d, clamp, X, row64, col64, e->sp64, e->bm64,
                           status, scal + 2, cs);
  if (err != cudaSuccess) return err;
  eng_after_residual_kernel<<<G, BT, 0, cs>>>(ed, e->sp64, e->bm32, row64, col64, B, X, r);
  eng_expand_kernel<<<G, BT, 0, cs>>>(ed, 0, -1, r, z, 0);
  eng_update_p_kernel<<<G, BT, 0, cs>>>(ed, 0, -1, z, p, 0);
  eng_compact_kernel<<<1, kCompactThreads, 0, cs>>>(ed, 0, e->at<int>(L.o_acti),
                                                    e->at<int64_t>(L.o_actp), scal + 1);
  return cudaGetLastError();
}

constexpr int kLaunchesPerIteration = 9;

// Moves `bytes` from src down to dst (dst < src, ranges may overlap) in
// stream order, in pieces that never overlap.
cudaError_t move_down(char* dst, const char* src, size_t bytes, cudaStream_t s) {
  if (dst == src || bytes == 0) return cudaSuccess;
  const size_t gap = (size_t)(src - dst);
  for (size_t o = 0; o < bytes; o += gap) {
    const size_t len = std::min(gap, bytes - o);
    cudaError_t e = cudaMemcpyAsync(dst + o, src + o, len, cudaMemcpyDeviceToDevice, s);
    if (e != cudaSuccess) return e;
  }
  return cudaSuccess;
}

// Operand image of a slot's points for the tensor-core FP32 kernel, from its
// packed FP32 embeddings in the arena.
cudaError_t pack_slot_image(EngineHost* e, const SlotInfo& si) {
  const EngineLayout& L = e->L;
  if (!L.tc) return cudaSuccess;
  return launch_k1t_pack(e->at<float>(L.o_p32) + (size_t)si.seg * L.dp, si.npts, e->cfg.d,
                         e->at<uint8_t>(L.o_img) + (size_t)si.blk_start * k1t_image_bytes(1),
                         si.nblk * RB, e->stream, L.fmt);
}

// Re-places a slot's record and block map (device) from its host record.
cudaError_t place_slot(EngineHost* e, int k, bool reset) {
  const EngineLayout& L = e->L;
  const SlotInfo& info = e->slots[k].info;
  eng_place_kernel<<<1, 1, 0, e->stream>>>(e->ed, e->at<SlotInfo>(L.o_slots),
                                          e->at<int64_t>(L.o_scal + 8 * 2), k, info, e->nb_used,
                                          reset ? 1 : 0);
  const int64_t nb = info.nblk;
  eng_fill_int_kernel<<<(unsigned)std::max<int64_t>(1, std::min<int64_t>(ceil_div(nb, 256), 1024)), 256, 0,
                        e->stream>>>(e->at<int>(L.o_binst), info.blk_start, info.blk_start + nb, k);
  return cudaGetLastError();
}

// Moves every resident instance down to the bottom of the arenas.
cudaError_t compact_arenas(EngineHost* e) {
  const EngineLayout& L = e->L;
  std::vector<int> live;
  for (int k = 0; k < e->cfg.max_slots; ++k)
    if (e->slots[k].state != kFree) live.push_back(k);
  std::sort(live.begin(), live.end(), [&](int a, int b) {
    return e->slots[a].info.blk_start < e->slots[b].info.blk_start;
  });
  const int64_t old_used = e->nb_used;
  int64_t nb = 0, np = 0;
  const size_t dp = (size_t)L.dp;
  cudaError_t err = cudaSuccess;
  for (int k : live) {
    SlotInfo& si = e->slots[k].info;
    const int64_t pts = si.nblk * RB;
    if (si.blk_start != nb) {
      const int64_t from = si.seg, to = nb * RB;
      auto mv = [&](size_t off, size_t elem) {
        if (err == cudaSuccess)
          err = move_down(e->base + off + (size_t)to * elem, e->base + off + (size_t)from * elem,
                          (size_t)pts * elem, e->stream);
      };
      mv(L.o_p32, dp * 4);
      mv(L.o_p64, dp * 8);
      mv(L.o_b, 8);
      mv(L.o_x, 8);
      mv(L.o_r, 8);
      mv(L.o_p, 4);
      si.blk_start = nb;
      si.seg = to;
      if (err == cudaSuccess) err = pack_slot_image(e, si);
    }
    si.pair_start = np;
    nb += si.nblk;
    np += si.nblk * (si.nblk + 1) / 2;
  }
  if (err != cudaSuccess) return err;
  e->nb_used = nb;
  e->pairs_used = np;
  for (int k : live) {
    err = place_slot(e, k, false);
    if (err != cudaSuccess) return err;
  }
  if (old_used > nb)
    eng_fill_int_kernel<<<(unsigned)std::min<int64_t>(ceil_div(old_used - nb, 256), 1024), 256, 0,
                          e->stream>>>(e->at<int>(L.o_binst), nb, old_used, -1);
  eng_set_i64_kernel<<<1, 1, 0, e->stream>>>(e->at<int64_t>(L.o_scal + 8 * 2), nb);
  return cudaGetLastError();
}

// Lowers the bump pointers to the top of the resident instances.
void lower_tops(EngineHost* e) {
  int64_t nb = 0, np = 0;
  for (int k = 0; k < e->cfg.max_slots; ++k) {
    if (e->slots[k].state == kFree) continue;
    const SlotInfo& si = e->slots[k].info;
    nb = std::max(nb, si.blk_start + si.nblk);
    np = std::max(np, si.pair_start + si.nblk * (si.nblk + 1) / 2);
  }
  e->nb_used = nb;
  e->pairs_used = np;
}

}  // namespace
}  // namespace laker

using namespace laker;

extern "C" size_t laker_engine_host_bytes(const laker_engine_config* cfg) {
  return config_valid(cfg) ? host_bytes_for(cfg->max_slots) : 0;
}

extern "C" size_t laker_engine_workspace_bytes(const laker_engine_config* cfg) {
  return config_valid(cfg) ? engine_layout(*cfg).bytes : 0;
}

extern "C" int laker_engine_init(void* host, size_t host_bytes, void* workspace,
                                 size_t workspace_bytes, const laker_engine_config* cfg,
                                 const laker_pcg_params* prm, void* stream) {
  if (!host || !workspace || !config_valid(cfg) || !prm) return LAKER_ERR_INVALID_ARG;
  if (prm->max_iter < 0 || !(prm->tol >= 0.0) || !(prm->reliable_delta > 0.0) || prm->has_x0)
    return LAKER_ERR_INVALID_ARG;
  if (host_bytes < host_bytes_for(cfg->max_slots)) return LAKER_ERR_WORKSPACE;
  const EngineLayout L = engine_layout(*cfg);
  if (workspace_bytes < L.bytes) return LAKER_ERR_WORKSPACE;

  EngineHost* e = static_cast<EngineHost*>(host);
  std::memset(host, 0, host_bytes_for(cfg->max_slots));
  e->cfg = *cfg;
  e->prm = *prm;
  e->L = L;
  e->base = static_cast<char*>(workspace);
  e->stream = static_cast<cudaStream_t>(stream);
  char* tail = static_cast<char*>(host) + round_up((int64_t)sizeof(EngineHost), 64);
  e->slots = reinterpret_cast<SlotHost*>(tail);
  e->done_h = reinterpret_cast<int*>(tail + (size_t)cfg->max_slots * sizeof(SlotHost));
  e->sp32 = L.tc ? k1t_plan_pairs(L.cap_blocks, L.cap_pairs)
                 : k1s_plan_pairs(L.cap_blocks, L.cap_pairs, cfg->d);
  e->sp64 = k4s_plan_pairs(L.cap_blocks, L.cap_pairs, cfg->d);
  e->block_grid = (int)std::max<int64_t>(1, std::min<int64_t>(L.cap_blocks, 4 * (int64_t)sm_count()));

  EngineDev& ed = e->ed;
  ed.max_slots = cfg->max_slots;
  ed.max_iter = prm->max_iter;
  ed.ustride = L.ustride;
  ed.delta = prm->reliable_delta;
  ed.eps = prm->breakdown_eps;
  ed.tol = prm->tol;
  ed.slots = e->at<SlotInfo>(L.o_slots);
  ed.blk_inst = e->at<int>(L.o_binst);
  int* scal = e->at<int>(L.o_scal);
  ed.active = scal;
  ed.nb_used = e->at<int64_t>(L.o_scal + 8 * 2);
  ed.st = e->at<InstState>(L.o_st);
  ed.done = e->at<int>(L.o_done);
  ed.ctr = e->at<unsigned int>(L.o_ctr);
  ed.bpart = e->at<double>(L.o_bpart);
  ed.upart = e->at<float>(L.o_upart);
  ed.vvec = e->at<float>(L.o_vvec);
  e->bm32 = BatchMap{ed.slots, scal + 1, e->at<int>(L.o_acti), e->at<int64_t>(L.o_actp)};
  e->bm64 = BatchMap{ed.slots, scal + 2, e->at<int>(L.o_needi), e->at<int64_t>(L.o_needp)};

  cudaStream_t s = e->stream;
  // every slot free (done), no block in use, empty lists
  cudaError_t err = cudaMemsetAsync(e->base + L.o_hdr, 0, kWsHeader, s);
  if (err == cudaSuccess) err = cudaMemsetAsync(e->base + L.o_scal, 0, 64, s);
  if (err == cudaSuccess) err = cudaMemsetAsync(e->base + L.o_slots, 0, (size_t)L.slots * sizeof(SlotInfo), s);
  if (err == cudaSuccess) err = cudaMemsetAsync(e->base + L.o_ctr, 0, (size_t)L.slots * 4, s);
  if (err == cudaSuccess) err = cudaMemsetAsync(e->base + L.o_binst, 0xFF, (size_t)L.cap_blocks * 4, s);
  if (err == cudaSuccess) err = cudaMemsetAsync(e->base + L.o_actp, 0, 8, s);
  if (err == cudaSuccess) err = cudaMemsetAsync(e->base + L.o_needp, 0, 8, s);
  if (err == cudaSuccess) {
    eng_fill_int_kernel<<<(unsigned)std::min<int64_t>(ceil_div(L.slots, 256), 1024), 256, 0, s>>>(
        ed.done, 0, L.slots, 1);
    err = cudaGetLastError();
  }
  // the iteration, captured once
  if (err == cudaSuccess) err = cudaStreamCreateWithFlags(&e->cap, cudaStreamNonBlocking);
  if (err == cudaSuccess) err = cudaStreamBeginCapture(e->cap, cudaStreamCaptureModeThreadLocal);
  if (err == cudaSuccess) {
    cudaError_t ce = cudaSuccess;
    for (int it = 0; it < cfg->chunk && ce == cudaSuccess; ++it) ce = engine_iteration(e, e->cap);
    err = cudaStreamEndCapture(e->cap, &e->graph);
    if (err == cudaSuccess) err = ce;
  }
  if (err == cudaSuccess) err = cudaGraphInstantiate(&e->exec, e->graph, 0);
  if (err == cudaSuccess) err = cudaStreamSynchronize(s);
  if (err != cudaSuccess) {
    if (e->exec) cudaGraphExecDestroy(e->exec);
    if (e->graph) cudaGraphDestroy(e->graph);
    if (e->cap) cudaStreamDestroy(e->cap);
    return fail_cuda(err);
  }
  e->magic = kEngineMagic;
  return LAKER_OK;
}

extern "C" int laker_engine_admit(void* host, int64_t n, double lambda_reg, const float* packed32,
                                  const double* packed64, const laker_precond* pc, const double* b,
                                  int* slot) {
  EngineHost* e = engine_of(host);
  if (!e || n < 1 || !packed32 || !packed64 || !b || !slot) return LAKER_ERR_INVALID_ARG;
  if (e->launched) return LAKER_ERR_INVALID_ARG;  // between replays only
  if (pc && (pc->n != n || pc->nr < 1 || pc->nr > e->cfg.max_nr || pc->ldq < pc->nr ||
             pc->ldq > e->L.ustride || (pc->ldq % 4) || !pc->q_basis || !pc->w_core ||
             (reinterpret_cast<uintptr_t>(pc->q_basis) % 16)))
    return LAKER_ERR_INVALID_ARG;
  int k = -1;
  for (int i = 0; i < e->cfg.max_slots; ++i)
    if (e->slots[i].state == kFree) {
      k = i;
      break;
    }
  if (k < 0) return LAKER_ERR_CAPACITY;
  const int64_t nb = ceil_div(n, RB), np = nb * (nb + 1) / 2;
  if (e->nb_used + nb > e->L.cap_blocks || e->pairs_used + np > e->L.cap_pairs) {
    // compact when the free space suffices in total
    int64_t live_b = 0, live_p = 0;
    for (int i = 0; i < e->cfg.max_slots; ++i)
      if (e->slots[i].state != kFree) {
        live_b += e->slots[i].info.nblk;
        live_p += e->slots[i].info.nblk * (e->slots[i].info.nblk + 1) / 2;
      }
    if (live_b + nb > e->L.cap_blocks || live_p + np > e->L.cap_pairs) return LAKER_ERR_CAPACITY;
    cudaError_t ce = compact_arenas(e);
    if (ce != cudaSuccess) return fail_cuda(ce);
  }
  const EngineLayout& L = e->L;
  SlotInfo info{};
  info.blk_start = e->nb_used;
  info.seg = e->nb_used * RB;
  info.npts = n;
  info.nblk = nb;
  info.pair_start = e->pairs_used;
  info.lam = lambda_reg;
  info.cis = pc ? pc->inv_sqrt_iso : 1.0;
  info.q = pc ? reinterpret_cast<uint64_t>(pc->q_basis) : 0;
  info.w = pc ? reinterpret_cast<uint64_t>(pc->w_core) : 0;
  info.nr = pc ? pc->nr : 0;
  info.ldq = pc ? pc->ldq : 4;
  e->nb_used += nb;
  e->pairs_used += np;
  e->slots[k].info = info;
  e->slots[k].state = kRunning;

  cudaStream_t s = e->stream;
  const size_t dp = (size_t)L.dp;
  const size_t n32 = (size_t)round_up(n, 256) * dp, n64 = (size_t)round_up(n, 128) * dp;
  cudaError_t err = cudaMemcpyAsync(e->at<float>(L.o_p32) + (size_t)info.seg * dp, packed32, n32 * 4,
                                    cudaMemcpyDeviceToDevice, s);
  if (err == cudaSuccess)
    err = cudaMemcpyAsync(e->at<double>(L.o_p64) + (size_t)info.seg * dp, packed64, n64 * 8,
                          cudaMemcpyDeviceToDevice, s);
  if (err == cudaSuccess)
    err = cudaMemcpyAsync(e->at<double>(L.o_b) + info.seg, b, (size_t)n * 8, cudaMemcpyDeviceToDevice, s);
  if (err == cudaSuccess) err = pack_slot_image(e, info);
  if (err == cudaSuccess) err = place_slot(e, k, true);
  if (err == cudaSuccess) {
    const EngineDev& ed = e->ed;
    const int64_t g0 = info.blk_start, g1 = info.blk_start + nb;
    const unsigned G = (unsigned)std::min<int64_t>(nb, e->block_grid);
    double* X = e->at<double>(L.o_x);
    double* r = e->at<double>(L.o_r);
    float* z = e->at<float>(L.o_z);
    eng_init_kernel<<<G, BT, 0, s>>>(ed, g0, g1, e->at<double>(L.o_b), X, r);
    eng_expand_kernel<<<G, BT, 0, s>>>(ed, g0, g1, r, z, 1);
    eng_update_p_kernel<<<G, BT, 0, s>>>(ed, g0, g1, z, e->at<float>(L.o_p), 1);
    eng_compact_kernel<<<1, kCompactThreads, 0, s>>>(ed, 0, e->at<int>(L.o_acti),
                                                     e->at<int64_t>(L.o_actp), e->at<int>(L.o_scal) + 1);
    err = cudaGetLastError();
  }
  if (err != cudaSuccess) return fail_cuda(err);
  e->running += 1;  // refreshed by the next step
  *slot = k;
  return LAKER_OK;
}

extern "C" int laker_engine_launch(void* host) {
  EngineHost* e = engine_of(host);
  if (!e) return LAKER_ERR_INVALID_ARG;
  if (e->launched) return LAKER_ERR_INVALID_ARG;
  const EngineLayout& L = e->L;
  // the replay, then the running count, stop flags and device status into
  // the host state (pageable: the copies complete before laker_engine_sync
  // returns)
  cudaError_t err = cudaGraphLaunch(e->exec, e->stream);
  if (err == cudaSuccess)
    err = cudaMemcpyAsync(e->readback, e->at<int>(L.o_scal), 4, cudaMemcpyDeviceToHost, e->stream);
  if (err == cudaSuccess)
    err = cudaMemcpyAsync(e->readback + 1, &e->at<WsHeader>(L.o_hdr)->status, 4,
                          cudaMemcpyDeviceToHost, e->stream);
  if (err == cudaSuccess)
    err = cudaMemcpyAsync(e->done_h, e->at<int>(L.o_done), (size_t)L.slots * 4, cudaMemcpyDeviceToHost,
                          e->stream);
  if (err != cudaSuccess) return fail_cuda(err);
  e->launched = 1;
  return LAKER_OK;
}

extern "C" int laker_engine_sync(void* host, int* running) {
  EngineHost* e = engine_of(host);
  if (!e || !running) return LAKER_ERR_INVALID_ARG;
  if (!e->launched) {
    *running = e->running;
    return LAKER_OK;
  }
  cudaError_t err = cudaStreamSynchronize(e->stream);
  e->launched = 0;
  if (err != cudaSuccess) return fail_cuda(err);
  const EngineLayout& L = e->L;
  for (int k = 0; k < L.slots; ++k)
    if (e->slots[k].state == kRunning && e->done_h[k]) e->slots[k].state = kStopped;
  e->running = e->readback[0];
  *running = e->running;
  return e->readback[1] ? e->readback[1] : LAKER_OK;
}

extern "C" int laker_engine_step(void* host, int* running) {
  const int st = laker_engine_launch(host);
  if (st != LAKER_OK) return st;
  return laker_engine_sync(host, running);
}

extern "C" int laker_engine_finished(void* host, int* slots, int max_slots, int* count) {
  EngineHost* e = engine_of(host);
  if (!e || !count || (max_slots > 0 && !slots)) return LAKER_ERR_INVALID_ARG;
  int c = 0;
  for (int k = 0; k < e->cfg.max_slots && c < max_slots; ++k)
    if (e->slots[k].state == kStopped) slots[c++] = k;
  *count = c;
  return LAKER_OK;
}

extern "C" int laker_engine_collect(void* host, int slot, double* x, laker_pcg_result* res) {
  EngineHost* e = engine_of(host);
  if (!e || slot < 0 || slot >= e->cfg.max_slots || !x || !res) return LAKER_ERR_INVALID_ARG;
  if (e->launched) return LAKER_ERR_INVALID_ARG;  // between replays only
  if (e->slots[slot].state != kStopped) return LAKER_ERR_INVALID_ARG;
  const EngineLayout& L = e->L;
  const SlotInfo& si = e->slots[slot].info;
  InstState hs{};
  cudaError_t err = cudaMemcpyAsync(x, e->at<double>(L.o_x) + si.seg, (size_t)si.npts * 8,
                                    cudaMemcpyDeviceToDevice, e->stream);
  if (err == cudaSuccess)
    err = cudaMemcpyAsync(&hs, e->at<InstState>(L.o_st) + slot, sizeof(InstState),
                          cudaMemcpyDeviceToHost, e->stream);
  if (err == cudaSuccess) {
    eng_fill_int_kernel<<<(unsigned)std::min<int64_t>(ceil_div(si.nblk, 256), 1024), 256, 0, e->stream>>>(
        e->at<int>(L.o_binst), si.blk_start, si.blk_start + si.nblk, -1);
    err = cudaGetLastError();
  }
  if (err == cudaSuccess) err = cudaStreamSynchronize(e->stream);
  if (err != cudaSuccess) return fail_cuda(err);
  *res = laker_pcg_result{};
  res->status = hs.done ? hs.status : LAKER_ERR_NOT_CONVERGED;
  res->iterations = hs.iter;
  res->accurate_matvecs = hs.n_accurate;
  res->residual_norm = hs.bnorm == 0.0 ? 0.0 : hs.true_rnorm;
  res->rhs_norm = hs.bnorm;
  res->recurrence_norm = hs.rnorm;
  e->slots[slot].state = kFree;
  lower_tops(e);
  eng_set_i64_kernel<<<1, 1, 0, e->stream>>>(e->at<int64_t>(L.o_scal + 8 * 2), e->nb_used);
  err = cudaGetLastError();
  return err == cudaSuccess ? LAKER_OK : fail_cuda(err);
}

extern "C" int laker_engine_release(void* host) {
  EngineHost* e = engine_of(host);
  if (!e) return LAKER_ERR_INVALID_ARG;
  cudaStreamSynchronize(e->stream);
  if (e->exec) cudaGraphExecDestroy(e->exec);
  if (e->graph) cudaGraphDestroy(e->graph);
  if (e->cap) cudaStreamDestroy(e->cap);
  e->exec = nullptr;
  e->graph = nullptr;
  e->cap = nullptr;
  e->magic = 0;
  return LAKER_OK;
}

// ---- one-shot batch ---------------------------------------------------------------
namespace {

laker_engine_config batch_config(int count, const int64_t* n, int d, int max_nr, int clamp,
                                 int chunk) {
  laker_engine_config cfg{};
  cfg.max_slots = count;
  cfg.d = d;
  cfg.max_nr = max_nr;
  cfg.clamp = clamp;
  cfg.chunk = chunk;
  for (int k = 0; k < count; ++k) {
    const int64_t nk = n[k] > 0 ? n[k] : 1, nb = ceil_div(nk, RB);
    cfg.max_points += nb * RB;
    cfg.max_pairs += nb * (nb + 1) / 2;
  }
  return cfg;
}

}  // namespace

extern "C" int64_t laker_batch_layout(int count, const int64_t* n, int64_t* offsets) {
  if (count < 0 || (count > 0 && !n)) return -1;
  int64_t o = 0;
  for (int k = 0; k < count; ++k) {
    if (offsets) offsets[k] = o;
    o += round_up(n[k] > 0 ? n[k] : 1, 256);
  }
  if (offsets) offsets[count] = o;
  return o;
}

extern "C" size_t laker_pcg_batched_workspace_bytes(int count, const int64_t* n, int d, int max_nr) {
  if (count < 1 || !n || d < 1 || d > 16 || max_nr < 0 || max_nr > kMaxNr) return 0;
  for (int k = 0; k < count; ++k)
    if (n[k] < 1) return 0;
  const laker_engine_config cfg = batch_config(count, n, d, max_nr, 1, 8);
  return engine_layout(cfg).bytes;
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
  int max_nr = 0;
  for (int k = 0; k < count; ++k) {
    if (batch->n[k] < 1) return LAKER_ERR_INVALID_ARG;
    if (batch->precond) max_nr = std::max(max_nr, batch->precond[k].nr);
  }
  if (max_nr > kMaxNr) return LAKER_ERR_INVALID_ARG;
  int chunk = prm->check_every > 0 ? prm->check_every : 8;
  if (prm->max_iter > 0 && chunk > prm->max_iter) chunk = prm->max_iter;
  const laker_engine_config cfg = batch_config(count, batch->n, d, max_nr, batch->clamp ? 1 : 0, chunk);
  if (workspace_bytes < engine_layout(cfg).bytes) return LAKER_ERR_WORKSPACE;
  std::vector<char> host(host_bytes_for(count));
  int st = laker_engine_init(host.data(), host.size(), workspace, workspace_bytes, &cfg, prm, stream);
  if (st != LAKER_OK) return st;
  std::vector<int64_t> off(count + 1);
  laker_batch_layout(count, batch->n, off.data());
  const size_t dp = (size_t)padded_dim(d);
  std::vector<int> slot_of(count, -1);
  for (int k = 0; k < count && st == LAKER_OK; ++k) {
    const laker_precond* pc = batch->precond ? &batch->precond[k] : nullptr;
    st = laker_engine_admit(host.data(), batch->n[k], batch->lambda_reg[k],
                            batch->packed32 + (size_t)off[k] * dp, batch->packed64 + (size_t)off[k] * dp,
                            pc, B + off[k], &slot_of[k]);
  }
  int64_t iters = 0, steps = 0;
  int running = st == LAKER_OK ? count : 0;
  while (st == LAKER_OK && running > 0 && iters < (int64_t)prm->max_iter) {
    st = laker_engine_step(host.data(), &running);
    iters += chunk;
    ++steps;
  }
  EngineHost* e = engine_of(host.data());
  const int launches = (int)(steps * cfg.chunk * kLaunchesPerIteration + 4 * count);
  int dev_status = st;
  for (int k = 0; k < count && e; ++k) {
    results[k] = laker_pcg_result{};
    if (slot_of[k] < 0) {
      results[k].status = LAKER_ERR_INVALID_ARG;
      continue;
    }
    if (e->slots[slot_of[k]].state == kRunning) e->slots[slot_of[k]].state = kStopped;
    const int c = laker_engine_collect(host.data(), slot_of[k], X + off[k], &results[k]);
    if (c != LAKER_OK && dev_status == LAKER_OK) dev_status = c;
    results[k].kernel_launches = launches;
  }
  laker_engine_release(host.data());
  return dev_status;
}
