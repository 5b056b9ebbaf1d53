// Mixed-precision preconditioned conjugate gradient, device resident.
//
// Iteration (single RHS), all scalars on the device:
//   part = K32 p                         FP32 fused matvec (K1), FP64 partials
//   Ap = lam p + sum(part); p.Ap, |p|, |Ap|      -> alpha, breakdown test
//   x += alpha p; r -= alpha Ap; |r|             (x, r in FP64)
//   if |r| <= delta |r_last_true| or |r| <= tol |b| or iter == max_iter:
//       r = b - A64 x                    FP64 fused residual (K4), |r|
//       converged when |r| <= tol |b|
//   u = Q^T r; v = W u; z = c^-1/2 r + Q v; r.z   -> beta
//   p = z + beta p
// The recurrence follows solve_1d (laker/solvers.py:189-295); the reliable
// update (FP64 residual replacement) is what lets an FP32 operator reach the
// float64 reference's residual: the stop test is always taken on the FP64
// residual.  Every kernel reads the device state first and does nothing once
// the solve has finished, so the host can launch several iterations between
// status polls.
#include <cstdlib>
#include "pcg_state.cuh"
#include "sym.cuh"

namespace laker {
int precond_grid();
// Grid of the preconditioner apply inside a solve: one CTA per 64 rows, at
// most precond_grid() (small problems then do not leave most CTAs idle, and
// the last CTA of the projection sums few partials).  Depends on n only.
inline int precond_grid_for(int64_t n) {
  const int64_t g = (n + 63) / 64;
  const int cap = precond_grid();
  return (int)(g < 1 ? 1 : (g > cap ? cap : g));
}
bool precond_valid(const laker_precond* pc);

namespace {

constexpr int T = kVecThreads;

// Grid of the kernels that finish an operator application (each row adds the
// partial sums of its block pairs, ~n / 512 loads): one row per thread, up to
// 4 CTAs per SM, so that enough loads are in flight.
int fin_grid(int64_t n) {
  int64_t g = ceil_div(n, T);
  const int64_t cap = 4 * (int64_t)sm_count();
  if (g > cap) g = cap;
  return (int)(g < 1 ? 1 : g);
}

int vec_grid(int64_t n) {
  int64_t g = ceil_div(n, T * 4);
  const int64_t cap = 2 * (int64_t)sm_count();
  if (g > cap) g = cap;
  return (int)(g < 1 ? 1 : g);
}

// Fixed-order total of the NQ per-block partials bp[NQ * b + q] over the
// grid, computed by the whole (last) block: thread t adds blocks t, t + T, ...
// in order, then a fixed shuffle tree and warp order.  Result in thread 0.
// (One thread walking every block's partial serialises on the L2 latency.)
template <int NQ>
__device__ __forceinline__ void grid_total(const double* bp, double (&out)[NQ], double* scratch) {
#pragma unroll
  for (int q = 0; q < NQ; ++q) out[q] = 0.0;
  for (unsigned int b = threadIdx.x; b < gridDim.x; b += T) {
#pragma unroll
    for (int q = 0; q < NQ; ++q) out[q] += __ldcg(bp + (int64_t)NQ * b + q);
  }
  block_sum<T, NQ>(out, scratch);
}

// x = 0 (unless warm start), r = b, |b| -> bnorm, tol_abs, rmax.
__global__ void __launch_bounds__(T)
    pcg_init_kernel(const double* __restrict__ b, double* __restrict__ x, double* __restrict__ r,
                    int64_t n, int has_x0, double tol, double* blockpart, PcgState* st) {
  __shared__ double s_red[T / 32];
  double acc = 0.0;
  for (int64_t i = blockIdx.x * (int64_t)T + threadIdx.x; i < n; i += (int64_t)gridDim.x * T) {
    const double bi = b[i];
    r[i] = bi;
    if (!has_x0) x[i] = 0.0;
    acc = fma(bi, bi, acc);
  }
  double v[1] = {acc};
  block_sum<T, 1>(v, s_red);
  if (threadIdx.x == 0) blockpart[blockIdx.x] = v[0];
  if (!arrive_last_block(&st->counters[kCtrBnorm])) return;
  double tot[1];
  grid_total<1>(blockpart, tot, s_red);
  if (threadIdx.x == 0) {
    const double bn = sqrt(tot[0]);
    st->bnorm = bn;
    st->tol_abs = tol * bn;
    st->rnorm = bn;
    st->rmax = bn;
    st->true_rnorm = bn;
    if (!isfinite(bn)) {
      st->status = LAKER_ERR_NONFINITE;
      st->done = 1;
      st->active = 0;
    }
  }
}

// Ap = lam p + (partial sums of the FP32 matvec); p.Ap, p.p, Ap.Ap ->
// breakdown test and alpha.  SYM: per-pair row and column sums of the
// symmetric kernel, else S column-segment partials in `part`.
template <bool SYM>
__global__ void __launch_bounds__(T)
    pcg_after_matvec_kernel(const double* __restrict__ part, int S, SymPlan sp,
                            const double* __restrict__ rowpart,
                            const float* __restrict__ colpart, const float* __restrict__ p,
                            float* __restrict__ Ap, int64_t n, double* blockpart, PcgState* st,
                            const int* dstatus) {
  if (st->done) return;
  __shared__ double s_red[3 * (T / 32)];
  const double lam = st->lam;
  double d0 = 0.0, d1 = 0.0, d2 = 0.0;
  for (int64_t i = blockIdx.x * (int64_t)T + threadIdx.x; i < n; i += (int64_t)gridDim.x * T) {
    const double pi = p[i];
    double a = lam * pi;
    if (SYM) {
      a += sym_row_sum(sp, rowpart, colpart, i);
    } else {
      for (int s = 0; s < S; ++s) a += part[(int64_t)s * n + i];
    }
    const float af = (float)a;
    Ap[i] = af;
    d0 = fma(pi, (double)af, d0);
    d1 = fma(pi, pi, d1);
    d2 = fma((double)af, (double)af, d2);
  }
  double v[3] = {d0, d1, d2};
  block_sum<T, 3>(v, s_red);
  if (threadIdx.x == 0) {
    blockpart[3 * blockIdx.x + 0] = v[0];
    blockpart[3 * blockIdx.x + 1] = v[1];
    blockpart[3 * blockIdx.x + 2] = v[2];
  }
  if (!arrive_last_block(&st->counters[kCtrMatvec])) return;
  double tot[3];
  grid_total<3>(blockpart, tot, s_red);
  if (threadIdx.x == 0) {
    const double pap = tot[0], pp = tot[1], aa = tot[2];
    st->pAp = pap;
    if (status_failed(dstatus)) {
      // the operator kernel recorded a device-side failure: its partials are
      // not a product
      st->status = *dstatus;
      st->done = 1;
      st->active = 0;
    } else if (!isfinite(pap) || !isfinite(pp) || !isfinite(aa)) {
      st->status = LAKER_ERR_NONFINITE;
      st->done = 1;
      st->active = 0;
    } else if (pap <= -st->eps * sqrt(pp) * sqrt(aa)) {
      // non-positive curvature (laker/solvers.py:232-246)
      st->status = LAKER_ERR_BREAKDOWN;
      st->done = 1;
      st->active = 0;
    } else {
      st->alpha = st->rz / pap;
    }
  }
}

// x += alpha p; r -= alpha Ap; |r| -> decide on the FP64 recomputation.
__global__ void __launch_bounds__(T)
    pcg_update_xr_kernel(const float* __restrict__ p, const float* __restrict__ Ap,
                         double* __restrict__ x, double* __restrict__ r, int64_t n,
                         double* blockpart, PcgState* st) {
  if (st->done) return;
  __shared__ double s_red[T / 32];
  const double alpha = st->alpha;
  double acc = 0.0;
  for (int64_t i = blockIdx.x * (int64_t)T + threadIdx.x; i < n; i += (int64_t)gridDim.x * T) {
    x[i] = fma(alpha, (double)p[i], x[i]);
    const double ri = fma(-alpha, (double)Ap[i], r[i]);
    r[i] = ri;
    acc = fma(ri, ri, acc);
  }
  double v[1] = {acc};
  block_sum<T, 1>(v, s_red);
  if (threadIdx.x == 0) blockpart[blockIdx.x] = v[0];
  if (!arrive_last_block(&st->counters[kCtrUpdate])) return;
  double tot[1];
  grid_total<1>(blockpart, tot, s_red);
  if (threadIdx.x == 0) {
    const double rn = sqrt(tot[0]);
    st->rnorm = rn;
    st->iter += 1;
    // Reliable-update trigger against the running maximum of the recurrence
    // residual since the last FP64 recomputation: PCG residual norms
    // oscillate, and comparing with the peak replaces the residual as soon
    // as the recurrence has made real progress (n = 20k: 274 iterations
    // instead of 412 when compared with the residual at the replacement).
    if (rn > st->rmax) st->rmax = rn;
    st->need_update =
        (rn <= st->delta * st->rmax || rn <= st->tol_abs || st->iter >= st->max_iter || !isfinite(rn))
            ? 1
            : 0;
  }
}

// After the FP64 matvec: r = b - (lam x + K64 x), |r| -> stop test.  SYM:
// per-pair row and column sums of the symmetric FP64 kernel, else S
// column-segment partials in `part`.  `init` seeds the state for a warm start
// (no iteration has run yet).
template <bool SYM>
__global__ void __launch_bounds__(T)
    pcg_after_residual_kernel(const double* __restrict__ part, int S, SymPlan sp,
                              const double* __restrict__ rowpart, const double* __restrict__ colpart,
                              const double* __restrict__ b, const double* __restrict__ x,
                              double* __restrict__ r, int64_t n, int init, double* blockpart,
                              PcgState* st) {
  if (st->done || (!init && !st->need_update)) return;
  __shared__ double s_red[T / 32];
  const double lam = st->lam;
  double acc = 0.0;
  for (int64_t i = blockIdx.x * (int64_t)T + threadIdx.x; i < n; i += (int64_t)gridDim.x * T) {
    double a = lam * x[i];
    if (SYM) {
      a += sym_row_sum(sp, rowpart, colpart, i);
    } else {
      for (int s = 0; s < S; ++s) a += part[(int64_t)s * n + i];
    }
    const double ri = b[i] - a;
    r[i] = ri;
    acc = fma(ri, ri, acc);
  }
  double v[1] = {acc};
  block_sum<T, 1>(v, s_red);
  if (threadIdx.x == 0) blockpart[blockIdx.x] = v[0];
  if (!arrive_last_block(&st->counters[kCtrResid])) return;
  double tot[1];
  grid_total<1>(blockpart, tot, s_red);
  if (threadIdx.x == 0) {
    const double rn = sqrt(tot[0]);
    st->rnorm = rn;
    st->true_rnorm = rn;
    st->rmax = rn;
    st->n_accurate += 1;
    st->need_update = 0;
    if (!isfinite(rn)) {
      st->status = LAKER_ERR_NONFINITE;
      st->done = 1;
      st->active = 0;
    } else if (!init && rn <= st->tol_abs) {
      st->status = LAKER_OK;
      st->done = 1;
      st->active = 0;
    } else if (!init && st->iter >= st->max_iter) {
      st->status = LAKER_ERR_NOT_CONVERGED;
      st->done = 1;
      st->active = 0;
    }
  }
}

// p = z + beta p; on the first call (init) p = z, without reading the
// uninitialised p.
__global__ void __launch_bounds__(T)
    pcg_update_p_kernel(const float* __restrict__ z, float* __restrict__ p, int64_t n,
                        const PcgState* st, int init) {
  if (st->done) return;
  const float beta = (float)st->beta;
  for (int64_t i = blockIdx.x * (int64_t)T + threadIdx.x; i < n; i += (int64_t)gridDim.x * T)
    p[i] = init ? z[i] : fmaf(beta, p[i], z[i]);
}

// Identity preconditioner: z = r, and r.z folded into beta like the fused apply.
__global__ void __launch_bounds__(T)
    identity_expand_kernel(const double* __restrict__ r, float* __restrict__ z, int64_t n,
                           double* blockpart, PcgState* st, int init) {
  if (st->done) return;
  __shared__ double s_red[T / 32];
  double acc = 0.0;
  for (int64_t i = blockIdx.x * (int64_t)T + threadIdx.x; i < n; i += (int64_t)gridDim.x * T) {
    const float zi = (float)r[i];
    z[i] = zi;
    acc = fma(r[i], (double)zi, acc);
  }
  double v[1] = {acc};
  block_sum<T, 1>(v, s_red);
  if (threadIdx.x == 0) blockpart[blockIdx.x] = v[0];
  if (!arrive_last_block(&st->counters[kCtrExpand])) return;
  double tot[1];
  grid_total<1>(blockpart, tot, s_red);
  if (threadIdx.x == 0) {
    const double t = tot[0];
    if (init) {
      st->rz = t;
      st->beta = 0.0;
    } else {
      st->beta = t / st->rz;
      st->rz = t;
    }
  }
}

// Optional per-launch CUDA-event timing of the fused matvecs (params.profile):
// events bracket each launch on the solve's stream and are read after the
// status poll that synchronises it.
struct LaunchTimer {
  static constexpr int kMax = 64;
  bool on = false;
  int used = 0, count = 0;
  double total_ms = 0.0;
  cudaEvent_t ev[2 * kMax];
  void init(bool enable) {
    on = enable;
    if (!on) return;
    for (auto& e : ev)
      if (cudaEventCreate(&e) != cudaSuccess) on = false;
  }
  void begin(cudaStream_t s) {
    if (on && used < kMax) cudaEventRecord(ev[2 * used], s);
  }
  void end(cudaStream_t s) {
    if (on && used < kMax) cudaEventRecord(ev[2 * used + 1], s), ++used;
  }
  void collect() {
    for (int i = 0; i < used; ++i) {
      float ms = 0.0f;
      if (cudaEventElapsedTime(&ms, ev[2 * i], ev[2 * i + 1]) == cudaSuccess) total_ms += ms, ++count;
    }
    used = 0;
  }
  ~LaunchTimer() {
    if (on)
      for (auto& e : ev) cudaEventDestroy(e);
  }
};

// Workspace carve-up of one single-RHS solve.
struct PcgWs {
  WsHeader* hdr;
  PcgState* st;
  double* r;
  float* Ap;
  float* z;
  float* p;
  double* part32;  // S1 x n FP64 partials of the FP32 matvec
  double* part64;  // S4 x n FP64 partials of the FP64 matvec
  double* blockpart;
  double* upart;
  double* v;
  uint8_t* img;  // operand image of the tensor-core symmetric kernel (or null)
  size_t bytes;
};

// The captured iteration of a solve (released when the solve returns; a
// graph still executing on the caller's stream is freed by the runtime once it
// completes).
struct IterGraph {
  cudaStream_t cap = nullptr;
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  ~IterGraph() {
    if (exec) cudaGraphExecDestroy(exec);
    if (graph) cudaGraphDestroy(graph);
    if (cap) cudaStreamDestroy(cap);
  }
};

// Whether laker_pcg_solve replays its iteration as a CUDA graph
// (LAKER_PCG_GRAPH=0 launches the kernels one by one).
bool pcg_use_graph() {
  static int v = -1;
  if (v < 0) {
    const char* e = getenv("LAKER_PCG_GRAPH");
    v = (e && e[0] == '0') ? 0 : 1;
  }
  return v == 1;
}

PcgWs carve(void* base, int64_t n, int d, int nr) {
  PcgWs w{};
  char* p = static_cast<char*>(base);
  size_t off = 0;
  auto take = [&](size_t bytes) {
    char* q = p ? p + off : nullptr;
    off += (size_t)round_up((int64_t)bytes, 256);
    return q;
  };
  const SegPlan p1 = k1_plan(n, n, d), p4 = k4_plan(n, n, d);
  int G = vec_grid(n) > precond_grid() ? vec_grid(n) : precond_grid();
  if (fin_grid(n) > G) G = fin_grid(n);
  w.hdr = reinterpret_cast<WsHeader*>(take(kWsHeader));
  w.st = reinterpret_cast<PcgState*>(take(sizeof(PcgState)));
  w.r = reinterpret_cast<double*>(take(n * sizeof(double)));
  w.Ap = reinterpret_cast<float*>(take(n * sizeof(float)));
  w.z = reinterpret_cast<float*>(take(n * sizeof(float)));
  w.p = reinterpret_cast<float*>(take(n * sizeof(float)));
  {
    // FP32 matvec partials: column segments, or the symmetric kernel's layout
    size_t b32 = (size_t)p1.S * n * sizeof(double);
    const size_t bs = sym_partial_bytes<float>(k1s_plan(n, d));
    w.part32 = reinterpret_cast<double*>(take(b32 > bs ? b32 : bs));
  }
  {
    // FP64 matvec partials: column segments, or the symmetric kernel's layout
    const size_t b64 = (size_t)p4.S * n * sizeof(double);
    const size_t bs = sym_partial_bytes<double>(k4s_plan(n, d));
    w.part64 = reinterpret_cast<double*>(take(b64 > bs ? b64 : bs));
  }
  w.blockpart = reinterpret_cast<double*>(take((size_t)G * 4 * sizeof(double)));
  (void)nr;  // the apply's partials are sized for the largest padded row (1024)
  w.upart = reinterpret_cast<double*>(take((size_t)precond_grid() * kMaxNr * sizeof(double)));
  w.v = reinterpret_cast<double*>(take((size_t)kMaxNr * sizeof(double)));
  w.img = k1t_enabled(d) ? reinterpret_cast<uint8_t*>(take(k1t_image_bytes(n))) : nullptr;
  w.bytes = off;
  return w;
}

}  // namespace
}  // namespace laker

using namespace laker;

extern "C" size_t laker_pcg_workspace_bytes(int64_t n, int d, int nr, int k) {
  if (n < 1 || d < 1 || d > 16 || nr < 0 || nr > kMaxNr || k < 1) return 0;
  if (k != 1) return pcg_multi_workspace_bytes(n, d, nr, k);
  return carve(nullptr, n, d, nr).bytes;
}

extern "C" int laker_pcg_solve(const laker_operator* op, const laker_precond* pc, const double* B,
                               int k, double* X, const laker_pcg_params* prm, void* workspace,
                               size_t workspace_bytes, laker_pcg_result* res, void* stream) {
  if (!op || !prm || !res || !B || !X || !workspace) return LAKER_ERR_INVALID_ARG;
  if (op->n < 1 || op->d < 1 || op->d > 16 || !op->packed32 || !op->packed64) return LAKER_ERR_INVALID_ARG;
  if (k < 1) return LAKER_ERR_INVALID_ARG;
  if (pc && (pc->n != op->n || !precond_valid(pc))) return LAKER_ERR_INVALID_ARG;
  if (prm->max_iter < 0 || !(prm->tol >= 0.0) || !(prm->reliable_delta > 0.0)) return LAKER_ERR_INVALID_ARG;
  const int64_t n = op->n;
  const int d = op->d;
  const int nr = pc ? pc->nr : 0;
  if (workspace_bytes < laker_pcg_workspace_bytes(n, d, nr, k)) return LAKER_ERR_WORKSPACE;

  cudaStream_t s = static_cast<cudaStream_t>(stream);
  if (k > 1) return pcg_solve_multi(op, pc, B, k, X, prm, workspace, res, s);
  PcgWs w = carve(workspace, n, d, nr);
  const SegPlan p1 = k1_plan(n, n, d), p4 = k4_plan(n, n, d);
  const bool sym = k1_symmetric_for(n);
  const bool tc = sym && k1t_enabled(d);
  const SymPlan sp = tc ? k1t_plan(n) : k1s_plan(n, d);
  double* sym_row = w.part32;
  float* sym_col = sym_colpart_ptr<float>(w.part32, sp);
  const int G = vec_grid(n), Gp = precond_grid_for(n), Gf = fin_grid(n);
  int* dstatus = &w.hdr->status;
  const bool sym64 = k4_use_symmetric();
  const SymPlan sp64 = k4s_plan(n, d);
  double* row64 = w.part64;
  double* col64 = sym_colpart_ptr<double>(w.part64, sp64);
  // r = b - A64 x (gated on the device by `gate`)
  auto launch_residual = [&](int init, const int* gate, cudaStream_t cs) -> cudaError_t {
    cudaError_t ee;
    if (sym64) {
      ee = launch_k4s(op->packed64, n, d, op->clamp, X, row64, col64, sp64, dstatus, gate, cs);
      if (ee == cudaSuccess)
        pcg_after_residual_kernel<true><<<Gf, T, 0, cs>>>(nullptr, 0, sp64, row64, col64, B, X, w.r,
                                                         n, init, w.blockpart, w.st);
    } else {
      ee = launch_k4(op->packed64, n, op->packed64, n, d, op->clamp, X, w.part64, p4, dstatus, gate, cs);
      if (ee == cudaSuccess)
        pcg_after_residual_kernel<false><<<Gf, T, 0, cs>>>(w.part64, p4.S, sp64, nullptr, nullptr, B,
                                                          X, w.r, n, init, w.blockpart, w.st);
    }
    return ee;
  };
  const PcView view{pc ? pc->q_basis : nullptr, pc ? pc->w_core : nullptr, n, nr,
                    pc ? pc->ldq : 4, pc ? pc->inv_sqrt_iso : 1.0};

  *res = laker_pcg_result{};
  PcgState h{};
  h.delta = prm->reliable_delta;
  h.eps = prm->breakdown_eps;
  h.lam = op->lambda_reg;
  h.max_iter = prm->max_iter;
  h.active = 1;
  cudaError_t e = cudaMemsetAsync(w.hdr, 0, kWsHeader, s);
  if (e == cudaSuccess) e = cudaMemcpyAsync(w.st, &h, sizeof(PcgState), cudaMemcpyHostToDevice, s);
  const int tfmt = k1t_format(op->clamp, d);  // image format: the pack and every launch
  if (e == cudaSuccess && tc) e = launch_k1t_pack(op->packed32, n, d, w.img, sp.nb * sp.B, s, tfmt);
  if (e != cudaSuccess) return fail_cuda(e);

  int launches = tc ? 1 : 0;
  LaunchTimer t32, t64;
  t32.init(prm->profile != 0);
  t64.init(prm->profile != 0);
  auto launch_precond = [&](int init, cudaStream_t cs) {
    if (pc) {
      launch_precond_apply<float>(view, Gp, w.r, w.upart, w.v, w.z, w.blockpart,
                                  &w.st->counters[kCtrProject], &w.st->counters[kCtrExpand], w.st,
                                  init, nullptr, &w.st->active, cs);
      launches += 2;
    } else {
      identity_expand_kernel<<<G, T, 0, cs>>>(w.r, w.z, n, w.blockpart, w.st, init);
      launches += 1;
    }
    pcg_update_p_kernel<<<G, T, 0, cs>>>(w.z, w.p, n, w.st, init);
    launches += 1;
  };

  // ---- initialisation ------------------------------------------------------
  pcg_init_kernel<<<G, T, 0, s>>>(B, X, w.r, n, prm->has_x0, prm->tol, w.blockpart, w.st);
  launches += 1;
  e = cudaGetLastError();
  if (e != cudaSuccess) return fail_cuda(e);
  if (prm->has_x0) {
    // warm start: r = b - A x0 with the FP64 operator (laker/solvers.py:165-173)
    e = launch_residual(1, nullptr, s);
    if (e != cudaSuccess) return fail_cuda(e);
    launches += 2;
  }
  e = cudaMemcpyAsync(&h, w.st, sizeof(PcgState), cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  if (e != cudaSuccess) return fail_cuda(e);
  res->rhs_norm = h.bnorm;
  res->kernel_launches = launches;
  if (h.bnorm == 0.0) {
    // zero right-hand side: x is returned unchanged (zero, or x0), as in
    // laker/solvers.py:177-182
    res->status = LAKER_OK;
    res->residual_norm = 0.0;
    return LAKER_OK;
  }
  if (h.done) {
    res->status = h.status;
    res->residual_norm = h.true_rnorm;
    return h.status;
  }
  launch_precond(1, s);

  // ---- iterations ----------------------------------------------------------
  // One iteration: FP32 operator, alpha / x / r, the gated FP64 residual, the
  // preconditioner and p.  Every decision is on the device (gates), so the
  // iteration is launched as a CUDA graph captured once per solve (one graph
  // launch instead of ~8 kernel launches per iteration); profiling runs launch
  // the kernels directly so that the operator launches can be timed.
  auto iteration = [&](cudaStream_t cs, bool timed) {
    if (timed) t32.begin(cs);
    if (tc) {
      launch_k1t(w.img, n, op->clamp, w.p, sym_row, sym_col, sp, dstatus, &w.st->active, cs, tfmt);
    } else if (sym) {
      launch_k1s(op->packed32, n, d, op->clamp, w.p, sym_row, sym_col, sp, dstatus, &w.st->active, cs);
    } else {
      launch_k1(op->packed32, n, op->packed32, n, d, op->clamp, w.p, w.part32, p1, dstatus,
                &w.st->active, cs);
    }
    if (timed) t32.end(cs);
    if (sym)
      pcg_after_matvec_kernel<true><<<Gf, T, 0, cs>>>(w.part32, 0, sp, sym_row, sym_col, w.p, w.Ap, n,
                                                     w.blockpart, w.st, dstatus);
    else
      pcg_after_matvec_kernel<false><<<Gf, T, 0, cs>>>(w.part32, p1.S, sp, nullptr, nullptr, w.p, w.Ap,
                                                      n, w.blockpart, w.st, dstatus);
    pcg_update_xr_kernel<<<G, T, 0, cs>>>(w.p, w.Ap, X, w.r, n, w.blockpart, w.st);
    if (timed) t64.begin(cs);
    launch_residual(0, &w.st->need_update, cs);
    if (timed) t64.end(cs);
    launches += 5;
    launch_precond(0, cs);
  };
  IterGraph ig;
  int iter_launches = 0;
  if (prm->profile == 0 && pcg_use_graph()) {
    const int before = launches;
    e = cudaStreamCreateWithFlags(&ig.cap, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaStreamBeginCapture(ig.cap, cudaStreamCaptureModeThreadLocal);
    if (e == cudaSuccess) {
      iteration(ig.cap, false);
      const cudaError_t ce = cudaGetLastError();
      e = cudaStreamEndCapture(ig.cap, &ig.graph);
      if (e == cudaSuccess) e = ce;
    }
    if (e == cudaSuccess) e = cudaGraphInstantiate(&ig.exec, ig.graph, 0);
    if (e != cudaSuccess) return fail_cuda(e);
    iter_launches = launches - before;
    launches = before;
  }
  int check = prm->check_every;
  if (check < 1) {
    // poll roughly every 10 ms of FP32 operator work (~2e12 entries/s)
    const double est_s = (double)n * (double)n / 2e12 + 40e-6;
    check = (int)(0.01 / est_s);
    if (check < 1) check = 1;
  }
  if (check > LaunchTimer::kMax) check = LaunchTimer::kMax;
  int launched = 0;
  while (launched < prm->max_iter) {
    const int chunk = (prm->max_iter - launched) < check ? (prm->max_iter - launched) : check;
    for (int c = 0; c < chunk; ++c) {
      if (ig.exec) {
        e = cudaGraphLaunch(ig.exec, s);
        if (e != cudaSuccess) return fail_cuda(e);
        launches += iter_launches;
      } else {
        iteration(s, true);
      }
    }
    launched += chunk;
    e = cudaGetLastError();
    if (e == cudaSuccess) e = cudaMemcpyAsync(&h, w.st, sizeof(PcgState), cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) return fail_cuda(e);
    t32.collect();
    t64.collect();
    if (h.done) break;
  }

  int dev_status = 0;
  e = cudaMemcpy(&dev_status, dstatus, sizeof(int), cudaMemcpyDeviceToHost);
  if (e != cudaSuccess) return fail_cuda(e);
  res->iterations = h.iter;
  res->accurate_matvecs = h.n_accurate;
  res->residual_norm = h.true_rnorm;
  res->recurrence_norm = h.rnorm;
  res->rhs_norm = h.bnorm;
  res->kernel_launches = launches;
  res->fp32_matvec_ms = t32.total_ms;
  res->fp32_matvec_launches = t32.count;
  res->fp64_matvec_ms = t64.total_ms;
  res->fp64_matvec_launches = t64.count;
  if (dev_status != 0) {
    res->status = dev_status;
    return dev_status;
  }
  if (!h.done) {
    // max_iter == 0: nothing ran
    res->status = LAKER_ERR_NOT_CONVERGED;
    return LAKER_ERR_NOT_CONVERGED;
  }
  res->status = h.status;
  return h.status;
}
