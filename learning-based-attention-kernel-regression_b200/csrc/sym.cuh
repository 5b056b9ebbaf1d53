// Work decomposition of the symmetric fused matvec (matvec_sym.cu) and the
// fixed-order finish that turns its partial sums into A x.
#pragma once

#include <math.h>

#include "internal.cuh"

namespace laker {

// Blocks of B points; pairs (a, b), a <= b, row-major over the upper triangle;
// CTA c owns pairs [c*q + min(c, rem), ... + q + (c < rem)).
struct SymPlan {
  int64_t nb;      // number of point blocks (all instances)
  int64_t npairs;  // number of block pairs (all instances)
  int64_t q, rem;  // pairs per CTA
  int grid;        // CTAs
  int B;           // points per block
  int cfg;         // kernel variant
};

// Placement of one instance of a batched launch: its points [seg, seg + npts)
// (seg a multiple of 512, so its packed embeddings start on a column tile and
// its blocks are whole), blocks blk_start .. blk_start + nblk - 1 and block
// pairs pair_start .. pair_start + nblk (nblk + 1) / 2 - 1 (the slots of its
// partial sums).  Pairs only pair blocks of the same instance, so the
// operator is block diagonal.
struct SlotInfo {
  int64_t seg, npts, nblk, blk_start, pair_start;
  double lam, cis;  // lambda, c^-1/2 of the preconditioner
  uint64_t q, w;    // preconditioner factors (0: none)
  int nr, ldq;
};

// Several independent problems in one launch: slot k is described by
// slots[k]; the launch covers the instances act_inst[0 .. *act_count), whose
// pairs are numbered consecutively (act_ps, exclusive prefix sums) and split
// evenly over the grid.  All arrays are device memory.
struct BatchMap {
  const SlotInfo* slots;
  const int* act_count;   // number of instances in the launch
  const int* act_inst;    // their slots
  const int64_t* act_ps;  // [count + 1]
};

// Index of pair (a, b), a <= b, among the nb (nb + 1) / 2 pairs of nb blocks.
__host__ __device__ inline int64_t sym_pair_index(int64_t a, int64_t b, int64_t nb) {
  return a * nb - a * (a - 1) / 2 + (b - a);
}

// First pair of row block a.
__host__ __device__ inline int64_t sym_first_pair(int64_t a, int64_t nb) {
  return a * nb - a * (a - 1) / 2;
}

// Pair p -> (a, b).
__host__ __device__ inline void sym_pair_coords(int64_t p, int64_t nb, int64_t* a, int64_t* b) {
  const double tn = 2.0 * (double)nb + 1.0;
  int64_t r = (int64_t)floor((tn - sqrt(tn * tn - 8.0 * (double)p)) * 0.5);
  if (r < 0) r = 0;
  if (r > nb - 1) r = nb - 1;
  while (r > 0 && sym_first_pair(r, nb) > p) --r;
  while (r + 1 < nb && sym_first_pair(r + 1, nb) <= p) ++r;
  *a = r;
  *b = r + (p - sym_first_pair(r, nb));
}

// sum_j K_ij x_j for local row li of an instance whose pairs start at global
// pair ps: the row sums of its pairs (a, b >= a), then the column sums of its
// pairs (a' < a, a), in that fixed order.  Both partial arrays hold one
// B-vector per pair (FP32 kernel: double row sums, float column sums; FP64
// kernel: both double).
// The terms go round-robin into four partial sums (independent chains, so
// the loads overlap), combined as (s0 + s1) + (s2 + s3): a fixed order.
template <typename RP, typename CP>
__device__ inline double sym_instance_row_sum(int64_t nb, int64_t ps, int B,
                                              const RP* __restrict__ rowpart,
                                              const CP* __restrict__ colpart, int64_t li) {
  const int64_t a = li / B, o = li - a * B;
  const int64_t f = ps + sym_first_pair(a, nb);
  double s[4] = {0.0, 0.0, 0.0, 0.0};
  const int64_t nq = nb - a;
  int64_t q = 0;
  for (; q + 4 <= nq; q += 4) {
#pragma unroll
    for (int u = 0; u < 4; ++u) s[u] += (double)rowpart[(f + q + u) * B + o];
  }
  for (int u = 0; q < nq; ++q, ++u) s[u] += (double)rowpart[(f + q) * B + o];
  int64_t ap = 0;
  for (; ap + 4 <= a; ap += 4) {
#pragma unroll
    for (int u = 0; u < 4; ++u) s[u] += (double)colpart[(ps + sym_pair_index(ap + u, a, nb)) * B + o];
  }
  for (int u = 0; ap < a; ++ap, ++u) s[u] += (double)colpart[(ps + sym_pair_index(ap, a, nb)) * B + o];
  return (s[0] + s[1]) + (s[2] + s[3]);
}

// Single instance.
template <typename RP, typename CP>
__device__ inline double sym_row_sum(const SymPlan& sp, const RP* __restrict__ rowpart,
                                     const CP* __restrict__ colpart, int64_t i) {
  return sym_instance_row_sum<RP, CP>(sp.nb, 0, sp.B, rowpart, colpart, i);
}

// Batched layout: local row li of instance k.
template <typename RP, typename CP>
__device__ inline double sym_row_sum_batched(const SymPlan& sp, const BatchMap& bm,
                                             const RP* __restrict__ rowpart,
                                             const CP* __restrict__ colpart, int k, int64_t li) {
  return sym_instance_row_sum<RP, CP>(bm.slots[k].nblk, bm.slots[k].pair_start, sp.B, rowpart,
                                      colpart, li);
}

// Points per block of the symmetric kernel.
int sym_block_points();
// Plan for n points of padded dimension from d.
SymPlan k1s_plan(int64_t n, int d);
// Plan for an explicit pair list (batched layout: nb = total blocks; the
// batched kernel takes only the grid from it and splits the running pairs at
// run time).
SymPlan k1s_plan_pairs(int64_t nb, int64_t npairs, int d);
// Workspace pieces: row and column partials, one B-vector per pair.
inline size_t sym_rowpart_elems(const SymPlan& sp) { return (size_t)sp.npairs * sp.B; }
inline size_t sym_colpart_elems(const SymPlan& sp) { return (size_t)sp.npairs * sp.B; }
cudaError_t launch_k1s(const float* E32, int64_t n, int d, int clamp, const float* x,
                       double* rowpart, float* colpart, const SymPlan& sp, int* status,
                       const int* gate, cudaStream_t s);
cudaError_t launch_k1s_batched(const float* E32, int d, int clamp, const float* x,
                               double* rowpart, float* colpart, const SymPlan& sp,
                               const BatchMap& bm, int* status, const int* gate, cudaStream_t s);
// Tensor-core symmetric FP32 kernel (matvec_symtc.cu): same blocks, pair
// slots and partial layout as k1s, logits by tcgen05 split-TF32 MMAs from an
// operand image of k1t_image_bytes(points) bytes (128 KB per 512 points,
// indexed by point: an instance at seg uses blocks seg / 512 ...).
bool k1t_enabled(int d);
// Operand formats of the image: split TF32 (kind::tf32 MMAs, two K steps of
// 8, three products each) or split FP16 (kind::f16, one K step of 16, three
// products: H H' + Hs L' + L Hs' with H = fp16(v), L = fp16((v - H) 2^12),
// Hs = fp16(H 2^-12)), used only for unclamped operators (every |e_k| < 9, so
// no FP16 overflow).  k1t_format(clamp, d) is the format a pack and the launches
// that read its image use (LAKER_VARIANT_K1T_LOGITS).  For embeddings of at
// most 10 (padded) dimensions the three split-FP16 products fit two K = 16
// MMAs (kK1tF16x2): the correction products Hs L' and L Hs' fill H H''s
// padding and a second K step, with the same FP16 values and products.
constexpr int kK1tTf32 = 0, kK1tF16 = 1, kK1tF16x2 = 2;
int k1t_format(int clamp, int d);
size_t k1t_image_bytes(int64_t points);
SymPlan k1t_plan(int64_t n);
SymPlan k1t_plan_pairs(int64_t nb, int64_t npairs);
// image of `rows` points (a multiple of 512) from the packed FP32 layout;
// points at or past npts are zero
cudaError_t launch_k1t_pack(const float* packed32, int64_t npts, int d, uint8_t* img, int64_t rows,
                            cudaStream_t s, int fmt = kK1tTf32);
cudaError_t launch_k1t(const uint8_t* img, int64_t n, int clamp, const float* x, double* rowpart,
                       float* colpart, const SymPlan& sp, int* status, const int* gate,
                       cudaStream_t s, int fmt = kK1tTf32);
cudaError_t launch_k1t_batched(const uint8_t* img, int clamp, const float* x, double* rowpart,
                               float* colpart, const SymPlan& sp, const BatchMap& bm, int* status,
                               const int* gate, cudaStream_t s, int fmt = kK1tTf32);
// y = lam x + (sum of the partials) for the standalone matvec.
// Outputs are NaN when *status reports a failure of the kernel that wrote the
// partials (status may be null).
cudaError_t launch_sym_finish(const SymPlan& sp, const double* rowpart, const float* colpart,
                              int64_t n, float lam, const float* x, float* y, int64_t ldy,
                              const int* status, cudaStream_t s);
// Whether square FP32 matvecs use the symmetric kernel (LAKER_K1_SYMMETRIC=0
// selects the plain one, for comparisons).
bool k1_use_symmetric();
// Whether a square FP32 operator of n points takes the symmetric kernel
// (k1_use_symmetric and more than LAKER_VARIANT_SYM_MIN_BLOCKS x 512 points).
bool k1_symmetric_for(int64_t n);
// Bytes of the symmetric partials: row sums (double), then column sums (CP:
// float for the FP32 kernel, double for the FP64 one) at a 256-byte boundary.
template <typename CP>
inline size_t sym_partial_bytes(const SymPlan& sp) {
  return (size_t)round_up((int64_t)(sym_rowpart_elems(sp) * sizeof(double)), 256) +
         sym_colpart_elems(sp) * sizeof(CP);
}
template <typename CP>
inline CP* sym_colpart_ptr(void* partials, const SymPlan& sp) {
  return reinterpret_cast<CP*>(static_cast<char*>(partials) +
                               round_up((int64_t)(sym_rowpart_elems(sp) * sizeof(double)), 256));
}

// FP64 symmetric kernel (same blocks and pair slots; its own grid).
SymPlan k4s_plan(int64_t n, int d);
SymPlan k4s_plan_pairs(int64_t nb, int64_t npairs, int d);
cudaError_t launch_k4s(const double* E64, int64_t n, int d, int clamp, const double* x,
                       double* rowpart, double* colpart, const SymPlan& sp, int* status,
                       const int* gate, cudaStream_t s);
cudaError_t launch_k4s_batched(const double* E64, int d, int clamp, const double* x,
                               double* rowpart, double* colpart, const SymPlan& sp,
                               const BatchMap& bm, int* status, const int* gate, cudaStream_t s);
// y = [b -] (lam x + K64 x) from the FP64 partials (b may be null).
cudaError_t launch_sym_finish64(const SymPlan& sp, const double* rowpart, const double* colpart,
                                int64_t n, double lam, const double* x, const double* b,
                                int64_t ldb, double* y, int64_t ldy, const int* status,
                                cudaStream_t s);
// Whether the FP64 residual uses the symmetric kernel (LAKER_K4_SYMMETRIC=0
// selects the plain one).
bool k4_use_symmetric();

}  // namespace laker
