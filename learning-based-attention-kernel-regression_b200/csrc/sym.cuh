// Work decomposition of the symmetric fused matvec (matvec_sym.cu) and the
// fixed-order finish that turns its partial sums into A x.
#pragma once

#include <math.h>

#include "internal.cuh"

namespace laker {

// Blocks of B points; pairs (a, b), a <= b, row-major over the upper triangle;
// CTA c owns pairs [c*q + min(c, rem), ... + q + (c < rem)).
struct SymPlan {
  int64_t nb;      // number of point blocks
  int64_t npairs;  // nb (nb + 1) / 2
  int64_t q, rem;  // pairs per CTA
  int grid;        // CTAs
  int B;           // points per block
  int cfg;         // kernel variant
};

// Index of pair (a, b), a <= b.
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

// CTA that owns pair p.
__host__ __device__ inline int64_t sym_cta_of(int64_t p, const SymPlan& sp) {
  const int64_t big = sp.rem * (sp.q + 1);
  if (p < big) return p / (sp.q + 1);
  return sp.q > 0 ? sp.rem + (p - big) / sp.q : sp.rem;
}

// sum_j K_ij x_j for row i from the partials of one symmetric matvec:
// the row-sum runs of the CTAs that processed row block a = i / B (slot
// cta + a), then the column sums of the pairs (a', a), a' < a, in order.
__device__ inline double sym_row_sum(const SymPlan& sp, const double* __restrict__ rowpart,
                                     const float* __restrict__ colpart, int64_t i) {
  const int64_t a = i / sp.B, o = i - a * sp.B;
  const int64_t c0 = sym_cta_of(sym_first_pair(a, sp.nb), sp);
  const int64_t c1 = sym_cta_of(sym_first_pair(a, sp.nb) + (sp.nb - a) - 1, sp);
  double s = 0.0;
  for (int64_t c = c0; c <= c1; ++c) s += rowpart[(c + a) * sp.B + o];
  for (int64_t ap = 0; ap < a; ++ap) s += (double)colpart[sym_pair_index(ap, a, sp.nb) * sp.B + o];
  return s;
}

// Plan for n points of padded dimension from d.
SymPlan k1s_plan(int64_t n, int d);
// Workspace pieces: rowpart (grid + nb) x B doubles, colpart npairs x B floats.
inline size_t sym_rowpart_elems(const SymPlan& sp) { return (size_t)(sp.grid + sp.nb) * sp.B; }
inline size_t sym_colpart_elems(const SymPlan& sp) { return (size_t)sp.npairs * sp.B; }
cudaError_t launch_k1s(const float* E32, int64_t n, int d, int clamp, const float* x,
                       double* rowpart, float* colpart, const SymPlan& sp, int* status,
                       const int* gate, cudaStream_t s);
// y = lam x + (sum of the partials) for the standalone matvec.
cudaError_t launch_sym_finish(const SymPlan& sp, const double* rowpart, const float* colpart,
                              int64_t n, float lam, const float* x, float* y, int64_t ldy,
                              cudaStream_t s);
// Whether square FP32 matvecs use the symmetric kernel (LAKER_K1_SYMMETRIC=0
// selects the plain one, for comparisons).
bool k1_use_symmetric();
// Bytes of the symmetric partials (rowpart, then colpart at a 256-byte boundary).
inline size_t sym_partial_bytes(const SymPlan& sp) {
  return (size_t)round_up((int64_t)(sym_rowpart_elems(sp) * sizeof(double)), 256) +
         sym_colpart_elems(sp) * sizeof(float);
}

}  // namespace laker
