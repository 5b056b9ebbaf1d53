/*
 * OpenMP float64 attention-kernel matvec -- TEST INFRASTRUCTURE ONLY (oracle).
 *
 *   Y = lam * X + exp(Er Ec^T) X          (lam applied when `square`)
 *
 * Restates dense_attention_matvec / AttentionKernelOperator.matvec_impl
 * (laker/kernels.py:121-130, 209-270) in float64 without materialising the
 * kernel: each output row is one OpenMP work item, the row's kernel entries
 * are evaluated on the fly and accumulated in row order.  `clamp_value` is
 * the exp_safe clamp (kernels.py:98-107); pass +inf for no clamp.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

int oracle_num_threads(void) {
#ifdef _OPENMP
  return omp_get_max_threads();
#else
  return 1;
#endif
}

void oracle_attn_matvec(const double* Er, int64_t m, const double* Ec, int64_t n, int d,
                        double lam, double clamp_value, const double* X, int64_t k, double* Y,
                        int square) {
#pragma omp parallel
  {
    double* g = (double*)malloc(sizeof(double) * (size_t)(n > 0 ? n : 1));
#pragma omp for schedule(dynamic, 16)
    for (int64_t i = 0; i < m; ++i) {
      const double* ei = Er + i * d;
      for (int64_t j = 0; j < n; ++j) {
        const double* ej = Ec + j * d;
        double s = 0.0;
        for (int q = 0; q < d; ++q) s += ei[q] * ej[q];
        g[j] = s < clamp_value ? s : clamp_value;
      }
#pragma omp simd
      for (int64_t j = 0; j < n; ++j) g[j] = exp(g[j]);
      double* yi = Y + i * k;
      for (int64_t c = 0; c < k; ++c) yi[c] = square ? lam * X[i * k + c] : 0.0;
      if (k == 1) {
        double acc = 0.0;
        for (int64_t j = 0; j < n; ++j) acc += g[j] * X[j];
        yi[0] += acc;
      } else {
        for (int64_t j = 0; j < n; ++j) {
          const double gj = g[j];
          const double* xj = X + j * k;
          for (int64_t c = 0; c < k; ++c) yi[c] += gj * xj[c];
        }
      }
    }
    free(g);
  }
}
