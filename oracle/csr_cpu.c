/*
 * CPU CSR kernels for the oracle and the timed CPU baseline.
 *
 * TEST INFRASTRUCTURE ONLY (see oracle/__init__.py).
 *
 * csr_spmm_f64: y = diag * x + A x for row-major blocks x, y [n x k]
 *   (LinearOperator::apply, src/operator.rs:176-223).  Rows are split over
 *   OpenMP threads.  For k == 1 the inner product uses 4-wide AVX2 gathers
 *   with FMA and a scalar tail, the restatement of spmv_avx2_gather_inner
 *   (src/operator.rs:96-145); for k > 1 each entry updates the k-vector row
 *   accumulator (the row-major csr_mulacc_dense_rowmaj pattern).
 * column_sum_f32: deg[col] += w in CSR order, f32 (src/laplacian.rs:8-16).
 */
#include <stddef.h>
#include <stdint.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif
#if defined(__AVX2__) && defined(__FMA__)
#include <immintrin.h>
#endif

int csr_threads(void) {
#ifdef _OPENMP
  return omp_get_max_threads();
#else
  return 1;
#endif
}

void csr_set_threads(int t) {
#ifdef _OPENMP
  if (t > 0) omp_set_num_threads(t);
#else
  (void)t;
#endif
}

static double row_dot_k1(const uint64_t* indptr, const uint32_t* indices, const double* data, const double* x,
                         int64_t i) {
  uint64_t s = indptr[i], e = indptr[i + 1], b = s;
  double r = 0.0;
#if defined(__AVX2__) && defined(__FMA__)
  __m256d acc = _mm256_setzero_pd();
  for (; b + 4 <= e; b += 4) {
    __m128i vi = _mm_set_epi32((int)indices[b + 3], (int)indices[b + 2], (int)indices[b + 1], (int)indices[b]);
    __m256d xv = _mm256_i32gather_pd(x, vi, 8);
    __m256d dv = _mm256_loadu_pd(data + b);
    acc = _mm256_fmadd_pd(dv, xv, acc);
  }
  __m128d lo = _mm256_castpd256_pd128(acc), hi = _mm256_extractf128_pd(acc, 1);
  __m128d s2 = _mm_add_pd(lo, hi);
  r = _mm_cvtsd_f64(_mm_hadd_pd(s2, s2));
#endif
  for (; b < e; ++b) r += data[b] * x[indices[b]];
  return r;
}

void csr_spmm_f64(int64_t n, const uint64_t* indptr, const uint32_t* indices, const double* data, double diag,
                  const double* x, double* y, int k) {
  if (k == 1) {
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < n; ++i) y[i] = diag * x[i] + row_dot_k1(indptr, indices, data, x, i);
    return;
  }
#pragma omp parallel for schedule(static)
  for (int64_t i = 0; i < n; ++i) {
    double acc[64];
    const int kk = k < 64 ? k : 64;
    for (int c = 0; c < kk; ++c) acc[c] = diag * x[i * k + c];
    for (uint64_t q = indptr[i]; q < indptr[i + 1]; ++q) {
      const double v = data[q];
      const double* xr = x + (int64_t)indices[q] * k;
      for (int c = 0; c < kk; ++c) acc[c] += v * xr[c];
    }
    memcpy(y + i * k, acc, sizeof(double) * kk);
  }
}

void column_sum_f32(int64_t nnz, const uint32_t* indices, const float* data, float* deg) {
  for (int64_t q = 0; q < nnz; ++q) deg[indices[q]] += data[q];
}
