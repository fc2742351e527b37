// Block conjugate gradients for (L + eps I) Y = B, one independent CG per
// column (the inner solve of the shift-invert eigensolver).  Each iteration
// is four launches on the context stream:
//   Q = M P                (the CSR SpMM, diagonal coefficient 1 + eps)
//   alpha = rr / (P.Q)     (column dots, last CTA turns them into alpha)
//   Y += alpha P, R -= alpha Q, rr' = R.R  (last CTA: beta = rr'/rr, convergence)
//   P = R + beta P
// Reductions are deterministic (per-CTA partials added in CTA order).
#include <algorithm>
#include <cfloat>

#include "si_internal.h"

namespace si {

namespace {

constexpr int kCgT = 256;

struct CgScalars {
  double rr[MAXM];
  double rr0[MAXM];
  double alpha[MAXM];
  double beta[MAXM];
  int active[MAXM];
  int n_active;
};

// Reduce per-thread column sums acc[0..m) over the grid: per-CTA partials,
// the last CTA adds them in CTA order into tot[] (shared) and returns true.
__device__ bool reduce_cols(const double (&acc)[MAXM], int m, double* __restrict__ partial,
                            unsigned* __restrict__ counter, double* tot) {
  __shared__ double red[kCgT / 32][MAXM];
  __shared__ bool last;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
#pragma unroll
  for (int c = 0; c < MAXM; ++c) {
    const double s = warp_sum(acc[c]);
    if (lane == 0) red[warp][c] = s;
  }
  __syncthreads();
  if (threadIdx.x < m) {
    double s = 0.0;
    for (int w = 0; w < kCgT / 32; ++w) s += red[w][threadIdx.x];
    partial[static_cast<int64_t>(threadIdx.x) * gridDim.x + blockIdx.x] = s;
  }
  __threadfence();
  __syncthreads();
  if (threadIdx.x == 0) last = (atomicAdd(counter, 1u) == gridDim.x - 1);
  __syncthreads();
  if (!last) return false;
  __threadfence();
  if (threadIdx.x < m) {
    double s = 0.0;
    for (int bb = 0; bb < static_cast<int>(gridDim.x); ++bb)
      s += __ldcg(&partial[static_cast<int64_t>(threadIdx.x) * gridDim.x + bb]);
    tot[threadIdx.x] = s;
  }
  __syncthreads();
  if (threadIdx.x == 0) *counter = 0u;
  return true;
}

// per-thread column sums of a[i,c] * b[i,c] over this thread's rows
__device__ void row_dots(const double* __restrict__ a, const double* __restrict__ b, int m, int ld, int64_t n,
                         double (&acc)[MAXM]) {
#pragma unroll
  for (int c = 0; c < MAXM; ++c) acc[c] = 0.0;
  const int64_t stride = static_cast<int64_t>(gridDim.x) * blockDim.x;
  for (int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; i < n; i += stride) {
#pragma unroll
    for (int c = 0; c < MAXM; ++c)
      if (c < m) acc[c] = fma(a[i * ld + c], b[i * ld + c], acc[c]);
  }
}

__global__ void __launch_bounds__(kCgT) k_cg_alpha(const double* __restrict__ p, const double* __restrict__ q, int m,
                                                   int ld, int64_t n, double* partial, unsigned* counter,
                                                   CgScalars* sc) {
  __shared__ double tot[MAXM];
  double acc[MAXM];
  row_dots(p, q, m, ld, n, acc);
  if (!reduce_cols(acc, m, partial, counter, tot)) return;
  if (threadIdx.x < m) {
    const int c = threadIdx.x;
    const double pq = tot[c];
    sc->alpha[c] = (sc->active[c] && pq > 0.0) ? sc->rr[c] / pq : 0.0;
  }
}

// Y += alpha P ; R -= alpha Q ; then rr' = R.R, beta, convergence (last CTA)
__global__ void __launch_bounds__(kCgT) k_cg_update(double* __restrict__ y, double* __restrict__ r,
                                                    const double* __restrict__ p, const double* __restrict__ q, int m,
                                                    int ld, int64_t n, double tol2, double* partial, unsigned* counter,
                                                    CgScalars* sc) {
  __shared__ double al[MAXM];
  __shared__ double tot[MAXM];
  if (threadIdx.x < MAXM) al[threadIdx.x] = threadIdx.x < m ? sc->alpha[threadIdx.x] : 0.0;
  __syncthreads();
  // each thread updates its own rows and sums the new residual over them
  double acc[MAXM];
#pragma unroll
  for (int c = 0; c < MAXM; ++c) acc[c] = 0.0;
  const int64_t stride = static_cast<int64_t>(gridDim.x) * blockDim.x;
  for (int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; i < n; i += stride) {
#pragma unroll
    for (int c = 0; c < MAXM; ++c) {
      if (c < m) {
        const int64_t o = i * ld + c;
        y[o] = fma(al[c], p[o], y[o]);
        const double rv = fma(-al[c], q[o], r[o]);
        r[o] = rv;
        acc[c] = fma(rv, rv, acc[c]);
      }
    }
  }
  if (!reduce_cols(acc, m, partial, counter, tot)) return;
  if (threadIdx.x == 0) {
    int act = 0;
    for (int c = 0; c < m; ++c) {
      const double rn = tot[c];
      sc->beta[c] = (sc->active[c] && sc->rr[c] > 0.0) ? rn / sc->rr[c] : 0.0;
      sc->rr[c] = rn;
      if (sc->active[c] && !(rn > tol2 * sc->rr0[c])) sc->active[c] = 0;
      act += sc->active[c];
    }
    sc->n_active = act;
  }
}

__global__ void k_cg_dir(double* __restrict__ p, const double* __restrict__ r, int m, int ld, int64_t n,
                         const CgScalars* sc) {
  __shared__ double be[MAXM];
  __shared__ int ac[MAXM];
  if (threadIdx.x < MAXM) {
    be[threadIdx.x] = threadIdx.x < m ? sc->beta[threadIdx.x] : 0.0;
    ac[threadIdx.x] = threadIdx.x < m ? sc->active[threadIdx.x] : 0;
  }
  __syncthreads();
  const int64_t total = n * m;
  const int64_t stride = static_cast<int64_t>(gridDim.x) * blockDim.x;
  for (int64_t e = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; e < total; e += stride) {
    const int64_t i = e / m;
    const int c = static_cast<int>(e - i * m);
    const int64_t o = i * ld + c;
    p[o] = ac[c] ? fma(be[c], p[o], r[o]) : 0.0;
  }
}

// rr = rr0 = B.B, all columns with a nonzero right-hand side active
__global__ void __launch_bounds__(kCgT) k_cg_init(const double* __restrict__ b, int m, int ld, int64_t n,
                                                  double* partial, unsigned* counter, CgScalars* sc) {
  __shared__ double tot[MAXM];
  double acc[MAXM];
  row_dots(b, b, m, ld, n, acc);
  if (!reduce_cols(acc, m, partial, counter, tot)) return;
  if (threadIdx.x == 0) {
    int act = 0;
    for (int c = 0; c < MAXM; ++c) {
      const double v = c < m ? tot[c] : 0.0;
      sc->rr[c] = v;
      sc->rr0[c] = v;
      sc->alpha[c] = 0.0;
      sc->beta[c] = 0.0;
      sc->active[c] = (c < m && v > 0.0) ? 1 : 0;
      act += sc->active[c];
    }
    sc->n_active = act;
  }
}

int cg_grid(const Exec& ex, int64_t items) {
  return static_cast<int>(std::max<int64_t>(1, std::min<int64_t>((items + kCgT - 1) / kCgT, int64_t(ex.sms) * 4)));
}

}  // namespace

int cg_solve_block_dev(const Exec& ex, const OpDev& M, const double* b, double* y, int m, int ld, int64_t n,
                       double rtol, int maxit, CgWork& w, bool* converged) {
  SI_REQUIRE(m >= 1 && m <= MAXM && ld >= m, SI_INVALID_ARGUMENT, "cg: block width");
  const size_t sz = static_cast<size_t>(n) * ld;
  if (w.r.size() < sz) {
    w.r.alloc(sz, ex.stream);
    w.p.alloc(sz, ex.stream);
    w.q.alloc(sz, ex.stream);
  }
  const int grid_red = cg_grid(ex, n);
  if (w.partial.size() < static_cast<size_t>(MAXM) * grid_red) w.partial.alloc(static_cast<size_t>(MAXM) * grid_red, ex.stream);
  if (w.counter.size() < 1) {
    w.counter.alloc(1, ex.stream);
    w.counter.zero();
  }
  if (w.scal.size() < sizeof(CgScalars)) w.scal.alloc(sizeof(CgScalars), ex.stream);
  CgScalars* sc = reinterpret_cast<CgScalars*>(w.scal.get());
  SI_CUDA(cudaMemsetAsync(y, 0, sizeof(double) * sz, ex.stream));
  SI_CUDA(cudaMemcpyAsync(w.r.get(), b, sizeof(double) * sz, cudaMemcpyDeviceToDevice, ex.stream));
  SI_CUDA(cudaMemcpyAsync(w.p.get(), b, sizeof(double) * sz, cudaMemcpyDeviceToDevice, ex.stream));
  k_cg_init<<<grid_red, kCgT, 0, ex.stream>>>(b, m, ld, n, w.partial.get(), w.counter.get(), sc);
  SI_LAUNCH_CHECK();
  const double tol2 = rtol * rtol;
  const int grid_el = cg_grid(ex, n * m);
  Epilogue<double> ep;
  int it = 0;
  constexpr int kCheck = 16;
  while (it < maxit) {
    for (int j = 0; j < kCheck && it < maxit; ++j, ++it) {
      spmm_dev<double>(ex, M, w.p.get(), w.q.get(), ld, m, ep);
      k_cg_alpha<<<grid_red, kCgT, 0, ex.stream>>>(w.p.get(), w.q.get(), m, ld, n, w.partial.get(), w.counter.get(),
                                                   sc);
      SI_LAUNCH_CHECK();
      k_cg_update<<<grid_red, kCgT, 0, ex.stream>>>(y, w.r.get(), w.p.get(), w.q.get(), m, ld, n, tol2,
                                                    w.partial.get(), w.counter.get(), sc);
      SI_LAUNCH_CHECK();
      k_cg_dir<<<grid_el, kCgT, 0, ex.stream>>>(w.p.get(), w.r.get(), m, ld, n, sc);
      SI_LAUNCH_CHECK();
    }
    int act = 0;
    SI_CUDA(cudaMemcpyAsync(&act, &sc->n_active, sizeof(int), cudaMemcpyDeviceToHost, ex.stream));
    SI_CUDA(cudaStreamSynchronize(ex.stream));
    if (act == 0) {
      if (converged != nullptr) *converged = true;
      return it;
    }
  }
  if (converged != nullptr) {
    int act = 1;
    SI_CUDA(cudaMemcpyAsync(&act, &sc->n_active, sizeof(int), cudaMemcpyDeviceToHost, ex.stream));
    SI_CUDA(cudaStreamSynchronize(ex.stream));
    *converged = act == 0;
  }
  return it;
}

}  // namespace si
