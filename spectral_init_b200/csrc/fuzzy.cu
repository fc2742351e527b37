// Fuzzy-kNN graph construction on the device: the UMAP fuzzy simplicial set
// the crate consumes, built as its fixture generator builds it
// (tests/generate_fixtures.py:70-182 of the reference):
//   1. exact kNN, Euclidean, self excluded, ascending (ties by index);
//   2. smooth-kNN sigma / rho (umap-learn 0.5.11 smooth_knn_dist, as the
//      generator ran it: bisection for sum_{j>0} exp(-max(d - rho, 0) / sigma)
//      = log2(k) from sigma = 1, taking the midpoint against an infinite upper
//      bound, so a row whose root lies above 1 keeps sigma = +inf; floor
//      1e-3 x the row's (or all rows') mean distance);
//   3. membership strengths exp(-(d - rho) / sigma), 1 at or below rho;
//   4. the fuzzy union A + A^T - A∘A^T;
//   5. pruning below max / n_epochs (500 for n <= 10000, else 200).
// Distances in f64, reported as f32 like the generator's; sigma / rho f32
// with the bisection in f64; memberships f32.
#include <cuda_runtime.h>

#include <algorithm>
#include <cfloat>
#include <cmath>

#include "si_internal.h"

namespace si {
namespace {

constexpr int kKnnMax = 32;
constexpr int kKnnThreads = 128;
constexpr int kKnnTile = 64;  // candidate rows staged per tile

int grid_items(const Exec& ex, int64_t items, int threads = 256) {
  const int64_t need = (items + threads - 1) / threads;
  return static_cast<int>(std::max<int64_t>(1, std::min<int64_t>(need, int64_t(ex.sms) * 16)));
}

// Stage 1: one query row per thread, candidates streamed through shared
// memory in tiles; the K nearest kept sorted in registers (a candidate goes
// after every kept one at the same distance, so ties keep index order).
template <int K>
__global__ void __launch_bounds__(kKnnThreads) k_knn_exact(const double* __restrict__ x, int64_t n, int d, int k,
                                                           int32_t* __restrict__ idx, float* __restrict__ dist) {
  extern __shared__ double tile[];  // kKnnTile x d
  const int64_t q = static_cast<int64_t>(blockIdx.x) * kKnnThreads + threadIdx.x;
  double bd[K];
  int32_t bi[K];
#pragma unroll
  for (int t = 0; t < K; ++t) {
    bd[t] = INFINITY;
    bi[t] = -1;
  }
  for (int64_t c0 = 0; c0 < n; c0 += kKnnTile) {
    const int cn = static_cast<int>(std::min<int64_t>(kKnnTile, n - c0));
    __syncthreads();
    for (int t = threadIdx.x; t < cn * d; t += kKnnThreads) tile[t] = x[c0 * d + t];
    __syncthreads();
    if (q >= n) continue;
    for (int c = 0; c < cn; ++c) {
      const int64_t j = c0 + c;
      if (j == q) continue;
      double s = 0.0;
      for (int f = 0; f < d; ++f) {
        const double df = x[q * d + f] - tile[c * d + f];
        s = fma(df, df, s);
      }
      if (!(s < bd[K - 1])) continue;
      // insert (s, j) after every kept entry with a distance <= s
      double cd = s;
      int32_t ci = static_cast<int32_t>(j);
#pragma unroll
      for (int t = 0; t < K; ++t) {
        if (cd < bd[t]) {
          const double td = bd[t];
          const int32_t ti = bi[t];
          bd[t] = cd;
          bi[t] = ci;
          cd = td;
          ci = ti;
        }
      }
    }
  }
  if (q >= n) return;
  for (int t = 0; t < k; ++t) {
    idx[q * k + t] = bi[t];
    dist[q * k + t] = static_cast<float>(sqrt(bd[t]));
  }
}

// mean of all distances (f64 sum in row order, one block)
__global__ void k_dist_mean(const float* __restrict__ dist, int64_t total, double* __restrict__ out) {
  __shared__ double red[256];
  double s = 0.0;
  for (int64_t e = threadIdx.x; e < total; e += blockDim.x) s += static_cast<double>(dist[e]);
  red[threadIdx.x] = s;
  __syncthreads();
  for (int o = 128; o > 0; o >>= 1) {
    if (threadIdx.x < o) red[threadIdx.x] += red[threadIdx.x + o];
    __syncthreads();
  }
  if (threadIdx.x == 0) out[0] = red[0] / static_cast<double>(total > 0 ? total : 1);
}

// Stage 2: one row per thread
__global__ void k_smooth_knn(const float* __restrict__ dist, int64_t n, int k, const double* __restrict__ mean_all,
                             float* __restrict__ sigma, float* __restrict__ rho) {
  const double target = log2(static_cast<double>(k));
  const int64_t stride = static_cast<int64_t>(gridDim.x) * blockDim.x;
  for (int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += stride) {
    const float* row = dist + i * k;
    float r = 0.0f;
    double rsum = 0.0;
    for (int j = 0; j < k; ++j) {
      rsum += static_cast<double>(row[j]);
      if (r == 0.0f && row[j] > 0.0f) r = row[j];
    }
    double lo = 0.0, hi = INFINITY, mid = 1.0;
    for (int it = 0; it < 64; ++it) {
      double psum = 0.0;
      for (int j = 1; j < k; ++j) {
        const float dd = row[j] - r;
        psum += dd > 0.0f ? exp(-(static_cast<double>(dd) / mid)) : 1.0;
      }
      if (fabs(psum - target) < 1e-5) break;
      if (psum > target) {
        hi = mid;
        mid = (lo + hi) / 2.0;
      } else {
        lo = mid;
        mid = (lo + hi) / 2.0;  // an infinite upper bound keeps mid infinite (see above)
      }
    }
    const double floor = 1e-3 * (r > 0.0f ? rsum / k : mean_all[0]);
    sigma[i] = static_cast<float>(mid < floor ? floor : mid);
    rho[i] = r;
  }
}

// Stage 3: membership of neighbour t of row i (0 for the row itself)
__device__ __forceinline__ float membership_of(const int32_t* idx, const float* dist, const float* sigma,
                                               const float* rho, int k, int64_t i, int t) {
  const int32_t j = idx[i * k + t];
  if (j == i || j < 0) return 0.0f;
  const float diff = dist[i * k + t] - rho[i];
  const float sg = sigma[i];
  if (diff <= 0.0f || sg == 0.0f) return 1.0f;
  return expf(-(diff / sg));
}

// membership of the reverse edge j -> i (0 when i is not among j's neighbours)
__device__ __forceinline__ float reverse_membership(const int32_t* idx, const float* dist, const float* sigma,
                                                    const float* rho, int k, int64_t i, int64_t j) {
  for (int t = 0; t < k; ++t)
    if (idx[j * k + t] == i) return membership_of(idx, dist, sigma, rho, k, j, t);
  return 0.0f;
}

// Stage 4, counting: every directed edge i -> j with a > 0 gives (i, j); it
// also gives (j, i) when j -> i is absent (its union value is then a).  Each
// (row, column) pair of the union arises exactly once.
__global__ void k_union_count(const int32_t* __restrict__ idx, const float* __restrict__ dist,
                              const float* __restrict__ sigma, const float* __restrict__ rho, int64_t n, int k,
                              unsigned long long* __restrict__ counts) {
  const int64_t total = n * k;
  const int64_t stride = static_cast<int64_t>(gridDim.x) * blockDim.x;
  for (int64_t e = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; e < total; e += stride) {
    const int64_t i = e / k;
    const int t = static_cast<int>(e % k);
    const float a = membership_of(idx, dist, sigma, rho, k, i, t);
    if (a == 0.0f) continue;
    const int64_t j = idx[e];
    atomicAdd(counts + i, 1ull);
    if (reverse_membership(idx, dist, sigma, rho, k, i, j) == 0.0f) atomicAdd(counts + j, 1ull);
  }
}

// Stage 4, filling: union value (a + b) - a b in f32 as scipy forms it
__global__ void k_union_fill(const int32_t* __restrict__ idx, const float* __restrict__ dist,
                             const float* __restrict__ sigma, const float* __restrict__ rho, int64_t n, int k,
                             const uint64_t* __restrict__ ptr, unsigned long long* __restrict__ cursor,
                             uint32_t* __restrict__ cols, float* __restrict__ vals) {
  const int64_t total = n * k;
  const int64_t stride = static_cast<int64_t>(gridDim.x) * blockDim.x;
  for (int64_t e = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; e < total; e += stride) {
    const int64_t i = e / k;
    const int t = static_cast<int>(e % k);
    const float a = membership_of(idx, dist, sigma, rho, k, i, t);
    if (a == 0.0f) continue;
    const int64_t j = idx[e];
    const float b = reverse_membership(idx, dist, sigma, rho, k, i, j);
    const float u = (a + b) - a * b;
    const uint64_t p = ptr[i] + atomicAdd(cursor + i, 1ull);
    cols[p] = static_cast<uint32_t>(j);
    vals[p] = u;
    if (b == 0.0f) {
      const uint64_t q = ptr[j] + atomicAdd(cursor + j, 1ull);
      cols[q] = static_cast<uint32_t>(i);
      vals[q] = u;
    }
  }
}

// each row's entries in column order (the fill order above is not fixed)
__global__ void k_sort_rows(int64_t n, const uint64_t* __restrict__ ptr, uint32_t* __restrict__ cols,
                            float* __restrict__ vals) {
  const int64_t stride = static_cast<int64_t>(gridDim.x) * blockDim.x;
  for (int64_t r = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; r < n; r += stride) {
    const uint64_t s = ptr[r], e = ptr[r + 1];
    for (uint64_t a = s + 1; a < e; ++a) {
      const uint32_t c = cols[a];
      const float v = vals[a];
      uint64_t b = a;
      while (b > s && cols[b - 1] > c) {
        cols[b] = cols[b - 1];
        vals[b] = vals[b - 1];
        --b;
      }
      cols[b] = c;
      vals[b] = v;
    }
  }
}

__global__ void k_max_f32(const float* __restrict__ v, int64_t count, float* __restrict__ out) {
  __shared__ float red[256];
  float m = 0.0f;
  for (int64_t e = threadIdx.x; e < count; e += blockDim.x) m = fmaxf(m, v[e]);
  red[threadIdx.x] = m;
  __syncthreads();
  for (int o = 128; o > 0; o >>= 1) {
    if (threadIdx.x < o) red[threadIdx.x] = fmaxf(red[threadIdx.x], red[threadIdx.x + o]);
    __syncthreads();
  }
  if (threadIdx.x == 0) out[0] = red[0];
}

// Stage 5a: entries kept per row, then the compacted CSR
__global__ void k_prune_count(int64_t n, const uint64_t* __restrict__ ptr, const float* __restrict__ vals,
                              const float* __restrict__ vmax, float n_epochs, unsigned long long* __restrict__ keep) {
  const float thr = vmax[0] / n_epochs;
  const int64_t stride = static_cast<int64_t>(gridDim.x) * blockDim.x;
  for (int64_t r = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; r <= n; r += stride) {
    if (r == n) {
      keep[n] = 0;
      continue;
    }
    unsigned long long c = 0;
    for (uint64_t p = ptr[r]; p < ptr[r + 1]; ++p) c += (vals[p] < thr) ? 0 : 1;
    keep[r] = c;
  }
}

__global__ void k_prune_fill(int64_t n, const uint64_t* __restrict__ ptr, const uint32_t* __restrict__ cols,
                             const float* __restrict__ vals, const float* __restrict__ vmax, float n_epochs,
                             const uint64_t* __restrict__ optr, uint32_t* __restrict__ ocols,
                             float* __restrict__ ovals) {
  const float thr = vmax[0] / n_epochs;
  const int64_t stride = static_cast<int64_t>(gridDim.x) * blockDim.x;
  for (int64_t r = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; r < n; r += stride) {
    uint64_t o = optr[r];
    for (uint64_t p = ptr[r]; p < ptr[r + 1]; ++p) {
      if (vals[p] < thr) continue;
      ocols[o] = cols[p];
      ovals[o] = vals[p];
      ++o;
    }
  }
}

}  // namespace

void fuzzy_graph_dev(const Exec& ex, const double* x, int64_t n, int d, int k, int32_t* knn_idx, float* knn_dist,
                     float* sigma, float* rho, uint64_t* indptr, uint32_t* indices, float* data, uint64_t capacity,
                     uint64_t* nnz_out) {
  SI_REQUIRE(n >= 2 && d >= 1 && k >= 1 && k < n, SI_INVALID_ARGUMENT, "fuzzy graph: need n >= 2, d >= 1, 1 <= k < n");
  SI_REQUIRE(k <= kKnnMax, SI_INVALID_ARGUMENT, "fuzzy graph: k must be at most 32");
  SI_REQUIRE(d <= 256, SI_INVALID_ARGUMENT, "fuzzy graph: at most 256 features");
  SI_REQUIRE(n < (int64_t(1) << 31), SI_INVALID_ARGUMENT, "fuzzy graph: n must fit in int32");
  // 1. exact kNN
  const int smem = kKnnTile * d * static_cast<int>(sizeof(double));
  const unsigned grid = static_cast<unsigned>((n + kKnnThreads - 1) / kKnnThreads);
  if (k <= 16) {
    SI_CUDA(cudaFuncSetAttribute(k_knn_exact<16>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
    k_knn_exact<16><<<grid, kKnnThreads, smem, ex.stream>>>(x, n, d, k, knn_idx, knn_dist);
  } else {
    SI_CUDA(cudaFuncSetAttribute(k_knn_exact<32>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
    k_knn_exact<32><<<grid, kKnnThreads, smem, ex.stream>>>(x, n, d, k, knn_idx, knn_dist);
  }
  SI_LAUNCH_CHECK();
  // 2. smooth-kNN
  DevBuf<double> mean_all(1, ex.stream);
  k_dist_mean<<<1, 256, 0, ex.stream>>>(knn_dist, n * k, mean_all.get());
  SI_LAUNCH_CHECK();
  k_smooth_knn<<<grid_items(ex, n), 256, 0, ex.stream>>>(knn_dist, n, k, mean_all.get(), sigma, rho);
  SI_LAUNCH_CHECK();
  // 3 + 4. memberships and their fuzzy union as CSR
  DevBuf<unsigned long long> cnt(static_cast<size_t>(n + 1), ex.stream);
  cnt.zero();
  k_union_count<<<grid_items(ex, n * k), 256, 0, ex.stream>>>(knn_idx, knn_dist, sigma, rho, n, k, cnt.get());
  SI_LAUNCH_CHECK();
  DevBuf<uint64_t> uptr(static_cast<size_t>(n + 1), ex.stream);
  const uint64_t unnz = exclusive_scan_u64(ex, reinterpret_cast<const uint64_t*>(cnt.get()), uptr.get(), n);
  DevBuf<uint32_t> ucols(std::max<uint64_t>(unnz, 1), ex.stream);
  DevBuf<float> uvals(std::max<uint64_t>(unnz, 1), ex.stream);
  cnt.zero();
  k_union_fill<<<grid_items(ex, n * k), 256, 0, ex.stream>>>(knn_idx, knn_dist, sigma, rho, n, k, uptr.get(),
                                                               cnt.get(), ucols.get(), uvals.get());
  SI_LAUNCH_CHECK();
  k_sort_rows<<<grid_items(ex, n), 256, 0, ex.stream>>>(n, uptr.get(), ucols.get(), uvals.get());
  SI_LAUNCH_CHECK();
  // 5a. pruning
  DevBuf<float> vmax(1, ex.stream);
  k_max_f32<<<1, 256, 0, ex.stream>>>(uvals.get(), static_cast<int64_t>(unnz), vmax.get());
  SI_LAUNCH_CHECK();
  const float n_epochs = n <= 10000 ? 500.0f : 200.0f;
  k_prune_count<<<grid_items(ex, n + 1), 256, 0, ex.stream>>>(n, uptr.get(), uvals.get(), vmax.get(), n_epochs,
                                                              cnt.get());
  SI_LAUNCH_CHECK();
  const uint64_t pnnz = exclusive_scan_u64(ex, reinterpret_cast<const uint64_t*>(cnt.get()), indptr, n);
  SI_REQUIRE(pnnz <= capacity, SI_INVALID_ARGUMENT, "fuzzy graph: output capacity too small (need 2 n k entries)");
  k_prune_fill<<<grid_items(ex, n), 256, 0, ex.stream>>>(n, uptr.get(), ucols.get(), uvals.get(), vmax.get(), n_epochs,
                                                        indptr, indices, data);
  SI_LAUNCH_CHECK();
  SI_CUDA(cudaStreamSynchronize(ex.stream));
  *nnz_out = pnnz;
}

}  // namespace si
