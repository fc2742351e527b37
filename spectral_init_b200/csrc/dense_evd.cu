// Dense symmetric eigensolver on the device for the k smallest eigenpairs
// (dense_evd, src/solvers/dense.rs:9-46; Levels 0 and 5 of the chain).
//
//   1. densify the operator (lower triangle mirrored, like faer's Side::Lower);
//   2. Householder tridiagonalisation T = Q^T A Q (dsytd2-style, one CTA,
//      matrix resident in L2 for n <= 2000);
//   3. split T where off-diagonals are negligible, then for every block the
//      smallest eigenvalues by Sturm-count bisection; the k smallest overall
//      are kept;
//   4. eigenvectors of T by inverse iteration restricted to the block (LU with
//      partial pivoting of T - lambda I), re-orthogonalised within clusters of
//      close eigenvalues (modified Gram-Schmidt);
//   5. back-transformation v = Q y with the stored reflectors.
#include <cfloat>

#include "si_internal.h"

namespace si {
namespace {

constexpr int DT = 1024;
constexpr int64_t kTriMultiMin = 192;  // from this n the tridiagonalisation runs as multi-CTA steps

__global__ void k_densify(int64_t n, const uint64_t* __restrict__ indptr, const uint32_t* __restrict__ indices,
                          const double* __restrict__ vals, double diag, double* __restrict__ A) {
  const int64_t stride = static_cast<int64_t>(gridDim.x) * blockDim.x;
  for (int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; i < n; i += stride) {
    for (uint64_t k = indptr[i]; k < indptr[i + 1]; ++k) A[i * n + indices[k]] += vals[k];
    A[i * n + i] += diag;
  }
}

// A[i][j] = A[j][i] for i < j (use the lower triangle).
__global__ void k_mirror_lower(int64_t n, double* A) {
  const int64_t total = n * n;
  const int64_t stride = static_cast<int64_t>(gridDim.x) * blockDim.x;
  for (int64_t t = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; t < total; t += stride) {
    const int64_t i = t / n, j = t % n;
    if (i < j) A[i * n + j] = A[j * n + i];
  }
}

__device__ double block_sum_all(double v, double* red) {
  v = warp_sum(v);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = v;
  __syncthreads();
  double t = 0.0;
  const int nw = blockDim.x >> 5;
  for (int i = 0; i < nw; ++i) t += red[i];
  __syncthreads();
  return t;
}

__global__ void __launch_bounds__(DT) k_tridiag(double* A, int n, double* d, double* e, double* tau) {
  extern __shared__ double sm[];
  double* v = sm;
  double* w = sm + n;
  __shared__ double red[32];
  __shared__ double s_tau, s_scal;
  const int tid = threadIdx.x, nt = blockDim.x, lane = tid & 31, warp = tid >> 5, nwarps = nt >> 5;
  for (int j = 0; j + 2 < n; ++j) {
    double part = 0.0;
    for (int i = j + 2 + tid; i < n; i += nt) {
      const double x = A[static_cast<int64_t>(i) * n + j];
      part += x * x;
    }
    const double sigma = block_sum_all(part, red);
    if (tid == 0) {
      const double alpha = A[static_cast<int64_t>(j + 1) * n + j];
      double t = 0.0, beta = alpha, scal = 0.0;
      if (sigma > 0.0) {
        const double nrm = sqrt(alpha * alpha + sigma);
        beta = alpha >= 0.0 ? -nrm : nrm;
        t = (beta - alpha) / beta;
        scal = 1.0 / (alpha - beta);
      }
      s_tau = t;
      s_scal = scal;
      e[j] = beta;
      tau[j] = t;
      d[j] = A[static_cast<int64_t>(j) * n + j];
    }
    __syncthreads();
    const double t = s_tau;
    if (t == 0.0) continue;
    const double scal = s_scal;
    for (int i = j + 1 + tid; i < n; i += nt) {
      const double vi = (i == j + 1) ? 1.0 : A[static_cast<int64_t>(i) * n + j] * scal;
      v[i] = vi;
      if (i >= j + 2) A[static_cast<int64_t>(j) * n + i] = vi;  // keep the reflector in row j
    }
    __syncthreads();
    for (int r = j + 1 + warp; r < n; r += nwarps) {
      double acc = 0.0;
      const double* row = A + static_cast<int64_t>(r) * n;
      for (int c = j + 1 + lane; c < n; c += 32) acc = fma(row[c], v[c], acc);
      acc = warp_sum(acc);
      if (lane == 0) w[r] = t * acc;
    }
    __syncthreads();
    part = 0.0;
    for (int r = j + 1 + tid; r < n; r += nt) part += w[r] * v[r];
    const double K = 0.5 * t * block_sum_all(part, red);
    for (int r = j + 1 + tid; r < n; r += nt) w[r] -= K * v[r];
    __syncthreads();
    const int len = n - j - 1;
    for (int idx = tid; idx < len * len; idx += nt) {
      const int r = j + 1 + idx / len, c = j + 1 + idx % len;
      A[static_cast<int64_t>(r) * n + c] -= v[r] * w[c] + w[r] * v[c];
    }
    __syncthreads();
  }
  if (tid == 0) {
    if (n >= 2) {
      d[n - 2] = A[static_cast<int64_t>(n - 2) * n + n - 2];
      e[n - 2] = A[static_cast<int64_t>(n - 1) * n + n - 2];
      tau[n - 2] = 0.0;
    }
    d[n - 1] = A[static_cast<int64_t>(n - 1) * n + n - 1];
  }
}

// ---- multi-CTA tridiagonalisation: the same Householder steps as k_tridiag,
// each step three launches so the trailing-matrix passes use the whole GPU.
// Step j:  (1) one CTA forms the reflector of column j (d, e, tau; v in vbuf
// and in row j of A); (2) w = tau A v over the trailing rows, one warp per
// row, per-CTA partial dots w.v, the last CTA subtracts K v with
// K = tau (w.v) / 2 (deterministic order); (3) A -= v w^T + w v^T.
__global__ void __launch_bounds__(256) k_tri_house(double* A, int n, int j, double* d, double* e, double* tau,
                                                   double* vbuf) {
  __shared__ double red[32];
  __shared__ double s_tau, s_scal;
  const int tid = threadIdx.x;
  double part = 0.0;
  for (int i = j + 2 + tid; i < n; i += blockDim.x) {
    const double x = A[static_cast<int64_t>(i) * n + j];
    part += x * x;
  }
  const double sigma = block_sum_all(part, red);
  if (tid == 0) {
    const double alpha = A[static_cast<int64_t>(j + 1) * n + j];
    double t = 0.0, beta = alpha, scal = 0.0;
    if (sigma > 0.0) {
      const double nrm = sqrt(alpha * alpha + sigma);
      beta = alpha >= 0.0 ? -nrm : nrm;
      t = (beta - alpha) / beta;
      scal = 1.0 / (alpha - beta);
    }
    s_tau = t;
    s_scal = scal;
    e[j] = beta;
    tau[j] = t;
    d[j] = A[static_cast<int64_t>(j) * n + j];
  }
  __syncthreads();
  if (s_tau == 0.0) return;
  const double scal = s_scal;
  for (int i = j + 1 + tid; i < n; i += blockDim.x) {
    const double vi = (i == j + 1) ? 1.0 : A[static_cast<int64_t>(i) * n + j] * scal;
    vbuf[i] = vi;
    if (i >= j + 2) A[static_cast<int64_t>(j) * n + i] = vi;  // keep the reflector in row j
  }
}

__global__ void __launch_bounds__(256) k_tri_matvec(const double* __restrict__ A, int n, int j,
                                                    const double* __restrict__ tau, const double* __restrict__ vbuf,
                                                    double* __restrict__ wbuf, double* __restrict__ partial,
                                                    unsigned* __restrict__ counter) {
  __shared__ double red[8];
  __shared__ bool last;
  const double t = tau[j];
  if (t == 0.0) return;  // uniform for the grid
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int r = j + 1 + blockIdx.x * 8 + warp;
  double wv = 0.0;
  if (r < n) {
    double acc = 0.0;
    const double* row = A + static_cast<int64_t>(r) * n;
    for (int c = j + 1 + lane; c < n; c += 32) acc = fma(row[c], vbuf[c], acc);
    acc = warp_sum(acc);
    if (lane == 0) {
      wbuf[r] = t * acc;
      wv = t * acc * vbuf[r];
    }
  }
  if (lane == 0) red[warp] = wv;
  __syncthreads();
  if (threadIdx.x == 0) {
    double s = 0.0;
    for (int w = 0; w < 8; ++w) s += red[w];
    partial[blockIdx.x] = s;
  }
  __threadfence();
  __syncthreads();
  if (threadIdx.x == 0) last = atomicAdd(counter, 1u) == gridDim.x - 1;
  __syncthreads();
  if (!last) return;
  __threadfence();
  __shared__ double s_k;
  if (threadIdx.x == 0) {
    double s = 0.0;
    for (int b = 0; b < static_cast<int>(gridDim.x); ++b) s += __ldcg(&partial[b]);
    s_k = 0.5 * t * s;
    *counter = 0u;
  }
  __syncthreads();
  const double K = s_k;
  for (int i = j + 1 + threadIdx.x; i < n; i += blockDim.x) wbuf[i] = __ldcg(&wbuf[i]) - K * vbuf[i];
}

__global__ void __launch_bounds__(256) k_tri_update(double* __restrict__ A, int n, int j,
                                                    const double* __restrict__ tau, const double* __restrict__ vbuf,
                                                    const double* __restrict__ wbuf) {
  if (tau[j] == 0.0) return;
  for (int r = j + 1 + blockIdx.x; r < n; r += gridDim.x) {
    const double vr = vbuf[r], wr = wbuf[r];
    double* row = A + static_cast<int64_t>(r) * n;
    for (int c = j + 1 + threadIdx.x; c < n; c += blockDim.x) row[c] -= vr * wbuf[c] + wr * vbuf[c];
  }
}

__global__ void k_tri_last(const double* A, int n, double* d, double* e, double* tau) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  if (n >= 2) {
    d[n - 2] = A[static_cast<int64_t>(n - 2) * n + n - 2];
    e[n - 2] = A[static_cast<int64_t>(n - 1) * n + n - 2];
    tau[n - 2] = 0.0;
  }
  d[n - 1] = A[static_cast<int64_t>(n - 1) * n + n - 1];
}

// number of eigenvalues of T[l..r] smaller than x (Sturm sequence)
__device__ int sturm_count(const double* d, const double* e, int l, int r, double x, double pivmin) {
  int cnt = 0;
  double q = d[l] - x;
  if (fabs(q) < pivmin) q = -pivmin;
  if (q < 0.0) ++cnt;
  for (int i = l + 1; i <= r; ++i) {
    q = d[i] - x - e[i - 1] * e[i - 1] / q;
    if (fabs(q) < pivmin) q = -pivmin;
    if (q < 0.0) ++cnt;
  }
  return cnt;
}

struct TriWork {
  int* bstart;      // [n + 1]
  double* es;       // [n] split off-diagonals
  double* cand;     // [n * k]
  int* cand_blk;    // [n * k]
  double* lu;       // [5 * n]
  int* piv;         // [n]
  double* xv;       // [n]
  int* sel_blk;     // [k]
  double* sel_val;  // [k]
};

__global__ void __launch_bounds__(DT) k_tri_eig(const double* __restrict__ d, const double* __restrict__ e, int n,
                                                int k, TriWork w, double* evals_out, double* Y, int ld) {
  __shared__ int s_nb;
  __shared__ double s_tnorm;
  const int tid = threadIdx.x;
  if (tid == 0) {
    double tn = 0.0;
    for (int i = 0; i < n; ++i) {
      const double rs = fabs(d[i]) + (i > 0 ? fabs(e[i - 1]) : 0.0) + (i + 1 < n ? fabs(e[i]) : 0.0);
      tn = fmax(tn, rs);
    }
    s_tnorm = tn;
    int nb = 0;
    w.bstart[nb++] = 0;
    for (int i = 0; i + 1 < n; ++i) {
      const double off = fabs(e[i]);
      if (off <= DBL_EPSILON * (fabs(d[i]) + fabs(d[i + 1])) || off <= 1e-300) {
        w.es[i] = 0.0;
        w.bstart[nb++] = i + 1;
      } else {
        w.es[i] = e[i];
      }
    }
    w.bstart[nb] = n;
    s_nb = nb;
  }
  __syncthreads();
  const int nb = s_nb;
  const double tnorm = s_tnorm;
  const double pivmin = fmax(DBL_MIN, tnorm * tnorm * DBL_MIN);
  // bisection for (block, index) items
  for (int q = tid; q < nb * k; q += blockDim.x) {
    const int b = q / k, t = q % k;
    const int l = w.bstart[b], r = w.bstart[b + 1] - 1;
    if (t > r - l) {
      w.cand[q] = DBL_MAX;
      w.cand_blk[q] = b;
      continue;
    }
    double lo = DBL_MAX, hi = -DBL_MAX;
    for (int i = l; i <= r; ++i) {
      const double rad = (i > l ? fabs(w.es[i - 1]) : 0.0) + (i < r ? fabs(w.es[i]) : 0.0);
      lo = fmin(lo, d[i] - rad);
      hi = fmax(hi, d[i] + rad);
    }
    lo -= 2.0 * DBL_EPSILON * tnorm + pivmin;
    hi += 2.0 * DBL_EPSILON * tnorm + pivmin;
    for (int it = 0; it < 200; ++it) {
      const double mid = 0.5 * (lo + hi);
      if (hi - lo <= 2.0 * DBL_EPSILON * fmax(fabs(lo), fabs(hi)) + pivmin || mid == lo || mid == hi) break;
      if (sturm_count(d, w.es, l, r, mid, pivmin) > t) hi = mid; else lo = mid;
    }
    w.cand[q] = 0.5 * (lo + hi);
    w.cand_blk[q] = b;
  }
  __syncthreads();
  if (tid != 0) return;
  // k smallest candidates (stable)
  int nsel = 0;
  for (int s = 0; s < k; ++s) {
    int best = -1;
    for (int q = 0; q < nb * k; ++q) {
      if (w.cand[q] == DBL_MAX) continue;
      bool taken = false;
      for (int u = 0; u < nsel; ++u)
        if (w.sel_blk[u] == q) taken = true;
      if (taken) continue;
      if (best < 0 || w.cand[q] < w.cand[best]) best = q;
    }
    if (best < 0) break;
    w.sel_blk[nsel++] = best;
  }
  for (int s = 0; s < nsel; ++s) {
    const int q = w.sel_blk[s];
    evals_out[s] = w.cand[q];
    w.sel_val[s] = w.cand[q];
  }
  const double tiny = DBL_EPSILON * fmax(tnorm, DBL_MIN);
  double* D = w.lu;
  double* DL = w.lu + n;
  double* DU = w.lu + 2 * n;
  double* DU2 = w.lu + 3 * n;
  for (int s = 0; s < nsel; ++s) {
    const int q = w.sel_blk[s];
    const int b = w.cand_blk[q];
    const int l = w.bstart[b], r = w.bstart[b + 1] - 1, sz = r - l + 1;
    const double lam = w.cand[q];
    double bnorm = 0.0;
    for (int i = l; i <= r; ++i)
      bnorm = fmax(bnorm, fabs(d[i]) + (i > l ? fabs(w.es[i - 1]) : 0.0) + (i < r ? fabs(w.es[i]) : 0.0));
    // LU with partial pivoting of T_b - lam I
    for (int i = 0; i < sz; ++i) {
      D[i] = d[l + i] - lam;
      DU[i] = (i + 1 < sz) ? w.es[l + i] : 0.0;
      DL[i] = DU[i];
      DU2[i] = 0.0;
    }
    for (int i = 0; i + 1 < sz; ++i) {
      if (fabs(D[i]) >= fabs(DL[i])) {
        if (D[i] == 0.0) D[i] = tiny;
        const double f = DL[i] / D[i];
        DL[i] = f;
        D[i + 1] -= f * DU[i];
        w.piv[i] = 0;
      } else {
        const double f = D[i] / DL[i];
        D[i] = DL[i];
        DL[i] = f;
        const double tmp = DU[i];
        DU[i] = D[i + 1];
        D[i + 1] = tmp - f * D[i + 1];
        if (i + 2 < sz) {
          DU2[i] = DU[i + 1];
          DU[i + 1] = -f * DU[i + 1];
        }
        w.piv[i] = 1;
      }
    }
    for (int i = 0; i < sz; ++i)
      if (fabs(D[i]) < tiny) D[i] = D[i] < 0.0 ? -tiny : tiny;
    // start vector
    for (int i = 0; i < sz; ++i) {
      double z0, z1;
      philox_normal2(0x0de75eedull + s, 7, static_cast<uint64_t>(i), z0, z1);
      w.xv[i] = z0;
    }
    for (int it = 0; it < 4; ++it) {
      // solve (T - lam I) y = x in place
      double* x = w.xv;
      for (int i = 0; i + 1 < sz; ++i) {
        if (w.piv[i] == 0) {
          x[i + 1] -= DL[i] * x[i];
        } else {
          const double tmp = x[i];
          x[i] = x[i + 1];
          x[i + 1] = tmp - DL[i] * x[i];
        }
      }
      x[sz - 1] /= D[sz - 1];
      if (sz >= 2) x[sz - 2] = (x[sz - 2] - DU[sz - 2] * x[sz - 1]) / D[sz - 2];
      for (int i = sz - 3; i >= 0; --i) x[i] = (x[i] - DU[i] * x[i + 1] - DU2[i] * x[i + 2]) / D[i];
      // re-orthogonalise against earlier vectors of the same block in the cluster
      for (int u = 0; u < s; ++u) {
        const int qu = w.sel_blk[u];
        if (w.cand_blk[qu] != b) continue;
        if (fabs(w.sel_val[u] - lam) > 1e-3 * bnorm) continue;
        double dot = 0.0;
        for (int i = 0; i < sz; ++i) dot += Y[static_cast<int64_t>(l + i) * ld + u] * x[i];
        for (int i = 0; i < sz; ++i) x[i] -= dot * Y[static_cast<int64_t>(l + i) * ld + u];
      }
      double nrm = 0.0;
      for (int i = 0; i < sz; ++i) nrm += x[i] * x[i];
      nrm = sqrt(nrm);
      if (!(nrm > 0.0)) {
        for (int i = 0; i < sz; ++i) x[i] = (i == s % sz) ? 1.0 : 0.0;
        nrm = 1.0;
      }
      for (int i = 0; i < sz; ++i) x[i] /= nrm;
    }
    for (int i = 0; i < n; ++i) Y[static_cast<int64_t>(i) * ld + s] = 0.0;
    for (int i = 0; i < sz; ++i) Y[static_cast<int64_t>(l + i) * ld + s] = w.xv[i];
  }
}

// Y <- Q Y with Q = H_0 H_1 ... H_{n-3}; reflector j: u = (1, A[j][j+2..n)) on rows j+1..n-1.
__global__ void __launch_bounds__(DT) k_backtransform(const double* __restrict__ A, const double* __restrict__ tau,
                                                      int n, double* Y, int ld, int k) {
  __shared__ double dots[MAXM];
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5, nwarps = blockDim.x >> 5;
  for (int j = n - 3; j >= 0; --j) {
    const double t = tau[j];
    if (t == 0.0) continue;
    for (int v = warp; v < k; v += nwarps) {
      double acc = 0.0;
      for (int r = j + 1 + lane; r < n; r += 32) {
        const double u = (r == j + 1) ? 1.0 : A[static_cast<int64_t>(j) * n + r];
        acc = fma(u, Y[static_cast<int64_t>(r) * ld + v], acc);
      }
      acc = warp_sum(acc);
      if (lane == 0) dots[v] = t * acc;
    }
    __syncthreads();
    const int len = n - j - 1;
    for (int idx = tid; idx < len * k; idx += blockDim.x) {
      const int r = j + 1 + idx / k, v = idx % k;
      const double u = (r == j + 1) ? 1.0 : A[static_cast<int64_t>(j) * n + r];
      Y[static_cast<int64_t>(r) * ld + v] -= dots[v] * u;
    }
    __syncthreads();
  }
}

}  // namespace

void dense_evd_dev(const Exec& ex, const OpDev& op, int k, double* evals_host, double* evecs, int ld) {
  const int64_t n = op.n;
  SI_REQUIRE(n >= 1 && k >= 1 && k <= n && k <= MAXM, SI_INVALID_ARGUMENT, "dense_evd: bad sizes");
  SI_REQUIRE(op.v64 != nullptr || op.nnz == 0, SI_INVALID_ARGUMENT, "dense_evd: f64 values required");
  DevBuf<double> A(static_cast<size_t>(n) * n, ex.stream), d(n, ex.stream), e(n, ex.stream), tau(n, ex.stream),
      ev(MAXM, ex.stream);
  A.zero();
  const int grid = static_cast<int>(std::max<int64_t>(1, std::min<int64_t>((n + 255) / 256, int64_t(ex.sms) * 8)));
  k_densify<<<grid, 256, 0, ex.stream>>>(n, op.indptr, op.indices, op.v64, op.diag, A.get());
  SI_LAUNCH_CHECK();
  k_mirror_lower<<<static_cast<int>(std::min<int64_t>((n * n + 255) / 256, int64_t(ex.sms) * 16)), 256, 0,
                   ex.stream>>>(n, A.get());
  SI_LAUNCH_CHECK();
  if (n < kTriMultiMin) {
    // small matrices: one CTA (launch latency would dominate the step kernels)
    const size_t smem = sizeof(double) * 2 * n;
    static std::atomic<bool> attr_set[128];
    if (ex.device >= 0 && ex.device < 128 && !attr_set[ex.device]) {
      SI_CUDA(cudaFuncSetAttribute(k_tridiag, cudaFuncAttributeMaxDynamicSharedMemorySize, 2 * 8192 * 8));
      attr_set[ex.device] = true;
    }
    k_tridiag<<<1, DT, smem, ex.stream>>>(A.get(), static_cast<int>(n), d.get(), e.get(), tau.get());
    SI_LAUNCH_CHECK();
  } else {
    const int ni = static_cast<int>(n);
    DevBuf<double> vbuf(n, ex.stream), wbuf(n, ex.stream), partial((n + 7) / 8, ex.stream);
    DevBuf<unsigned> counter(1, ex.stream);
    counter.zero();
    for (int j = 0; j + 2 < ni; ++j) {
      const int len = ni - j - 1;
      k_tri_house<<<1, 256, 0, ex.stream>>>(A.get(), ni, j, d.get(), e.get(), tau.get(), vbuf.get());
      SI_LAUNCH_CHECK();
      k_tri_matvec<<<(len + 7) / 8, 256, 0, ex.stream>>>(A.get(), ni, j, tau.get(), vbuf.get(), wbuf.get(),
                                                         partial.get(), counter.get());
      SI_LAUNCH_CHECK();
      k_tri_update<<<std::min(len, ex.sms * 8), 256, 0, ex.stream>>>(A.get(), ni, j, tau.get(), vbuf.get(),
                                                                    wbuf.get());
      SI_LAUNCH_CHECK();
    }
    k_tri_last<<<1, 32, 0, ex.stream>>>(A.get(), ni, d.get(), e.get(), tau.get());
    SI_LAUNCH_CHECK();
  }
  DevBuf<int> bstart(n + 1, ex.stream), cand_blk(static_cast<size_t>(n) * k, ex.stream), piv(n, ex.stream),
      sel_blk(MAXM, ex.stream);
  DevBuf<double> es(n, ex.stream), cand(static_cast<size_t>(n) * k, ex.stream), lu(5 * n, ex.stream),
      xv(n, ex.stream), sel_val(MAXM, ex.stream);
  TriWork w{bstart.get(), es.get(), cand.get(), cand_blk.get(), lu.get(), piv.get(), xv.get(), sel_blk.get(),
            sel_val.get()};
  SI_CUDA(cudaMemsetAsync(evecs, 0, sizeof(double) * n * ld, ex.stream));
  k_tri_eig<<<1, DT, 0, ex.stream>>>(d.get(), e.get(), static_cast<int>(n), k, w, ev.get(), evecs, ld);
  SI_LAUNCH_CHECK();
  k_backtransform<<<1, DT, 0, ex.stream>>>(A.get(), tau.get(), static_cast<int>(n), evecs, ld, k);
  SI_LAUNCH_CHECK();
  SI_CUDA(cudaMemcpyAsync(evals_host, ev.get(), sizeof(double) * k, cudaMemcpyDeviceToHost, ex.stream));
  SI_CUDA(cudaStreamSynchronize(ex.stream));
}

}  // namespace si
