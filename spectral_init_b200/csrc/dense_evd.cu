// Dense symmetric eigensolver on the device for the k smallest eigenpairs
// (dense_evd, src/solvers/dense.rs:9-46; Levels 0 and 5 of the chain).
//
//   1. densify the operator (lower triangle mirrored, like faer's Side::Lower);
//   2. Householder tridiagonalisation T = Q^T A Q (dsytd2-style): one CTA
//      below 192 rows, one cooperative launch with the matrix spread over the
//      shared memory of co-resident CTAs up to 2048 rows, and three launches
//      per column above that;
//   3. split T where off-diagonals are negligible, then for every block the
//      smallest eigenvalues by Sturm-count multisection (bisection when there
//      are many blocks) to LAPACK dstebz's default tolerance eps |T|; the k
//      smallest overall are kept;
//   4. eigenvectors of T by inverse iteration restricted to the block (LU with
//      partial pivoting of T - lambda I), re-orthogonalised within clusters of
//      close eigenvalues (modified Gram-Schmidt), stopped as LAPACK's dstein
//      once the growth shows a rounding-level residual;
//   5. back-transformation v = Q y with the stored reflectors (compact-WY
//      blocks of eight when Y and a block fit in shared memory).
#include <algorithm>
#include <cfloat>
#include <cmath>
#include <cstdlib>
#include <mutex>
#include <string>
#include <utility>
#include <vector>

#include "si_internal.h"

namespace si {
namespace {

constexpr int DT = 1024;
constexpr int TE_MS_ITEMS = 32;   // multisection when at most this many (block, index) items
constexpr int TE_MS_POINTS = 96;  // at most this many Sturm points per item and round
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

// ---- single-launch tridiagonalisation (kTriMultiMin <= n <= kTriCoopMax) ----
// The same Householder steps with the matrix held in the shared memory of G
// co-resident CTAs (cooperative launch): row r lives in CTA r % G, slot r / G,
// so a step touches on-chip data plus two n-vectors in L2.  Step j:
//   (1) warp 0 of the CTA holding row j forms the reflector from that row
//       (A is kept exactly symmetric, so row j equals column j), writes v, d,
//       e, tau and the reflector (row j of A in global memory) and publishes
//       the step with a release store (no CTA-wide barrier on this path);
//   (2) every CTA computes w_r = tau (A v)_r for its rows r > j; warp 0 adds
//       its share of w.v and arrives at the grid barrier (a release add on a
//       counter on its own 128-byte line, pollers back off 32 ns);
//   (3) every warp of every CTA adds the shares in CTA order (the same sum
//       everywhere), K = tau (w.v) / 2, w' = w - K v, and the CTA updates its
//       rows A -= v w'^T + w' v^T, each entry as round(v_r w'_c) +
//       round(w'_r v_c) so entries (r, c) and (c, r) stay identical.
// Four CTA barriers a step; own-row v and the columns of w are loaded ahead of
// the reductions that need them.
// v, w and the shares are double-buffered by step parity: a buffer is written
// again two steps later, after a barrier that all of its readers have passed.
// Every wait is bounded: a CTA that waits longer than the limit sets the error
// word, every CTA returns, and the host redoes the matrix with the
// multi-launch steps.
constexpr int CT_THREADS = 512;
constexpr int CT_RMAX = 16;                                    // rows per CTA
constexpr int CT_CMAX = 4;                                     // columns per thread
constexpr int64_t kTriCoopMax = int64_t(CT_THREADS) * CT_CMAX;  // 2048
constexpr uint64_t kCoopWaitNs = 2000000000ull;                // 2 s per wait
constexpr int kFlagStride = 32;                                // unsigned words per 128-byte line

struct CoopTri {
  double* A;  // n x n, exactly symmetric on entry; reflector of step j goes to row j
  int n, G, R;
  double *d, *e, *tau;
  double* vbuf;      // [2][n]
  double* wbuf;      // [2][n]
  double* share;     // [2][G]
  unsigned* vready;  // last step whose reflector is published
  unsigned* arrive;  // grid barrier arrivals (G per step)
  int* err;
  uint64_t wait_ns;  // limit of every wait
};

__device__ __forceinline__ uint64_t coop_ns() {
  uint64_t t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}
__device__ __forceinline__ unsigned ld_acquire_u32(const unsigned* p) {
  unsigned v;
  asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}
__device__ __forceinline__ void st_release_u32(unsigned* p, unsigned v) {
  asm volatile("st.release.gpu.global.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}
__device__ __forceinline__ void red_release_add_u32(unsigned* p, unsigned v) {
  asm volatile("red.release.gpu.global.add.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}
// One thread: wait until *p >= target, polling with a short back-off.  False
// when the wait ran past the limit (the error word is set) or another CTA gave
// up first.
__device__ bool coop_wait(const unsigned* p, unsigned target, int* err, uint64_t limit_ns) {
  if (ld_acquire_u32(p) >= target) return true;
  const uint64_t t0 = coop_ns();
  while (ld_acquire_u32(p) < target) {
    __nanosleep(32);
    if (*reinterpret_cast<volatile int*>(err) != 0) return false;
    if (coop_ns() - t0 > limit_ns) {
      atomicExch(err, 1);
      return false;
    }
  }
  return true;
}

__global__ void __launch_bounds__(CT_THREADS, 1) k_tridiag_coop(CoopTri p) {
  extern __shared__ double rows[];  // [R][n]
  __shared__ double red[CT_THREADS / 32][CT_RMAX];
  __shared__ double s_v[CT_RMAX], s_w[CT_RMAX];
  __shared__ int s_ok;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int n = p.n, G = p.G, R = p.R, b = blockIdx.x;
  for (int l = 0; l < R; ++l) {
    const int r = l * G + b;
    if (r >= n) break;
    for (int c = tid; c < n; c += CT_THREADS) rows[l * n + c] = p.A[static_cast<int64_t>(r) * n + c];
  }
  __syncthreads();
  for (int j = 0; j + 2 < n; ++j) {
    const int par = j & 1;
    double* vb = p.vbuf + par * n;
    double* wb = p.wbuf + par * n;
    double* sh = p.share + par * G;
    // (1) reflector of row j, formed by warp 0 of the CTA holding the row
    if (j % G == b && warp == 0) {
      const double* rj = rows + (j / G) * n;
      double part = 0.0;
      for (int i = j + 2 + lane; i < n; i += 32) part = fma(rj[i], rj[i], part);
      const double sigma = warp_sum(part);
      const double alpha = rj[j + 1];
      double t = 0.0, beta = alpha, scal = 0.0;
      if (sigma > 0.0) {
        const double nrm = sqrt(alpha * alpha + sigma);
        beta = alpha >= 0.0 ? -nrm : nrm;
        t = (beta - alpha) / beta;
        scal = 1.0 / (alpha - beta);
      }
      if (lane == 0) {
        p.d[j] = rj[j];
        p.e[j] = beta;
        p.tau[j] = t;
      }
      for (int i = j + 1 + lane; i < n; i += 32) {
        const double vi = (i == j + 1) ? 1.0 : rj[i] * scal;
        vb[i] = vi;
        if (i >= j + 2) p.A[static_cast<int64_t>(j) * n + i] = vi;
      }
      __syncwarp();
      if (lane == 0) {
        __threadfence();
        st_release_u32(p.vready, static_cast<unsigned>(j + 1));
      }
    }
    if (tid == 0) s_ok = coop_wait(p.vready, static_cast<unsigned>(j + 1), p.err, p.wait_ns) ? 1 : 0;
    __syncthreads();
    if (!s_ok) return;
    const double tau = __ldcg(p.tau + j);
    // slots below l0 hold finished rows (r <= j)
    const int l0 = j >= b ? (j - b) / G + 1 : 0;
    const int my_r = tid * G + b;
    const bool my_live = tid < R && my_r > j && my_r < n;
    const double my_v = my_live ? __ldcg(vb + my_r) : 0.0;
    // (2) w = tau A v on this CTA's rows r > j
    double vc[CT_CMAX], acc[CT_RMAX];
#pragma unroll
    for (int l = 0; l < CT_RMAX; ++l) acc[l] = 0.0;
#pragma unroll
    for (int q = 0; q < CT_CMAX; ++q) {
      const int c = j + 1 + tid + q * CT_THREADS;
      vc[q] = c < n ? __ldcg(vb + c) : 0.0;
      if (c < n) {
#pragma unroll
        for (int l = 0; l < CT_RMAX; ++l)
          if (l >= l0 && l < R) acc[l] = fma(rows[l * n + c], vc[q], acc[l]);
      }
    }
#pragma unroll
    for (int l = 0; l < CT_RMAX; ++l) {
      if (l >= l0 && l < R) {
        const double sum = warp_sum(acc[l]);
        if (lane == 0) red[warp][l] = sum;
      }
    }
    __syncthreads();
    // own rows (threads 0 .. R - 1, all in warp 0): w_r, and this CTA's share of w.v
    if (warp == 0) {
      double wr = 0.0;
      if (my_live) {
        double sum = 0.0;
        for (int w = 0; w < CT_THREADS / 32; ++w) sum += red[w][tid];
        wr = tau * sum;
        wb[my_r] = wr;
      }
      if (tid < R) {
        s_w[tid] = wr;
        s_v[tid] = my_v;
      }
      const double share = warp_sum(wr * my_v);
      __syncwarp();  // the lanes' w stores are ordered before lane 0's fence
      if (lane == 0) {
        sh[b] = share;
        __threadfence();
        red_release_add_u32(p.arrive, 1u);
        s_ok = coop_wait(p.arrive, static_cast<unsigned>(j + 1) * static_cast<unsigned>(G), p.err, p.wait_ns) ? 1 : 0;
      }
    }
    __syncthreads();
    if (!s_ok) return;
    // (3) w of this thread's columns and, in every warp, K = tau (w.v) / 2
    // from the CTAs' shares in CTA order (the same sum in every warp)
    double wcol[CT_CMAX];
#pragma unroll
    for (int q = 0; q < CT_CMAX; ++q) {
      const int c = j + 1 + tid + q * CT_THREADS;
      wcol[q] = c < n ? __ldcg(wb + c) : 0.0;
    }
    double ksum = 0.0;
    for (int c = lane; c < G; c += 32) ksum += __ldcg(sh + c);
    const double K = 0.5 * tau * warp_sum(ksum);
#pragma unroll
    for (int q = 0; q < CT_CMAX; ++q) {
      const int c = j + 1 + tid + q * CT_THREADS;
      if (c < n) {
        const double wc = fma(-K, vc[q], wcol[q]);
#pragma unroll
        for (int l = 0; l < CT_RMAX; ++l) {
          if (l >= l0 && l < R && l * G + b < n) {
            const double wr = fma(-K, s_v[l], s_w[l]);
            const double u = __dadd_rn(__dmul_rn(s_v[l], wc), __dmul_rn(wr, vc[q]));
            rows[l * n + c] -= u;
          }
        }
      }
    }
    __syncthreads();
  }
  if (tid == 0 && n >= 2) {
    const int r2 = n - 2, r1 = n - 1;
    if (r2 % G == b) {
      const double* row = rows + (r2 / G) * n;
      p.d[r2] = row[r2];
      p.e[r2] = row[r1];
      p.tau[r2] = 0.0;
    }
    if (r1 % G == b) p.d[r1] = rows[(r1 / G) * n + r1];
  }
}

// number of eigenvalues of T[l..r] smaller than x (Sturm sequence; e2 holds
// the squared off-diagonals)
__device__ int sturm_count(const double* d, const double* e2, int l, int r, double x, double pivmin) {
  int cnt = 0;
  double q = d[l] - x;
  if (fabs(q) < pivmin) q = -pivmin;
  if (q < 0.0) ++cnt;
  for (int i = l + 1; i <= r; ++i) {
    q = d[i] - x - e2[i - 1] / q;
    if (fabs(q) < pivmin) q = -pivmin;
    if (q < 0.0) ++cnt;
  }
  return cnt;
}

struct TriWork {
  int* bstart;      // [n + 1]
  double* es;       // [n] split off-diagonals
  double* e2;       // [n] their squares
  double* cand;     // [n * k]
  int* cand_blk;    // [n * k]
  double* lu;       // [5 * n]
  int* piv;         // [n]
  double* xv;       // [n]
  int* sel_blk;     // [k]
  double* sel_val;  // [k]
};

__global__ void __launch_bounds__(DT) k_tri_eig(const double* __restrict__ d, const double* __restrict__ e, int n,
                                                int k, TriWork w, double* evals_out, double* Y, int ld,
                                                int use_smem) {
  __shared__ int s_nb;
  __shared__ double s_tnorm;
  __shared__ double s_red[32];
  extern __shared__ double te_sm[];
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  // diagonal, split off-diagonals and their squares: in shared memory behind
  // the inverse-iteration arrays when it fits
  const double* dd = d;
  double* es = w.es;
  double* e2 = w.e2;
  if (use_smem) {
    double* dsm = te_sm + 6 * n;
    for (int i = tid; i < n; i += blockDim.x) dsm[i] = d[i];
    dd = dsm;
    es = te_sm + 7 * n;
    e2 = te_sm + 8 * n;
  }
  // |T| (row sums) and the splits where an off-diagonal is negligible
  double part = 0.0;
  for (int i = tid; i < n; i += blockDim.x) {
    part = fmax(part, fabs(d[i]) + (i > 0 ? fabs(e[i - 1]) : 0.0) + (i + 1 < n ? fabs(e[i]) : 0.0));
    if (i + 1 < n) {
      const double off = fabs(e[i]);
      const bool split = off <= DBL_EPSILON * (fabs(d[i]) + fabs(d[i + 1])) || off <= 1e-300;
      es[i] = split ? 0.0 : e[i];
      e2[i] = split ? 0.0 : e[i] * e[i];
    }
  }
  part = warp_max(part);
  if (lane == 0) s_red[warp] = part;
  __syncthreads();
  // block starts in order (one warp: ballot and prefix count per 32 entries)
  if (warp == 0) {
    double tn = 0.0;
    for (int i = lane; i < static_cast<int>(blockDim.x >> 5); i += 32) tn = fmax(tn, s_red[i]);
    tn = warp_max(tn);
    int cnt = 0;
    for (int base = 0; base + 1 < n; base += 32) {
      const int i = base + lane;
      const bool f = i + 1 < n && es[i] == 0.0;
      const unsigned bal = __ballot_sync(0xffffffffu, f);
      if (f) w.bstart[1 + cnt + __popc(bal & ((1u << lane) - 1u))] = i + 1;
      cnt += __popc(bal);
    }
    if (lane == 0) {
      w.bstart[0] = 0;
      w.bstart[cnt + 1] = n;
      s_nb = cnt + 1;
      s_tnorm = tn;
    }
  }
  __syncthreads();
  const int nb = s_nb;
  const double tnorm = s_tnorm;
  const double pivmin = fmax(DBL_MIN, tnorm * tnorm * DBL_MIN);
  // absolute tolerance of the eigenvalue intervals: eps |T| (the default of
  // LAPACK's dstebz); relative eps for eigenvalues away from zero
  const double atol = DBL_EPSILON * tnorm + pivmin;
  const int nitems = nb * k;
  // Gershgorin interval of item q's block; false if the block has no t-th eigenvalue
  auto item_interval = [&](int q, double& lo, double& hi) {
    const int b = q / k, t = q % k;
    const int l = w.bstart[b], r = w.bstart[b + 1] - 1;
    w.cand_blk[q] = b;
    if (t > r - l) {
      w.cand[q] = DBL_MAX;
      return false;
    }
    lo = DBL_MAX;
    hi = -DBL_MAX;
    for (int i = l; i <= r; ++i) {
      const double rad = (i > l ? fabs(es[i - 1]) : 0.0) + (i < r ? fabs(es[i]) : 0.0);
      lo = fmin(lo, dd[i] - rad);
      hi = fmax(hi, dd[i] + rad);
    }
    lo -= 2.0 * DBL_EPSILON * tnorm + pivmin;
    hi += 2.0 * DBL_EPSILON * tnorm + pivmin;
    return true;
  };
  auto converged = [&](double lo, double hi) {
    const double mid = 0.5 * (lo + hi);
    return hi - lo <= 2.0 * DBL_EPSILON * fmax(fabs(lo), fabs(hi)) + atol || mid == lo || mid == hi;
  };
  if (nitems <= TE_MS_ITEMS) {
    // multisection: the P threads of an item count eigenvalues below P interior
    // points of its interval per round, and the interval shrinks to the gap
    // between the two points around the wanted index (a factor P + 1 a round)
    __shared__ double s_lo[TE_MS_ITEMS], s_hi[TE_MS_ITEMS];
    __shared__ int s_live[TE_MS_ITEMS];
    __shared__ int s_cnt[DT];
    // points per item: each Sturm count is a chain of n FP64 divisions, so past
    // ~96 points per item the SM's FP64 pipe, not the chain, sets the round time
    const int P = min(static_cast<int>(blockDim.x) / nitems, TE_MS_POINTS);
    if (tid < nitems) {
      double lo = 0.0, hi = 0.0;
      const bool ok = item_interval(tid, lo, hi);
      s_lo[tid] = lo;
      s_hi[tid] = hi;
      s_live[tid] = ok && !converged(lo, hi);
      if (ok && !s_live[tid]) w.cand[tid] = 0.5 * (lo + hi);
    }
    __syncthreads();
    const int item = tid / P, pi = tid % P;
    auto point = [&](double lo, double hi, int p) { return lo + (hi - lo) * (static_cast<double>(p + 1) / (P + 1)); };
    for (int round = 0; round < 200; ++round) {
      if (item < nitems && s_live[item]) {
        const int b = item / k;
        s_cnt[tid] = sturm_count(dd, e2, w.bstart[b], w.bstart[b + 1] - 1, point(s_lo[item], s_hi[item], pi), pivmin);
      }
      __syncthreads();
      int more = 0;
      if (tid < nitems && s_live[tid]) {
        const int t = tid % k;
        const double lo = s_lo[tid], hi = s_hi[tid];
        int p = 0;
        while (p < P && s_cnt[tid * P + p] <= t) ++p;
        // count(point p - 1) <= t < count(point p)
        const double nlo = p == 0 ? lo : point(lo, hi, p - 1);
        const double nhi = p == P ? hi : point(lo, hi, p);
        s_lo[tid] = nlo;
        s_hi[tid] = nhi;
        if (converged(nlo, nhi) || (nlo == lo && nhi == hi)) {
          s_live[tid] = 0;
          w.cand[tid] = 0.5 * (nlo + nhi);
        } else {
          more = 1;
        }
      }
      if (!__syncthreads_or(more)) break;
    }
    if (tid < nitems && s_live[tid]) w.cand[tid] = 0.5 * (s_lo[tid] + s_hi[tid]);
  } else {
    // one thread per item, bisection
    for (int q = tid; q < nitems; q += blockDim.x) {
      double lo = 0.0, hi = 0.0;
      if (!item_interval(q, lo, hi)) continue;
      const int b = q / k, t = q % k;
      const int l = w.bstart[b], r = w.bstart[b + 1] - 1;
      for (int it = 0; it < 200 && !converged(lo, hi); ++it) {
        const double mid = 0.5 * (lo + hi);
        if (sturm_count(dd, e2, l, r, mid, pivmin) > t) hi = mid; else lo = mid;
      }
      w.cand[q] = 0.5 * (lo + hi);
    }
  }
  __syncthreads();
  // k smallest candidates (stable)
  __shared__ int s_nsel;
  if (tid == 0) {
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
    s_nsel = nsel;
  }
  __syncthreads();
  const int nsel = s_nsel;
  // Eigenvectors by inverse iteration.  The LU factorisation and the two
  // triangular sweeps are sequential (thread 0, working arrays in shared
  // memory when they fit, reciprocals of the pivots formed in parallel);
  // re-orthogonalisation and normalisation use the whole CTA.  Iteration stops
  // after the second solve once the growth ||y|| shows a residual at rounding
  // level (as LAPACK's dstein), at the latest after the fourth.
  double* D = use_smem ? te_sm : w.lu;
  double* DL = D + n;
  double* DU = D + 2 * n;
  double* DU2 = D + 3 * n;
  double* RD = D + 4 * n;  // 1 / D
  double* x = use_smem ? te_sm + 5 * n : w.xv;
  int* piv = use_smem ? reinterpret_cast<int*>(te_sm + 9 * n) : w.piv;
  double* red = s_red;
  const double tiny = DBL_EPSILON * fmax(tnorm, DBL_MIN);
  for (int s = 0; s < nsel; ++s) {
    const int q = w.sel_blk[s];
    const int b = w.cand_blk[q];
    const int l = w.bstart[b], r = w.bstart[b + 1] - 1, sz = r - l + 1;
    const double lam = w.cand[q];
    double bpart = 0.0;
    for (int i = l + tid; i <= r; i += blockDim.x)
      bpart = fmax(bpart, fabs(dd[i]) + (i > l ? fabs(es[i - 1]) : 0.0) + (i < r ? fabs(es[i]) : 0.0));
    bpart = warp_max(bpart);
    if ((tid & 31) == 0) red[tid >> 5] = bpart;
    __syncthreads();
    double bnorm = 0.0;
    for (int i = 0; i < static_cast<int>(blockDim.x >> 5); ++i) bnorm = fmax(bnorm, red[i]);
    // T_b - lam I, and the start vector
    for (int i = tid; i < sz; i += blockDim.x) {
      D[i] = dd[l + i] - lam;
      DU[i] = (i + 1 < sz) ? es[l + i] : 0.0;
      DL[i] = DU[i];
      DU2[i] = 0.0;
      double z0, z1;
      philox_normal2(0x0de75eedull + s, 7, static_cast<uint64_t>(i), z0, z1);
      x[i] = z0;
    }
    __syncthreads();
    // LU with partial pivoting
    if (tid == 0) {
      for (int i = 0; i + 1 < sz; ++i) {
        if (fabs(D[i]) >= fabs(DL[i])) {
          if (D[i] == 0.0) D[i] = tiny;
          const double f = DL[i] / D[i];
          DL[i] = f;
          D[i + 1] -= f * DU[i];
          piv[i] = 0;
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
          piv[i] = 1;
        }
      }
    }
    __syncthreads();
    for (int i = tid; i < sz; i += blockDim.x) {
      if (fabs(D[i]) < tiny) D[i] = D[i] < 0.0 ? -tiny : tiny;
      RD[i] = 1.0 / D[i];
    }
    __syncthreads();
    const double grow_ok = 1.0 / (static_cast<double>(sz) * DBL_EPSILON * fmax(bnorm, DBL_MIN));
    for (int it = 0; it < 4; ++it) {
      // solve (T - lam I) y = x in place
      if (tid == 0) {
        for (int i = 0; i + 1 < sz; ++i) {
          if (piv[i] == 0) {
            x[i + 1] -= DL[i] * x[i];
          } else {
            const double tmp = x[i];
            x[i] = x[i + 1];
            x[i + 1] = tmp - DL[i] * x[i];
          }
        }
        x[sz - 1] *= RD[sz - 1];
        if (sz >= 2) x[sz - 2] = (x[sz - 2] - DU[sz - 2] * x[sz - 1]) * RD[sz - 2];
        for (int i = sz - 3; i >= 0; --i) x[i] = (x[i] - DU[i] * x[i + 1] - DU2[i] * x[i + 2]) * RD[i];
      }
      __syncthreads();
      // re-orthogonalise against earlier vectors of the same block in the cluster
      for (int u = 0; u < s; ++u) {
        const int qu = w.sel_blk[u];
        if (w.cand_blk[qu] != b) continue;
        if (fabs(w.sel_val[u] - lam) > 1e-3 * bnorm) continue;
        double part = 0.0;
        for (int i = tid; i < sz; i += blockDim.x) part += Y[static_cast<int64_t>(l + i) * ld + u] * x[i];
        const double dot = block_sum_all(part, red);
        for (int i = tid; i < sz; i += blockDim.x) x[i] -= dot * Y[static_cast<int64_t>(l + i) * ld + u];
        __syncthreads();
      }
      double part = 0.0;
      for (int i = tid; i < sz; i += blockDim.x) part += x[i] * x[i];
      double nrm = sqrt(block_sum_all(part, red));
      const bool degenerate = !(nrm > 0.0);
      const double inv = degenerate ? 1.0 : 1.0 / nrm;
      for (int i = tid; i < sz; i += blockDim.x) x[i] = degenerate ? ((i == s % sz) ? 1.0 : 0.0) : x[i] * inv;
      __syncthreads();
      if (it >= 1 && nrm >= grow_ok) break;  // uniform: nrm is the same in every thread
    }
    for (int i = tid; i < sz; i += blockDim.x) Y[static_cast<int64_t>(l + i) * ld + s] = x[i];
    __syncthreads();
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

// The same product with Y (n x k) in shared memory: each of the 256 threads
// owns rows tid, tid + 256, ... (at most BT_RPT), so the only exchange per
// reflector is the k dot products (warp sums, then the eight warp partials in
// warp order; double-buffered, one barrier per reflector).  The reflector of
// the next step is loaded while the current one is applied.
constexpr int BT_THREADS = 256;
constexpr int BT_RPT = 8;  // rows per thread: n <= 2048

__global__ void __launch_bounds__(BT_THREADS) k_backtransform_smem(const double* __restrict__ A,
                                                                   const double* __restrict__ tau, int n,
                                                                   double* __restrict__ Y, int ld, int k) {
  extern __shared__ double ys[];  // [n][k]
  __shared__ double red[2][BT_THREADS / 32][MAXM];
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  for (int idx = tid; idx < n * k; idx += BT_THREADS) ys[idx] = Y[static_cast<int64_t>(idx / k) * ld + idx % k];
  // u of reflector j on this thread's rows (zero outside rows j + 1 .. n - 1)
  auto load_u = [&](int j, double* u) {
#pragma unroll
    for (int q = 0; q < BT_RPT; ++q) {
      const int r = tid + q * BT_THREADS;
      u[q] = r == j + 1 ? 1.0 : ((r > j + 1 && r < n) ? A[static_cast<int64_t>(j) * n + r] : 0.0);
    }
  };
  double u[BT_RPT], un[BT_RPT];
  load_u(n - 3, u);
  __syncthreads();
  int buf = 0;
  for (int j = n - 3; j >= 0; --j) {
    const double t = tau[j];
    if (j > 0) load_u(j - 1, un);
    if (t != 0.0) {
      double part[MAXM];
#pragma unroll
      for (int v = 0; v < MAXM; ++v) part[v] = 0.0;
#pragma unroll
      for (int q = 0; q < BT_RPT; ++q) {
        const int r = tid + q * BT_THREADS;
        if (r > j && r < n) {
#pragma unroll
          for (int v = 0; v < MAXM; ++v)
            if (v < k) part[v] = fma(u[q], ys[r * k + v], part[v]);
        }
      }
#pragma unroll
      for (int v = 0; v < MAXM; ++v) {
        if (v < k) {
          const double s = warp_sum(part[v]);
          if (lane == 0) red[buf][warp][v] = s;
        }
      }
      __syncthreads();
#pragma unroll
      for (int v = 0; v < MAXM; ++v) {
        if (v < k) {
          double dsum = 0.0;
#pragma unroll
          for (int w = 0; w < BT_THREADS / 32; ++w) dsum += red[buf][w][v];
          const double dv = t * dsum;
#pragma unroll
          for (int q = 0; q < BT_RPT; ++q) {
            const int r = tid + q * BT_THREADS;
            if (r > j && r < n) ys[r * k + v] -= dv * u[q];
          }
        }
      }
      buf ^= 1;
    }
#pragma unroll
    for (int q = 0; q < BT_RPT; ++q) u[q] = un[q];
  }
  __syncthreads();
  for (int idx = tid; idx < n * k; idx += BT_THREADS) Y[static_cast<int64_t>(idx / k) * ld + idx % k] = ys[idx];
}

// The same product, blocked: reflectors are applied eight at a time from the
// last block down, each block as one compact-WY product (the forward,
// column-wise form of LAPACK's dlarft):
//   H_j0 H_j0+1 ... H_j0+7 = I - V T V^T,   T upper triangular,
//   T[i][i] = tau_i,  T[0:i, i] = -tau_i T[0:i, 0:i] (V^T V)[0:i, i],
// so a block costs one pass of dot products (V^T V and V^T Y, one warp per
// product, lanes over rows), a small triangular product and one pass
// Y -= V (T V^T Y).  Y (n x k) and the block's reflectors stay in shared
// memory; a reflector with tau = 0 gets a zero row and column of T.
constexpr int BW_NB = 8;
constexpr int BW_THREADS = 512;

__global__ void __launch_bounds__(BW_THREADS) k_backtransform_wy(const double* __restrict__ A,
                                                                 const double* __restrict__ tau, int n,
                                                                 double* __restrict__ Y, int ld, int k) {
  extern __shared__ double bw_sm[];
  double* ys = bw_sm;          // [n][k]
  double* U = bw_sm + n * k;   // [BW_NB][n]
  __shared__ double G[BW_NB][BW_NB], T[BW_NB][BW_NB], Wt[BW_NB][MAXM], Wp[BW_NB][MAXM], st[BW_NB];
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  constexpr int NW = BW_THREADS / 32;
  for (int idx = tid; idx < n * k; idx += BW_THREADS) ys[idx] = Y[static_cast<int64_t>(idx / k) * ld + idx % k];
  const int nref = n - 2;  // reflectors 0 .. n - 3
  for (int bi = (nref + BW_NB - 1) / BW_NB - 1; bi >= 0; --bi) {
    const int j0 = bi * BW_NB, nb = min(BW_NB, nref - j0);
    const int r0 = j0 + 1, len = n - r0;  // rows where the block's reflectors can be nonzero
    for (int idx = tid; idx < nb * len; idx += BW_THREADS) {
      const int i = idx / len, r = r0 + idx % len;
      const int j = j0 + i;
      U[i * n + r] = r == j + 1 ? 1.0 : (r > j + 1 ? A[static_cast<int64_t>(j) * n + r] : 0.0);
    }
    if (tid < nb) st[tid] = tau[j0 + tid];
    __syncthreads();
    const int ng = nb * (nb + 1) / 2, nd = ng + nb * k;
    for (int dd = warp; dd < nd; dd += NW) {
      double acc = 0.0;
      int a = 0, b = 0, v = 0;
      if (dd < ng) {
        int e = dd;
        while (e >= nb - a) {
          e -= nb - a;
          ++a;
        }
        b = a + e;
        for (int r = r0 + lane; r < n; r += 32) acc = fma(U[a * n + r], U[b * n + r], acc);
      } else {
        a = (dd - ng) / k;
        v = (dd - ng) % k;
        for (int r = r0 + lane; r < n; r += 32) acc = fma(U[a * n + r], ys[r * k + v], acc);
      }
      acc = warp_sum(acc);
      if (lane == 0) {
        if (dd < ng) G[a][b] = acc;
        else Wt[a][v] = acc;
      }
    }
    __syncthreads();
    if (tid == 0) {
      for (int i = 0; i < nb; ++i) {
        T[i][i] = st[i];
        for (int p = 0; p < i; ++p) {
          double sum = 0.0;
          for (int q = p; q < i; ++q) sum = fma(T[p][q], G[q][i], sum);
          T[p][i] = -st[i] * sum;
        }
      }
      for (int a = 0; a < nb; ++a)
        for (int v = 0; v < k; ++v) {
          double sum = 0.0;
          for (int b = a; b < nb; ++b) sum = fma(T[a][b], Wt[b][v], sum);
          Wp[a][v] = sum;
        }
    }
    __syncthreads();
    for (int idx = tid; idx < len * k; idx += BW_THREADS) {
      const int r = r0 + idx / k, v = idx % k;
      double sum = 0.0;
      for (int a = 0; a < nb; ++a) sum = fma(U[a * n + r], Wp[a][v], sum);
      ys[r * k + v] -= sum;
    }
    __syncthreads();
  }
  for (int idx = tid; idx < n * k; idx += BW_THREADS) Y[static_cast<int64_t>(idx / k) * ld + idx % k] = ys[idx];
}

}  // namespace

namespace {

void densify(const Exec& ex, const OpDev& op, double* A) {
  const int64_t n = op.n;
  SI_CUDA(cudaMemsetAsync(A, 0, sizeof(double) * n * n, ex.stream));
  const int grid = static_cast<int>(std::max<int64_t>(1, std::min<int64_t>((n + 255) / 256, int64_t(ex.sms) * 8)));
  k_densify<<<grid, 256, 0, ex.stream>>>(n, op.indptr, op.indices, op.v64, op.diag, A);
  SI_LAUNCH_CHECK();
  k_mirror_lower<<<static_cast<int>(std::min<int64_t>((n * n + 255) / 256, int64_t(ex.sms) * 16)), 256, 0,
                   ex.stream>>>(n, A);
  SI_LAUNCH_CHECK();
}

// The multi-launch steps (three launches per column).
void tridiag_steps(const Exec& ex, double* A, int n, double* d, double* e, double* tau) {
  DevBuf<double> vbuf(n, ex.stream), wbuf(n, ex.stream), partial((n + 7) / 8, ex.stream);
  DevBuf<unsigned> counter(1, ex.stream);
  counter.zero();
  for (int j = 0; j + 2 < n; ++j) {
    const int len = n - j - 1;
    k_tri_house<<<1, 256, 0, ex.stream>>>(A, n, j, d, e, tau, vbuf.get());
    SI_LAUNCH_CHECK();
    k_tri_matvec<<<(len + 7) / 8, 256, 0, ex.stream>>>(A, n, j, tau, vbuf.get(), wbuf.get(), partial.get(),
                                                       counter.get());
    SI_LAUNCH_CHECK();
    k_tri_update<<<std::min(len, ex.sms * 8), 256, 0, ex.stream>>>(A, n, j, tau, vbuf.get(), wbuf.get());
    SI_LAUNCH_CHECK();
  }
  k_tri_last<<<1, 32, 0, ex.stream>>>(A, n, d, e, tau);
  SI_LAUNCH_CHECK();
}

// Per-device limits of the single-launch tridiagonalisation.
struct CoopLimits {
  int supported = 0;  // cooperative launch available
  int smem_max = 0;   // dynamic shared memory per CTA (opt-in limit less the static part)
};

const CoopLimits& coop_limits(int device) {
  static CoopLimits lim[128];
  static std::once_flag once[128];
  SI_REQUIRE(device >= 0 && device < 128, SI_INVALID_ARGUMENT, "dense_evd: device ordinal");
  std::call_once(once[device], [device] {
    int coop = 0, smem = 0;
    SI_CUDA(cudaDeviceGetAttribute(&coop, cudaDevAttrCooperativeLaunch, device));
    SI_CUDA(cudaDeviceGetAttribute(&smem, cudaDevAttrMaxSharedMemoryPerBlockOptin, device));
    cudaFuncAttributes fa{};
    SI_CUDA(cudaFuncGetAttributes(&fa, k_tridiag_coop));
    const int dyn = smem - static_cast<int>(fa.sharedSizeBytes);
    SI_CUDA(cudaFuncSetAttribute(k_tridiag_coop, cudaFuncAttributeMaxDynamicSharedMemorySize, dyn));
    lim[device].smem_max = dyn;
    lim[device].supported = coop;
  });
  return lim[device];
}

// Dynamic shared memory a kernel of this file may use on a device (the
// opt-in limit less its static shared memory), with the attribute raised to
// it on first use.
template <class F>
int smem_limit(int device, F* kernel) {
  static std::mutex mu;
  static std::vector<std::pair<std::pair<int, const void*>, int>> known;
  SI_REQUIRE(device >= 0 && device < 128, SI_INVALID_ARGUMENT, "dense_evd: device ordinal");
  const void* key = reinterpret_cast<const void*>(kernel);
  std::lock_guard<std::mutex> lk(mu);
  for (const auto& kv : known)
    if (kv.first.first == device && kv.first.second == key) return kv.second;
  int smem = 0;
  SI_CUDA(cudaDeviceGetAttribute(&smem, cudaDevAttrMaxSharedMemoryPerBlockOptin, device));
  cudaFuncAttributes fa{};
  SI_CUDA(cudaFuncGetAttributes(&fa, kernel));
  const int dyn = smem - static_cast<int>(fa.sharedSizeBytes);
  SI_CUDA(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, dyn));
  known.push_back({{device, key}, dyn});
  return dyn;
}

// Limit of every wait of the single-launch tridiagonalisation: 2 s, or less
// through SPECTRAL_INIT_COOP_WAIT_NS (a test seam: a limit of 0 makes the
// first wait that is not already satisfied give up, which exercises the
// recovery path -- every CTA leaves at its next wait and the multi-launch
// steps redo the matrix).
uint64_t coop_wait_limit_ns() {
  const char* v = std::getenv("SPECTRAL_INIT_COOP_WAIT_NS");
  if (v == nullptr) return kCoopWaitNs;
  char* end = nullptr;
  const unsigned long long x = std::strtoull(v, &end, 10);
  return (end != v) ? static_cast<uint64_t>(std::min<unsigned long long>(x, kCoopWaitNs)) : kCoopWaitNs;
}

// SPECTRAL_INIT_TRIDIAG=steps selects the multi-launch steps for every n
// (read on every call, so one process can exercise both paths).
bool coop_disabled() {
  const char* v = std::getenv("SPECTRAL_INIT_TRIDIAG");
  return v != nullptr && std::string(v) == "steps";
}

// Launch the single-launch tridiagonalisation if the matrix fits in the shared
// memory of co-resident CTAs; false (nothing launched) otherwise.  About
// 96 KB of rows per CTA: fewer CTAs make the barriers cheaper and leave SMs
// to concurrent solves, the largest matrices use every SM.
bool tridiag_coop(const Exec& ex, double* A, int n, double* d, double* e, double* tau, DevBuf<double>& work,
                  DevBuf<unsigned>& flags) {
  if (n < kTriMultiMin || n > kTriCoopMax || coop_disabled()) return false;
  const CoopLimits& lim = coop_limits(ex.device);
  if (!lim.supported) return false;
  const double bytes = 8.0 * n * n;
  int G = static_cast<int>(std::ceil(bytes / (96.0 * 1024.0)));
  G = std::max(G, ceil_div(n, CT_RMAX));
  G = std::min({G, n, ex.sms});
  const int R = ceil_div(n, G);
  G = ceil_div(n, R);
  const size_t smem = sizeof(double) * static_cast<size_t>(R) * n;
  if (R > CT_RMAX || smem > static_cast<size_t>(lim.smem_max)) return false;
  int occ = 0;
  SI_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k_tridiag_coop, CT_THREADS, smem));
  if (G > occ * ex.sms) return false;
  work.alloc(4 * static_cast<size_t>(n) + 2 * static_cast<size_t>(G), ex.stream);
  // the step flag, the barrier counter and the error word on separate 128-byte lines
  flags.alloc(3 * kFlagStride, ex.stream);
  flags.zero();
  CoopTri p{};
  p.A = A;
  p.n = n;
  p.G = G;
  p.R = R;
  p.d = d;
  p.e = e;
  p.tau = tau;
  p.vbuf = work.get();
  p.wbuf = work.get() + 2 * n;
  p.share = work.get() + 4 * n;
  p.vready = flags.get();
  p.arrive = flags.get() + kFlagStride;
  p.err = reinterpret_cast<int*>(flags.get() + 2 * kFlagStride);
  p.wait_ns = coop_wait_limit_ns();
  void* args[] = {&p};
  SI_CUDA(cudaLaunchCooperativeKernel(reinterpret_cast<const void*>(k_tridiag_coop), dim3(G), dim3(CT_THREADS), args,
                                      smem, ex.stream));
  SI_LAUNCH_CHECK();
  return true;
}

}  // namespace

void dense_evd_dev(const Exec& ex, const OpDev& op, int k, double* evals_host, double* evecs, int ld) {
  const int64_t n = op.n;
  SI_REQUIRE(n >= 1 && k >= 1 && k <= n && k <= MAXM, SI_INVALID_ARGUMENT, "dense_evd: bad sizes");
  SI_REQUIRE(op.v64 != nullptr || op.nnz == 0, SI_INVALID_ARGUMENT, "dense_evd: f64 values required");
  DevBuf<double> A(static_cast<size_t>(n) * n, ex.stream), d(n, ex.stream), e(n, ex.stream), tau(n, ex.stream),
      ev(MAXM, ex.stream);
  DevBuf<int> bstart(n + 1, ex.stream), cand_blk(static_cast<size_t>(n) * k, ex.stream), piv(n, ex.stream),
      sel_blk(MAXM, ex.stream);
  DevBuf<double> es(n, ex.stream), e2(n, ex.stream), cand(static_cast<size_t>(n) * k, ex.stream),
      lu(5 * n, ex.stream), xv(n, ex.stream), sel_val(MAXM, ex.stream);
  TriWork w{bstart.get(), es.get(), e2.get(), cand.get(), cand_blk.get(), lu.get(), piv.get(), xv.get(), sel_blk.get(),
            sel_val.get()};
  const int ni = static_cast<int>(n);
  auto finish = [&] {
    SI_CUDA(cudaMemsetAsync(evecs, 0, sizeof(double) * n * ld, ex.stream));
    const size_t te_smem = (sizeof(double) * 9 + sizeof(int)) * static_cast<size_t>(n);
    const bool te_in_smem = te_smem <= static_cast<size_t>(smem_limit(ex.device, k_tri_eig));
    k_tri_eig<<<1, DT, te_in_smem ? te_smem : 0, ex.stream>>>(d.get(), e.get(), ni, k, w, ev.get(), evecs, ld,
                                                              te_in_smem ? 1 : 0);
    SI_LAUNCH_CHECK();
    const size_t wy_smem = sizeof(double) * static_cast<size_t>(n) * (k + BW_NB);
    const size_t bt_smem = sizeof(double) * static_cast<size_t>(n) * k;
    if (n >= 3 && wy_smem <= static_cast<size_t>(smem_limit(ex.device, k_backtransform_wy))) {
      k_backtransform_wy<<<1, BW_THREADS, wy_smem, ex.stream>>>(A.get(), tau.get(), ni, evecs, ld, k);
    } else if (n >= 3 && n <= int64_t(BT_THREADS) * BT_RPT &&
               bt_smem <= static_cast<size_t>(smem_limit(ex.device, k_backtransform_smem))) {
      k_backtransform_smem<<<1, BT_THREADS, bt_smem, ex.stream>>>(A.get(), tau.get(), ni, evecs, ld, k);
    } else {
      k_backtransform<<<1, DT, 0, ex.stream>>>(A.get(), tau.get(), ni, evecs, ld, k);
    }
    SI_LAUNCH_CHECK();
    SI_CUDA(cudaMemcpyAsync(evals_host, ev.get(), sizeof(double) * k, cudaMemcpyDeviceToHost, ex.stream));
  };
  densify(ex, op, A.get());
  if (n < kTriMultiMin) {
    // small matrices: one CTA (launch latency would dominate the step kernels)
    const size_t smem = sizeof(double) * 2 * n;
    static std::atomic<bool> attr_set[128];
    if (ex.device >= 0 && ex.device < 128 && !attr_set[ex.device]) {
      SI_CUDA(cudaFuncSetAttribute(k_tridiag, cudaFuncAttributeMaxDynamicSharedMemorySize, 2 * 8192 * 8));
      attr_set[ex.device] = true;
    }
    k_tridiag<<<1, DT, smem, ex.stream>>>(A.get(), ni, d.get(), e.get(), tau.get());
    SI_LAUNCH_CHECK();
    finish();
    SI_CUDA(cudaStreamSynchronize(ex.stream));
    return;
  }
  DevBuf<double> cwork;
  DevBuf<unsigned> cflags;
  if (tridiag_coop(ex, A.get(), ni, d.get(), e.get(), tau.get(), cwork, cflags)) {
    finish();
    int err = 0;
    SI_CUDA(cudaMemcpyAsync(&err, cflags.get() + 2 * kFlagStride, sizeof(int), cudaMemcpyDeviceToHost, ex.stream));
    SI_CUDA(cudaStreamSynchronize(ex.stream));
    if (err == 0) return;
    // a wait of the single-launch kernel ran out: redo with the multi-launch steps
    densify(ex, op, A.get());
  }
  tridiag_steps(ex, A.get(), ni, d.get(), e.get(), tau.get());
  finish();
  SI_CUDA(cudaStreamSynchronize(ex.stream));
}

}  // namespace si
