// Small dense linear algebra in one CTA (matrices in shared memory):
// Cholesky, triangular solves and a parallel cyclic Jacobi eigensolver, and
// on top of them the per-iteration "small step" of block LOBPCG.
//
// LOBPCG small step (restatement of one iteration of the linfa-linalg 0.2
// LOBPCG loop that src/solvers/lobpcg.rs:327-358 calls; algorithm of Knyazev,
// SIAM J. Sci. Comput. 23(2), 2001):
//   1. residual norms of the current block from diag(R^T R) of the Gram,
//      best-iterate tracking (smallest sum of wanted residual norms), soft
//      locking (a wanted column stays locked once its norm <= tol), and the
//      convergence / iteration-cap decision;
//   2. Rayleigh-Ritz on span{X, R_active, P_active} as the generalised
//      problem (S^T A S) y = theta (S^T S) y, made well-scaled by the diagonal
//      of S^T S and reduced with a Cholesky factor; when the factor fails
//      with P present the step is retried on span{X, R_active} (the same
//      fallback as the reference iteration);
//   3. the coefficients Cx, Cr, Cp of the new X and P for the block update.
// The Gram matrices come from the fused device pass over the blocks, so the
// residuals never need an explicit orthogonalisation pass.
#include <cfloat>
#include <cstdlib>
#include <string>

#include "si_internal.h"

namespace si {
namespace {

constexpr int ST = 128;       // threads of the small-step CTA (blocks of up to 8 columns)
constexpr int ST_WIDE = 512;  // threads of the small-step CTA for wider blocks

struct SmallSmem {
  double* A;
  double* B;
  double* V;
  double* Z;
  double* T;  // second buffer of A for the double-buffered Jacobi
  int ld;
};

// Sweep stopping test of the Jacobi eigensolvers: the off-diagonal Frobenius
// mass against (4 s eps)^2 times the diagonal mass.  Rounding keeps a
// rotated s x s matrix's off-diagonal part at about eps * ||A|| per entry, so
// a test at eps^2 alone is rarely met and runs sweeps to the cap; at this
// level the eigenvalues are exact to rounding and the eigenvectors to
// s eps ||A|| / gap.
__device__ __forceinline__ double jacobi_stop2(int s) {
  const double t = 4.0 * static_cast<double>(s) * DBL_EPSILON;
  return t * t;
}

__device__ void cta_identity(double* V, int s, int ld) {
  for (int i = threadIdx.x; i < s * s; i += blockDim.x) V[(i / s) * ld + i % s] = (i / s == i % s) ? 1.0 : 0.0;
}

// In-place lower Cholesky; returns false if a pivot is <= tol.
__device__ bool cta_cholesky(double* B, int s, int ld, double tol, int* sflag) {
  for (int j = 0; j < s; ++j) {
    if (threadIdx.x == 0) {
      const double d = B[j * ld + j];
      if (!(d > tol)) {
        *sflag = 1;
      } else {
        B[j * ld + j] = sqrt(d);
        *sflag = 0;
      }
    }
    __syncthreads();
    if (*sflag) return false;
    const double piv = B[j * ld + j];
    for (int i = j + 1 + threadIdx.x; i < s; i += blockDim.x) B[i * ld + j] /= piv;
    __syncthreads();
    const int w = s - j - 1;
    for (int t = threadIdx.x; t < w * w; t += blockDim.x) {
      const int i = j + 1 + t / w, k = j + 1 + t % w;
      if (k <= i) B[i * ld + k] -= B[i * ld + j] * B[k * ld + j];
    }
    __syncthreads();
  }
  return true;
}

// M <- L^-1 M   (M: s x ncol), one thread per column.
__device__ void cta_trsm_left_lower(const double* L, double* M, int s, int ncol, int ld) {
  for (int c = threadIdx.x; c < ncol; c += blockDim.x) {
    for (int i = 0; i < s; ++i) {
      double v = M[i * ld + c];
      for (int k = 0; k < i; ++k) v -= L[i * ld + k] * M[k * ld + c];
      M[i * ld + c] = v / L[i * ld + i];
    }
  }
  __syncthreads();
}

// M <- M L^-T   (M: nrow x s), one thread per row.
__device__ void cta_trsm_right_lowerT(const double* L, double* M, int s, int nrow, int ld) {
  for (int r = threadIdx.x; r < nrow; r += blockDim.x) {
    for (int j = 0; j < s; ++j) {
      double v = M[r * ld + j];
      for (int k = 0; k < j; ++k) v -= M[r * ld + k] * L[j * ld + k];
      M[r * ld + j] = v / L[j * ld + j];
    }
  }
  __syncthreads();
}

// M <- L^-T M   (M: s x ncol), one thread per column (back substitution).
__device__ void cta_trsm_left_lowerT(const double* L, double* M, int s, int ncol, int ld) {
  for (int c = threadIdx.x; c < ncol; c += blockDim.x) {
    for (int i = s - 1; i >= 0; --i) {
      double v = M[i * ld + c];
      for (int k = i + 1; k < s; ++k) v -= L[k * ld + i] * M[k * ld + c];
      M[i * ld + c] = v / L[i * ld + i];
    }
  }
  __syncthreads();
}

__device__ double cta_sum(double v, double* red) {
  v = warp_sum(v);
  const int w = threadIdx.x >> 5;
  if ((threadIdx.x & 31) == 0) red[w] = v;
  __syncthreads();
  double t = 0.0;
  for (int i = 0; i < static_cast<int>(blockDim.x >> 5); ++i) t += red[i];
  __syncthreads();
  return t;
}

// Parallel cyclic Jacobi with one update phase per round: the round's
// disjoint rotations J are applied as A' = J^T A J and V' = V J in a single
// pass into second buffers (every element of A' depends on a 2 x 2 block of
// A), so a round is two barriers.  The rotation angle is taken in single
// precision,
//   t = h sgn(d) / (|d| + sqrt(d^2 + h^2)),  d = a_qq - a_pp, h = 2 a_pq,
//   c = 1/sqrt(1 + t^2), s = t c     (the smaller root of t^2 + 2 (d/h) t - 1),
// and (c, s) are then normalised in double precision by two Newton steps
// (c, s) *= 1.5 - (c^2 + s^2)/2, so every rotation is orthogonal to rounding:
// A and V stay exactly similar / orthogonal, and an angle off by ~1e-7 only
// leaves ~1e-7 of a_pq for the next sweep (quadratic convergence down to that
// level, then a factor ~1e-7 per sweep).  No f64 square root or division on
// the round's critical path.  On return A (diagonal) and V hold the result.
__device__ void cta_jacobi_db(double* A, double* V, double* A2, double* V2, int s, int ld, double* red) {
  __shared__ double al[3 * MAXM + 2], be[3 * MAXM + 2];
  __shared__ int pq[3 * MAXM + 2];
  constexpr int kItems = 9;  // per-thread update items resolved once when 2 s^2 <= 9 * threads
  const int s2 = s + (s & 1);
  const int np = s2 / 2;
  const int nitems = 2 * s * s;
  const bool pre = nitems <= kItems * static_cast<int>(blockDim.x);
  int it_i[kItems], it_j[kItems];
#pragma unroll
  for (int q = 0; q < kItems; ++q) {
    const int t = threadIdx.x + q * blockDim.x;
    const int u = t < s * s ? t : t - s * s;
    it_i[q] = u / s;
    it_j[q] = u - (u / s) * s;
  }
  double* cur = A;
  double* nxt = A2;
  double* vc = V;
  double* vn = V2;
  auto update_item = [&](int t, int i, int j) {
    if (t < s * s) {
      const int qi = pq[i], qj = pq[j];
      nxt[i * ld + j] = al[i] * (al[j] * cur[i * ld + j] + be[j] * cur[i * ld + qj]) +
                        be[i] * (al[j] * cur[qi * ld + j] + be[j] * cur[qi * ld + qj]);
    } else {
      vn[i * ld + j] = al[j] * vc[i * ld + j] + be[j] * vc[i * ld + pq[j]];
    }
  };
  for (int sweep = 0; sweep < 40; ++sweep) {
    double off = 0.0, dia = 0.0;
    for (int t = threadIdx.x; t < s * s; t += blockDim.x) {
      const int i = t / s, j = t - (t / s) * s;
      const double a = cur[i * ld + j];
      if (i == j) dia += a * a; else off += a * a;
    }
    off = cta_sum(off, red);
    dia = cta_sum(dia, red);
    if (!(off > jacobi_stop2(s) * dia)) break;
    for (int r = 0; r < s2 - 1; ++r) {
      for (int p = threadIdx.x; p < np; p += blockDim.x) {
        int a, b;
        if (p == 0) {
          a = r;
          b = s2 - 1;
        } else {
          a = (r + p) % (s2 - 1);
          b = (r - p + s2 - 1) % (s2 - 1);
        }
        if (a > b) {
          const int t = a;
          a = b;
          b = t;
        }
        double c = 1.0, sn = 0.0;
        if (b < s) {
          const double apq = cur[a * ld + b];
          const double app = cur[a * ld + a], aqq = cur[b * ld + b];
          const double tiny = DBL_EPSILON * 1e-3;
          if (fabs(apq) > 1e-300 && apq * apq > tiny * tiny * fabs(app * aqq)) {
            const float d = static_cast<float>(aqq - app), h = static_cast<float>(2.0 * apq);
            const float tf = (d >= 0.0f ? h : -h) / (fabsf(d) + sqrtf(fmaf(d, d, h * h)));
            const float cf = rsqrtf(fmaf(tf, tf, 1.0f));
            c = static_cast<double>(cf);
            sn = static_cast<double>(tf) * static_cast<double>(cf);
#pragma unroll
            for (int k = 0; k < 2; ++k) {
              const double f = fma(-0.5, fma(c, c, sn * sn), 1.5);
              c *= f;
              sn *= f;
            }
          }
        }
        // new row/column a = c a - s b ; new b = s a + c b
        al[a] = c;
        be[a] = -sn;
        pq[a] = (b < s) ? b : a;
        if (b < s) {
          al[b] = c;
          be[b] = sn;
          pq[b] = a;
        }
      }
      __syncthreads();
      if (pre) {
#pragma unroll
        for (int q = 0; q < kItems; ++q) {
          const int t = threadIdx.x + q * blockDim.x;
          if (t < nitems) update_item(t, it_i[q], it_j[q]);
        }
      } else {
        for (int t = threadIdx.x; t < nitems; t += blockDim.x) {
          const int u = t < s * s ? t : t - s * s;
          update_item(t, u / s, u - (u / s) * s);
        }
      }
      __syncthreads();
      double* tmp = cur;
      cur = nxt;
      nxt = tmp;
      tmp = vc;
      vc = vn;
      vn = tmp;
    }
  }
  if (cur != A) {
    for (int t = threadIdx.x; t < s * s; t += blockDim.x) {
      const int i = t / s, j = t - (t / s) * s;
      A[i * ld + j] = cur[i * ld + j];
      V[i * ld + j] = vc[i * ld + j];
    }
  }
  __syncthreads();
}

// Parallel cyclic Jacobi (round-robin pairing): A <- diag, V <- eigenvectors
// (columns).  A is symmetric s x s; V must hold the identity on entry.
__device__ void cta_jacobi(double* A, double* V, int s, int ld, double* red, double* rc, double* rs, int* ra,
                           int* rb) {
  const int s2 = s + (s & 1);
  const int np = s2 / 2;
  // this thread's (pair, index) items of a round, resolved once per call
  constexpr int MAXIT = 12;
  int itp[MAXIT], itk[MAXIT];
  int nit = 0;
  for (int t = threadIdx.x; t < np * s && nit < MAXIT; t += blockDim.x) {
    itp[nit] = t / s;
    itk[nit] = t % s;
    ++nit;
  }
  const bool fast = np * s <= MAXIT * static_cast<int>(blockDim.x);
  for (int sweep = 0; sweep < 40 && fast; ++sweep) {
    double off = 0.0, dia = 0.0;
    for (int t = threadIdx.x; t < s * s; t += blockDim.x) {
      const int i = t / s, j = t % s;
      const double a = A[i * ld + j];
      if (i == j) dia += a * a; else off += a * a;
    }
    off = cta_sum(off, red);
    dia = cta_sum(dia, red);
    if (!(off > jacobi_stop2(s) * dia)) return;
    for (int r = 0; r < s2 - 1; ++r) {
      for (int p = threadIdx.x; p < np; p += blockDim.x) {
        int a, b;
        if (p == 0) {
          a = r;
          b = s2 - 1;
        } else {
          a = (r + p) % (s2 - 1);
          b = (r - p + s2 - 1) % (s2 - 1);
        }
        if (a > b) {
          const int t = a;
          a = b;
          b = t;
        }
        double c = 1.0, sn = 0.0;
        if (b < s) {
          const double apq = A[a * ld + b];
          const double app = A[a * ld + a], aqq = A[b * ld + b];
          if (fabs(apq) > 1e-300 && fabs(apq) > DBL_EPSILON * 1e-3 * sqrt(fabs(app * aqq))) {
            const double theta = (aqq - app) / (2.0 * apq);
            const double t = (theta >= 0.0 ? 1.0 : -1.0) / (fabs(theta) + sqrt(theta * theta + 1.0));
            c = 1.0 / sqrt(t * t + 1.0);
            sn = t * c;
          }
        }
        rc[p] = c;
        rs[p] = sn;
        ra[p] = a;
        rb[p] = (b < s && sn != 0.0) ? b : -1;
      }
      __syncthreads();
      for (int q = 0; q < nit; ++q) {  // rows a, b
        const int p = itp[q], k = itk[q];
        const int a = ra[p], b = rb[p];
        if (b < 0) continue;
        const double x = A[a * ld + k], y = A[b * ld + k];
        A[a * ld + k] = rc[p] * x - rs[p] * y;
        A[b * ld + k] = rs[p] * x + rc[p] * y;
      }
      __syncthreads();
      for (int q = 0; q < nit; ++q) {  // columns a, b (the annihilated pair set to exact zero)
        const int p = itp[q], k = itk[q];
        const int a = ra[p], b = rb[p];
        if (b < 0) continue;
        const double x = A[k * ld + a], y = A[k * ld + b];
        A[k * ld + a] = (k == b) ? 0.0 : rc[p] * x - rs[p] * y;
        A[k * ld + b] = (k == a) ? 0.0 : rs[p] * x + rc[p] * y;
        const double vx = V[k * ld + a], vy = V[k * ld + b];
        V[k * ld + a] = rc[p] * vx - rs[p] * vy;
        V[k * ld + b] = rs[p] * vx + rc[p] * vy;
      }
      __syncthreads();
    }
  }
  if (fast) return;
  // wide problems (more items than the per-thread table holds): plain loops
  for (int sweep = 0; sweep < 40; ++sweep) {
    double off = 0.0, dia = 0.0;
    for (int t = threadIdx.x; t < s * s; t += blockDim.x) {
      const int i = t / s, j = t % s;
      const double a = A[i * ld + j];
      if (i == j) dia += a * a; else off += a * a;
    }
    off = cta_sum(off, red);
    dia = cta_sum(dia, red);
    if (!(off > jacobi_stop2(s) * dia)) break;
    for (int r = 0; r < s2 - 1; ++r) {
      for (int p = threadIdx.x; p < np; p += blockDim.x) {
        int a, b;
        if (p == 0) {
          a = r;
          b = s2 - 1;
        } else {
          a = (r + p) % (s2 - 1);
          b = (r - p + s2 - 1) % (s2 - 1);
        }
        if (a > b) {
          const int t = a;
          a = b;
          b = t;
        }
        double c = 1.0, sn = 0.0;
        if (b < s) {
          const double apq = A[a * ld + b];
          const double app = A[a * ld + a], aqq = A[b * ld + b];
          if (fabs(apq) > 1e-300 && fabs(apq) > DBL_EPSILON * 1e-3 * sqrt(fabs(app * aqq))) {
            const double theta = (aqq - app) / (2.0 * apq);
            const double t = (theta >= 0.0 ? 1.0 : -1.0) / (fabs(theta) + sqrt(theta * theta + 1.0));
            c = 1.0 / sqrt(t * t + 1.0);
            sn = t * c;
          }
        }
        rc[p] = c;
        rs[p] = sn;
        ra[p] = a;
        rb[p] = b < s ? b : -1;
      }
      __syncthreads();
      for (int t = threadIdx.x; t < np * s; t += blockDim.x) {
        const int p = t / s, k = t % s;
        const int a = ra[p], b = rb[p];
        if (b < 0 || rs[p] == 0.0) continue;
        const double x = A[a * ld + k], y = A[b * ld + k];
        A[a * ld + k] = rc[p] * x - rs[p] * y;
        A[b * ld + k] = rs[p] * x + rc[p] * y;
      }
      __syncthreads();
      for (int t = threadIdx.x; t < np * s; t += blockDim.x) {
        const int p = t / s, k = t % s;
        const int a = ra[p], b = rb[p];
        if (b < 0 || rs[p] == 0.0) continue;
        const double x = A[k * ld + a], y = A[k * ld + b];
        A[k * ld + a] = rc[p] * x - rs[p] * y;
        A[k * ld + b] = rs[p] * x + rc[p] * y;
        const double vx = V[k * ld + a], vy = V[k * ld + b];
        V[k * ld + a] = rc[p] * vx - rs[p] * vy;
        V[k * ld + b] = rs[p] * vx + rc[p] * vy;
      }
      __syncthreads();
      // the rotation annihilates a_pq: store the exact zero (the two-phase
      // update leaves O(eps) rounding there, which would never drop below the
      // skip threshold and would keep every sweep rotating)
      for (int p = threadIdx.x; p < np; p += blockDim.x) {
        if (rb[p] >= 0 && rs[p] != 0.0) {
          A[ra[p] * ld + rb[p]] = 0.0;
          A[rb[p] * ld + ra[p]] = 0.0;
        }
      }
      __syncthreads();
    }
  }
}

// order[0..s) = indices of diag(A) ascending (stable); thread 0 only.
__device__ void sort_eigs(const double* A, int s, int ld, int* order) {
  for (int i = 0; i < s; ++i) order[i] = i;
  for (int i = 1; i < s; ++i) {
    const int v = order[i];
    const double key = A[v * ld + v];
    int j = i - 1;
    while (j >= 0 && A[order[j] * ld + order[j]] > key) {
      order[j + 1] = order[j];
      --j;
    }
    order[j + 1] = v;
  }
}

// Generalised Rayleigh-Ritz on the Gram sub-matrices selected by idx[0..s):
// (D GA D) y = theta (D GB D) y.  On success Z[0..s) x [0..nsel) holds
// D L^-T V_sel and theta_out the selected Ritz values.
__device__ bool cta_rr_general(const double* gb, const double* ga, int P, const int* idx, int s, int nsel,
                               int largest, double chol_tol, SmallSmem sm, double* dsc, double* theta_out,
                               double* red, double* rc, double* rs, int* ra, int* rb, int* order, int* sflag) {
  const int ld = sm.ld;
  for (int t = threadIdx.x; t < s * s; t += blockDim.x) {
    const int i = t / s, j = t % s;
    sm.B[i * ld + j] = gb[idx[i] * P + idx[j]];
    sm.A[i * ld + j] = ga[idx[i] * P + idx[j]];
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    int bad = 0;
    for (int i = 0; i < s; ++i) {
      const double d = sm.B[i * ld + i];
      if (!(d > 0.0) || !isfinite(d)) bad = 1;
      dsc[i] = (d > 0.0) ? 1.0 / sqrt(d) : 0.0;
    }
    *sflag = bad;
  }
  __syncthreads();
  if (*sflag) return false;
  for (int t = threadIdx.x; t < s * s; t += blockDim.x) {
    const int i = t / s, j = t % s;
    const double f = dsc[i] * dsc[j];
    sm.B[i * ld + j] *= f;
    sm.A[i * ld + j] *= f;
  }
  __syncthreads();
  if (!cta_cholesky(sm.B, s, ld, chol_tol, sflag)) return false;
  // A <- L^-1 A L^-T
  cta_trsm_left_lower(sm.B, sm.A, s, s, ld);
  cta_trsm_right_lowerT(sm.B, sm.A, s, s, ld);
  // symmetrise
  for (int t = threadIdx.x; t < s * s; t += blockDim.x) {
    const int i = t / s, j = t % s;
    if (i < j) {
      const double v = 0.5 * (sm.A[i * ld + j] + sm.A[j * ld + i]);
      sm.A[i * ld + j] = v;
      sm.A[j * ld + i] = v;
    }
  }
  __syncthreads();
  cta_identity(sm.V, s, ld);
  __syncthreads();
  if (s <= 3 * MAXM) cta_jacobi_db(sm.A, sm.V, sm.T, sm.Z, s, ld, red);
  else cta_jacobi(sm.A, sm.V, s, ld, red, rc, rs, ra, rb);
  if (threadIdx.x == 0) {
    sort_eigs(sm.A, s, ld, order);
    if (largest) {
      for (int i = 0; i < s / 2; ++i) {
        const int t = order[i];
        order[i] = order[s - 1 - i];
        order[s - 1 - i] = t;
      }
    }
    for (int q = 0; q < nsel; ++q) theta_out[q] = sm.A[order[q] * ld + order[q]];
  }
  __syncthreads();
  // Z = V[:, order[0..nsel)]
  for (int t = threadIdx.x; t < s * nsel; t += blockDim.x) {
    const int i = t / nsel, q = t % nsel;
    sm.Z[i * ld + q] = sm.V[i * ld + order[q]];
  }
  __syncthreads();
  cta_trsm_left_lowerT(sm.B, sm.Z, s, nsel, ld);
  for (int t = threadIdx.x; t < s * nsel; t += blockDim.x) {
    const int i = t / nsel, q = t % nsel;
    sm.Z[i * ld + q] *= dsc[i];
  }
  __syncthreads();
  return true;
}

// ---------------------------------------------------------------------------
// The same generalised Rayleigh-Ritz for s <= 16 in one warp, in registers:
// lane j < 16 holds column j of B (then L) and of A (then C = L^-1 A L^-T),
// lane 16 + j holds column j of the eigenvector matrix V.  Every step is
// lane-local arithmetic and warp shuffles; no CTA barrier is involved.
//   * Cholesky, right-looking: at step k lane k forms column k of L, which is
//     broadcast by shuffles, and every lane j > k updates its own column;
//   * C = L^-1 (L^-1 A)^T (A symmetric), each lane solving for its column
//     with L read from shared memory, the transpose through shared memory,
//     then symmetrised;
//   * cyclic Jacobi with the round-robin pairing of 16 columns (15 rounds of
//     8 disjoint rotations per sweep; the round and pair indices are
//     compile-time constants, so every register index is static): a lane
//     exchanges its column with its partner lane for the column rotation and
//     applies the row rotations of all 8 pairs locally.  Rotation angles as in
//     cta_jacobi_db (f32 angle, two f64 Newton normalisation steps: every
//     rotation exactly orthogonal, a_pq left at ~1e-7 of itself for the next
//     sweep, never forced to zero), the same sweep stopping test;
//   * Z = D L^-T V_sel by back substitution, one lane per selected column.
// Padded columns (j >= s) carry B = I, A = 0 and are never selected.
constexpr int WRR = 16;

__device__ __forceinline__ double sel16(const double (&a)[WRR], int i) {
  double v = a[0];
#pragma unroll
  for (int t = 1; t < WRR; ++t)
    if (t == i) v = a[t];
  return v;
}

// One Jacobi sweep over 16 columns as 15 rounds of one fixed shape: the pairs
// are always the positions (2p, 2p + 1), and after every round the content
// moves to new positions by the fixed permutation sigma of the circle method
// (the player at position p goes to sigma[p]), so that every pair of columns
// meets once per sweep and after 15 rounds every column is back where it
// started.  With fixed pair positions every register index is a compile-time
// constant while the round loop stays a runtime loop (one copy of the code).
//   lane k < 16: column of C at position k (rows indexed by position);
//   lane 16 + k: column of V at position k (rows in the original basis).
// Moving to the next round permutes C's rows (a compile-time renaming of the
// registers, C lanes only) and the columns of C and V (one shuffle per row).
__device__ __constant__ int kJacSigmaInv[16] = {2, 1, 4, 0, 6, 3, 8, 5, 10, 7, 12, 9, 14, 11, 15, 13};

__device__ __forceinline__ void warp_jacobi_sweep(double (&col)[WRR], int k, bool isv, int src_lane) {
  const unsigned full = 0xffffffffu;
#pragma unroll 1
  for (int round = 0; round < WRR - 1; ++round) {
    // rotation of the pair (k & ~1, k | 1), formed by its even C lane
    const double dkk = sel16(col, k);
    const double dqq = __shfl_xor_sync(full, dkk, 1);
    const double akq = sel16(col, k ^ 1);
    double c = 1.0, sn = 0.0;
    if (!isv && (k & 1) == 0) {
      const double app = dkk, aqq = dqq, apq = akq;
      const double tiny = DBL_EPSILON * 1e-3;
      if (fabs(apq) > 1e-300 && apq * apq > tiny * tiny * fabs(app * aqq)) {
        const float d = static_cast<float>(aqq - app), h = static_cast<float>(2.0 * apq);
        const float tf = (d >= 0.0f ? h : -h) / (fabsf(d) + sqrtf(fmaf(d, d, h * h)));
        const float cf = rsqrtf(fmaf(tf, tf, 1.0f));
        c = static_cast<double>(cf);
        sn = static_cast<double>(tf) * static_cast<double>(cf);
#pragma unroll
        for (int t = 0; t < 2; ++t) {
          const double f = fma(-0.5, fma(c, c, sn * sn), 1.5);
          c *= f;
          sn *= f;
        }
      }
    }
    // column rotation: new even = c even - s odd ; new odd = s even + c odd
    const double cp = __shfl_sync(full, c, k & ~1);
    const double sp = __shfl_sync(full, sn, k & ~1);
    const bool even = (k & 1) == 0;
#pragma unroll
    for (int i = 0; i < WRR; ++i) {
      const double o = __shfl_xor_sync(full, col[i], 1);
      col[i] = even ? fma(cp, col[i], -sp * o) : fma(sp, o, cp * col[i]);
    }
    // row rotations of the 8 pairs (C lanes)
#pragma unroll
    for (int p = 0; p < WRR / 2; ++p) {
      const double cc = __shfl_sync(full, c, 2 * p);
      const double ss = __shfl_sync(full, sn, 2 * p);
      if (!isv) {
        const double x = col[2 * p], y = col[2 * p + 1];
        col[2 * p] = fma(cc, x, -ss * y);
        col[2 * p + 1] = fma(ss, x, cc * y);
      }
    }
    // next round's positions: rows of C renamed (row q takes row kJacSigmaInv[q]),
    // columns of C and V moved
    double t[WRR];
    t[0] = isv ? col[0] : col[2];
    t[1] = isv ? col[1] : col[1];
    t[2] = isv ? col[2] : col[4];
    t[3] = isv ? col[3] : col[0];
    t[4] = isv ? col[4] : col[6];
    t[5] = isv ? col[5] : col[3];
    t[6] = isv ? col[6] : col[8];
    t[7] = isv ? col[7] : col[5];
    t[8] = isv ? col[8] : col[10];
    t[9] = isv ? col[9] : col[7];
    t[10] = isv ? col[10] : col[12];
    t[11] = isv ? col[11] : col[9];
    t[12] = isv ? col[12] : col[14];
    t[13] = isv ? col[13] : col[11];
    t[14] = isv ? col[14] : col[15];
    t[15] = isv ? col[15] : col[13];
#pragma unroll
    for (int i = 0; i < WRR; ++i) col[i] = __shfl_sync(full, t[i], src_lane);
  }
}

// sh: 2 * 16 * 16 doubles of shared memory; Z (ldz) and theta_out in shared memory.
__device__ bool warp_rr_general(const double* gb, const double* ga, int P, const int* idx, int s, int nsel,
                                int largest, double chol_tol, double* Z, int ldz, double* sh, double* theta_out) {
  const unsigned full = 0xffffffffu;
  const int lane = threadIdx.x & 31;
  const int j = lane & (WRR - 1);
  const bool isv = lane >= WRR;
  const bool live = j < s;
  // D scaling from diag(B)
  double dj = 0.0;
  int bad = 0;
  if (!isv && live) {
    const double d = gb[idx[j] * P + idx[j]];
    bad = (!(d > 0.0) || !isfinite(d)) ? 1 : 0;
    dj = d > 0.0 ? 1.0 / sqrt(d) : 0.0;
  }
  if (__any_sync(full, bad)) return false;
  double colB[WRR], col[WRR];
#pragma unroll
  for (int i = 0; i < WRR; ++i) {
    const double di = __shfl_sync(full, dj, i);
    if (!isv && live && i < s) {
      const double f = di * dj;
      colB[i] = gb[idx[i] * P + idx[j]] * f;
      col[i] = ga[idx[i] * P + idx[j]] * f;
    } else {
      colB[i] = (!isv && i == j) ? 1.0 : 0.0;
      col[i] = 0.0;
    }
  }
  // Cholesky B = L L^T (lanes 0..15; the V lanes follow the shuffles)
  int fail = 0;
#pragma unroll
  for (int k = 0; k < WRR; ++k) {
    const double pk = __shfl_sync(full, colB[k], k);
    if (k < s && !(pk > chol_tol)) fail = 1;
    const double piv = sqrt(fmax(pk, 1e-300));
    const double inv = 1.0 / piv;
    if (j == k && !isv) {
      colB[k] = piv;
#pragma unroll
      for (int i = k + 1; i < WRR; ++i) colB[i] *= inv;
    }
    double lk[WRR];
#pragma unroll
    for (int i = k + 1; i < WRR; ++i) lk[i] = __shfl_sync(full, colB[i], k);
    double ljk = 0.0;
#pragma unroll
    for (int i = k + 1; i < WRR; ++i)
      if (i == j) ljk = lk[i];
    if (!isv && j > k) {
#pragma unroll
      for (int i = k + 1; i < WRR; ++i) colB[i] = fma(-lk[i], ljk, colB[i]);
    }
  }
  if (fail) return false;
  double* Ls = sh;              // L, row-major 16 x 16 (lower part)
  double* Ts = sh + WRR * WRR;  // transpose staging
  if (!isv) {
#pragma unroll
    for (int i = 0; i < WRR; ++i) Ls[i * WRR + j] = (i >= j) ? colB[i] : 0.0;
  }
  __syncwarp();
  // Y = L^-1 A (column j), then C = L^-1 Y^T
#pragma unroll
  for (int pass = 0; pass < 2; ++pass) {
    if (!isv) {
      double y[WRR];
#pragma unroll
      for (int i = 0; i < WRR; ++i) {
        double v = col[i];
#pragma unroll
        for (int k = 0; k < i; ++k) v = fma(-Ls[i * WRR + k], y[k], v);
        y[i] = v / Ls[i * WRR + i];
      }
#pragma unroll
      for (int i = 0; i < WRR; ++i) Ts[i * WRR + j] = y[i];
    }
    __syncwarp();
    if (!isv) {
#pragma unroll
      for (int i = 0; i < WRR; ++i) col[i] = Ts[j * WRR + i];  // column j of Y^T = row j of Y
    }
    __syncwarp();
  }
  // symmetrise C (col holds row j of C)
  if (!isv) {
#pragma unroll
    for (int i = 0; i < WRR; ++i) Ts[i * WRR + j] = col[i];
  }
  __syncwarp();
  if (!isv) {
#pragma unroll
    for (int i = 0; i < WRR; ++i) col[i] = 0.5 * (col[i] + Ts[j * WRR + i]);
  } else {
#pragma unroll
    for (int i = 0; i < WRR; ++i) col[i] = (i == j) ? 1.0 : 0.0;  // V = I
  }
  __syncwarp();
  const int src_lane = (isv ? WRR : 0) + kJacSigmaInv[j];
  for (int sweep = 0; sweep < 40; ++sweep) {
    double off = 0.0, dia = 0.0;
    if (!isv) {
#pragma unroll
      for (int i = 0; i < WRR; ++i) {
        const double v = col[i] * col[i];
        if (i == j) dia += v; else off += v;
      }
    }
#pragma unroll
    for (int o = 16; o >= 1; o >>= 1) {
      off += __shfl_xor_sync(full, off, o);
      dia += __shfl_xor_sync(full, dia, o);
    }
    if (!(off > jacobi_stop2(s) * dia)) break;
    warp_jacobi_sweep(col, j, isv, src_lane);
  }
  // eigenvalues (the diagonal) ranked among the live columns
  const double lam = isv ? 0.0 : sel16(col, j);
  int rank = 0;
#pragma unroll
  for (int i = 0; i < WRR; ++i) {
    const double li = __shfl_sync(full, lam, i);
    if (i < s && live && !isv) {
      const bool before = largest ? (li > lam || (li == lam && i < j)) : (li < lam || (li == lam && i < j));
      if (before) ++rank;
    }
  }
  int* ord = reinterpret_cast<int*>(Ts);
  if (!isv && live && rank < nsel) {
    ord[rank] = j;
    theta_out[rank] = lam;
  }
  __syncwarp();
  // Z[:, q] = D L^-T V[:, ord[q]]: lane q < nsel takes column ord[q] from the V lanes
  const int src = WRR + ((lane < nsel) ? ord[lane] : 0);
  double v[WRR], dall[WRR];
#pragma unroll
  for (int i = 0; i < WRR; ++i) {
    v[i] = __shfl_sync(full, col[i], src);
    dall[i] = __shfl_sync(full, dj, i);
  }
  if (lane < nsel) {
    double z[WRR];
#pragma unroll
    for (int i = WRR - 1; i >= 0; --i) {
      double t = v[i];
#pragma unroll
      for (int k = i + 1; k < WRR; ++k) t = fma(-Ls[k * WRR + i], z[k], t);
      z[i] = t / Ls[i * WRR + i];
    }
#pragma unroll
    for (int i = 0; i < WRR; ++i)
      if (i < s) Z[i * ldz + lane] = z[i] * dall[i];
  }
  __syncwarp();
  return true;
}

// The generalised Rayleigh-Ritz of cta_rr_general with its serial sections
// made parallel: the D-scale factors one per thread; a right-looking
// Cholesky with one barrier per pivot (every thread recomputes the pivot, the
// trailing update reads the unscaled pivot column, and the column scaling is
// one pass at the end); L^-1 formed once, one column per thread, so that
// C = L^-1 A L^-T and the Ritz vectors D L^-T V_sel are parallel matrix
// products instead of three one-thread-per-column triangular solves; the
// selection order by ranks.  Same results as cta_rr_general up to rounding.
__device__ bool cta_rr_general_par(const double* gb, const double* ga, int P, const int* idx, int s, int nsel,
                                   int largest, double chol_tol, SmallSmem sm, double* dsc, double* theta_out,
                                   double* red, int* order, int* sflag) {
  __shared__ double lsq[3 * MAXM];  // sqrt of the pivots, then 1 / L_jj
  const int ld = sm.ld;
  const int nt = blockDim.x;
  if (threadIdx.x == 0) *sflag = 0;
  for (int t = threadIdx.x; t < s * s; t += nt) {
    const int i = t / s, j = t % s;
    sm.B[i * ld + j] = gb[idx[i] * P + idx[j]];
    sm.A[i * ld + j] = ga[idx[i] * P + idx[j]];
  }
  __syncthreads();
  for (int i = threadIdx.x; i < s; i += nt) {
    const double d = sm.B[i * ld + i];
    const bool ok = d > 0.0 && isfinite(d);
    if (!ok) atomicExch(sflag, 1);
    dsc[i] = ok ? 1.0 / sqrt(d) : 0.0;
  }
  __syncthreads();
  if (*sflag) return false;
  for (int t = threadIdx.x; t < s * s; t += nt) {
    const int i = t / s, j = t % s;
    const double f = dsc[i] * dsc[j];
    sm.B[i * ld + j] *= f;
    sm.A[i * ld + j] *= f;
  }
  __syncthreads();
  // ---- Cholesky, one barrier per pivot ----
  for (int j = 0; j < s; ++j) {
    const double piv = sm.B[j * ld + j];
    if (!(piv > chol_tol)) return false;  // the same value in every thread
    const double inv2 = 1.0 / piv;        // (b_ij / l_jj)(b_kj / l_jj) = b_ij b_kj / b_jj
    if (threadIdx.x == 0) lsq[j] = sqrt(piv);
    const int w = s - j - 1;
    for (int t = threadIdx.x; t < w * w; t += nt) {
      const int i = j + 1 + t / w, k = j + 1 + t % w;
      if (k <= i) sm.B[i * ld + k] -= sm.B[i * ld + j] * sm.B[k * ld + j] * inv2;
    }
    __syncthreads();
  }
  for (int t = threadIdx.x; t < s * s; t += nt) {  // finish the columns: l_ij = b_ij / sqrt(b_jj)
    const int i = t / s, j = t % s;
    if (i > j) sm.B[i * ld + j] /= lsq[j];
    else if (i == j) sm.B[i * ld + i] = lsq[i];
  }
  __syncthreads();
  for (int i = threadIdx.x; i < s; i += nt) lsq[i] = 1.0 / lsq[i];
  __syncthreads();
  // ---- M = L^-1 (lower), one column per thread, into Z ----
  for (int c = threadIdx.x; c < s; c += nt) {
    for (int i = 0; i < c; ++i) sm.Z[i * ld + c] = 0.0;
    sm.Z[c * ld + c] = lsq[c];
    for (int i = c + 1; i < s; ++i) {
      double v = 0.0;
      for (int k = c; k < i; ++k) v = fma(sm.B[i * ld + k], sm.Z[k * ld + c], v);
      sm.Z[i * ld + c] = -v * lsq[i];
    }
  }
  __syncthreads();
  // keep M in B (L is no longer needed)
  for (int t = threadIdx.x; t < s * s; t += nt) {
    const int i = t / s, j = t % s;
    sm.B[i * ld + j] = sm.Z[i * ld + j];
  }
  __syncthreads();
  // ---- C = M A M^T: Y = M A into T, then C = Y M^T into A ----
  for (int t = threadIdx.x; t < s * s; t += nt) {
    const int i = t / s, j = t % s;
    double v = 0.0;
    for (int k = 0; k <= i; ++k) v = fma(sm.B[i * ld + k], sm.A[k * ld + j], v);
    sm.T[i * ld + j] = v;
  }
  __syncthreads();
  for (int t = threadIdx.x; t < s * s; t += nt) {
    const int i = t / s, j = t % s;
    if (j < i) continue;  // upper triangle, mirrored below
    double v = 0.0;
    for (int k = 0; k <= j; ++k) v = fma(sm.T[i * ld + k], sm.B[j * ld + k], v);
    double u = 0.0;  // the (j, i) entry, for the symmetrised average
    for (int k = 0; k <= i; ++k) u = fma(sm.T[j * ld + k], sm.B[i * ld + k], u);
    const double a = 0.5 * (v + u);
    sm.A[i * ld + j] = a;
    sm.A[j * ld + i] = a;
  }
  __syncthreads();
  cta_identity(sm.V, s, ld);
  __syncthreads();
  cta_jacobi_db(sm.A, sm.V, sm.T, sm.Z, s, ld, red);
  // ---- selection by ranks (ascending, or descending for `largest`; ties by index) ----
  for (int i = threadIdx.x; i < s; i += nt) {
    const double di = sm.A[i * ld + i];
    int rank = 0;
    for (int j = 0; j < s; ++j) {
      const double dj = sm.A[j * ld + j];
      // ascending and stable; for `largest` the reverse of that order
      const bool before = largest ? (dj > di || (dj == di && j > i)) : (dj < di || (dj == di && j < i));
      rank += before ? 1 : 0;
    }
    order[rank] = i;
  }
  __syncthreads();
  for (int q = threadIdx.x; q < nsel; q += nt) theta_out[q] = sm.A[order[q] * ld + order[q]];
  // ---- Z = D M^T V_sel ----
  for (int t = threadIdx.x; t < s * nsel; t += nt) {
    const int i = t / nsel, q = t % nsel;
    const int c = order[q];
    double v = 0.0;
    for (int k = i; k < s; ++k) v = fma(sm.B[k * ld + i], sm.V[k * ld + c], v);
    sm.Z[i * ld + q] = v * dsc[i];
  }
  __syncthreads();
  return true;
}

// Rayleigh-Ritz of the small step: the shared-memory CTA routines (PAR: the
// parallel form, the default for the CTA kernels; on a single-warp CTA their
// barriers are warp-cheap), or, with REG, the register-resident warp version
// (SPECTRAL_INIT_SMALL_STEP=reg).
template <int NT, bool REG, bool PAR>
__device__ bool rr_general(const double* gb, const double* ga, int P, const int* idx, int s, int nsel, int largest,
                           double chol_tol, SmallSmem sm, double* dsc, double* theta_out, double* red, double* rc,
                           double* rs, int* ra, int* rb, int* order, int* sflag) {
  if constexpr (NT == 32 && REG) {
    if (s <= WRR)
      return warp_rr_general(gb, ga, P, idx, s, nsel, largest, chol_tol, sm.Z, sm.ld, sm.T, theta_out);
  }
  if constexpr (PAR) {
    if (s <= 3 * MAXM)
      return cta_rr_general_par(gb, ga, P, idx, s, nsel, largest, chol_tol, sm, dsc, theta_out, red, order, sflag);
  }
  return cta_rr_general(gb, ga, P, idx, s, nsel, largest, chol_tol, sm, dsc, theta_out, red, rc, rs, ra, rb, order,
                        sflag);
}

// `ctrl` points to the CTA's shared-memory copy of the control block.
template <int NT, bool REG, bool PAR>
__device__ void small_step_body(LobpcgCtrl* ctrl, const double* __restrict__ gram, int ns, int mode,
                                double* smem) {
  __shared__ double red[ST_WIDE / 32];
  __shared__ double rc[SMAX / 2 + 1], rs[SMAX / 2 + 1], dsc[3 * MAXM], theta[MAXM], rn[MAXM];
  __shared__ int ra[SMAX / 2 + 1], rb[SMAX / 2 + 1], order[3 * MAXM], idx[3 * MAXM];
  __shared__ int sflag, sdone, s_na, s_withp;
  const int LDS = 3 * MAXM;
  SmallSmem sm{smem, smem + LDS * LDS, smem + 2 * LDS * LDS, smem + 3 * LDS * LDS, smem + 4 * LDS * LDS, LDS};
  const int m = ctrl->m;
  const int P = ns * m;
  const double* gb = gram;
  const double* ga = gram + P * P;
  if (threadIdx.x == 0) {
    sdone = ctrl->done;
    // iterations queued after convergence: the final best copy already happened
    if (sdone && mode == SM_ITER) ctrl->copy_best = 0;
  }
  __syncthreads();
  if (sdone) return;

  if (mode == SM_INIT) {
    for (int i = threadIdx.x; i < m; i += blockDim.x) idx[i] = i;
    __syncthreads();
    const bool ok = rr_general<NT, REG, PAR>(gb, ga, P, idx, m, m, ctrl->largest, ctrl->chol_tol, sm, dsc, theta, red, rc,
                                   rs, ra, rb, order, &sflag);
    if (threadIdx.x == 0) {
      ctrl->iter = 0;
      ctrl->copy_best = 0;
      ctrl->has_p = 0;
      ctrl->p_valid = 0;
      ctrl->best_sum = DBL_MAX;
      ctrl->best_iter = -1;
      ctrl->n_active = m;
      for (int c = 0; c < MAXM; ++c) ctrl->active[c] = c < m ? 1 : 0;
      if (!ok) {
        ctrl->done = 1;
        ctrl->status = ST_BREAKDOWN;
      } else {
        for (int q = 0; q < m; ++q) ctrl->lam[q] = theta[q];
      }
    }
    __syncthreads();
    if (ok) {
      for (int t = threadIdx.x; t < MAXM * MAXM; t += blockDim.x) {
        const int i = t / MAXM, q = t % MAXM;
        ctrl->Cx[t] = (i < m && q < m) ? sm.Z[i * LDS + q] : 0.0;
        ctrl->Cr[t] = 0.0;
        ctrl->Cp[t] = 0.0;
      }
    }
    return;
  }

  if (mode == SM_RR_PLAIN) {
    for (int t = threadIdx.x; t < m * m; t += blockDim.x) sm.A[(t / m) * LDS + t % m] = ga[t];
    __syncthreads();
    cta_identity(sm.V, m, LDS);
    __syncthreads();
    cta_jacobi_db(sm.A, sm.V, sm.T, sm.Z, m, LDS, red);
    if (threadIdx.x == 0) {
      sort_eigs(sm.A, m, LDS, order);
      for (int q = 0; q < m; ++q) ctrl->lam[q] = sm.A[order[q] * LDS + order[q]];
    }
    __syncthreads();
    for (int t = threadIdx.x; t < MAXM * MAXM; t += blockDim.x) {
      const int i = t / MAXM, q = t % MAXM;
      ctrl->Cx[t] = (i < m && q < m) ? sm.V[i * LDS + order[q]] : 0.0;
    }
    return;
  }

  if (mode == SM_CHOLQR) {
    for (int t = threadIdx.x; t < m * m; t += blockDim.x) sm.B[(t / m) * LDS + t % m] = gb[t];
    __syncthreads();
    const bool ok = cta_cholesky(sm.B, m, LDS, 0.0, &sflag);
    if (ok) {
      cta_identity(sm.Z, m, LDS);
      __syncthreads();
      cta_trsm_left_lowerT(sm.B, sm.Z, m, m, LDS);
    }
    for (int t = threadIdx.x; t < MAXM * MAXM; t += blockDim.x) {
      const int i = t / MAXM, q = t % MAXM;
      ctrl->Cx[t] = (ok && i < m && q < m) ? sm.Z[i * LDS + q] : 0.0;
    }
    if (threadIdx.x == 0) ctrl->status = ok ? ST_CONVERGED : ST_BREAKDOWN;
    return;
  }

  // ---- SM_ITER --------------------------------------------------------------
  if (threadIdx.x == 0) {
    const int k = ctrl->k_wanted;
    double sum = 0.0;
    for (int c = 0; c < m; ++c) {
      const double g = gb[(m + c) * P + (m + c)];
      rn[c] = sqrt(g > 0.0 ? g : 0.0);
      ctrl->rnorm[c] = rn[c];
      if (c < k) sum += rn[c];
    }
    int copy = 0;
    if (ctrl->best_sum > sum) {
      ctrl->best_sum = sum;
      ctrl->best_iter = ctrl->iter;
      for (int c = 0; c < m; ++c) {
        ctrl->best_lam[c] = ctrl->lam[c];
        ctrl->best_rnorm[c] = rn[c];
      }
      copy = 1;
    }
    ctrl->copy_best = copy;
    int na_wanted = 0;
    for (int c = 0; c < m; ++c) {
      if (c < k) {
        ctrl->active[c] = (ctrl->active[c] && rn[c] > ctrl->tol) ? 1 : 0;
        na_wanted += ctrl->active[c];
      } else {
        ctrl->active[c] = 1;
      }
    }
    int done = 0;
    if (na_wanted == 0) {
      done = 1;
      ctrl->status = ST_CONVERGED;
    } else if (ctrl->iter >= ctrl->maxiter) {
      done = 1;
      ctrl->status = ST_MAXITER;
    }
    ctrl->done = done;
    sdone = done;
    if (!done) ctrl->iter += 1;
    int na = 0;
    for (int c = 0; c < m; ++c)
      if (ctrl->active[c]) idx[m + na++] = m + c;
    for (int c = 0; c < m; ++c) idx[c] = c;
    s_na = na;
    s_withp = ctrl->p_valid;
  }
  __syncthreads();
  if (sdone) return;
  const int na = s_na;
  bool ok = false;
  int withp = s_withp;
  if (withp) {
    if (threadIdx.x == 0) {
      int q = 0;
      for (int c = 0; c < m; ++c)
        if (ctrl->active[c]) idx[m + na + q++] = 2 * m + c;
    }
    __syncthreads();
    ok = rr_general<NT, REG, PAR>(gb, ga, P, idx, m + 2 * na, m, ctrl->largest, ctrl->chol_tol, sm, dsc, theta, red, rc, rs,
                        ra, rb, order, &sflag);
    if (!ok) withp = 0;
  }
  if (!ok) {
    ok = rr_general<NT, REG, PAR>(gb, ga, P, idx, m + na, m, ctrl->largest, ctrl->chol_tol, sm, dsc, theta, red, rc, rs, ra,
                        rb, order, &sflag);
  }
  if (!ok) {
    if (threadIdx.x == 0) {
      ctrl->done = 1;
      ctrl->status = ST_BREAKDOWN;
    }
    return;
  }
  // scatter the coefficients
  for (int t = threadIdx.x; t < MAXM * MAXM; t += blockDim.x) {
    ctrl->Cx[t] = 0.0;
    ctrl->Cr[t] = 0.0;
    ctrl->Cp[t] = 0.0;
  }
  __syncthreads();
  for (int t = threadIdx.x; t < (m + na * (withp ? 2 : 1)) * m; t += blockDim.x) {
    const int row = t / m, q = t % m;
    const double v = sm.Z[row * LDS + q];
    const int col = idx[row];
    if (col < m)
      ctrl->Cx[col * MAXM + q] = v;
    else if (col < 2 * m)
      ctrl->Cr[(col - m) * MAXM + q] = v;
    else
      ctrl->Cp[(col - 2 * m) * MAXM + q] = v;
  }
  if (threadIdx.x == 0) {
    for (int q = 0; q < m; ++q) ctrl->lam[q] = theta[q];
    ctrl->has_p = withp;
    ctrl->p_valid = 1;
  }
}

// The control block is staged in shared memory for the whole step (the step
// is a long chain of small dependent updates) and written back at the end.
template <int NT, bool REG = false, bool PAR = false>
__global__ void __launch_bounds__(NT, 1) k_small_step(LobpcgCtrl* ctrl, const double* __restrict__ gram, int ns,
                                                   int mode) {
  extern __shared__ double smem[];
  __shared__ LobpcgCtrl sctrl;
  static_assert(sizeof(LobpcgCtrl) % sizeof(double) == 0, "control block must be a whole number of words");
  constexpr int W = sizeof(LobpcgCtrl) / sizeof(double);
  double* dst = reinterpret_cast<double*>(&sctrl);
  const double* src = reinterpret_cast<const double*>(ctrl);
  for (int i = threadIdx.x; i < W; i += blockDim.x) dst[i] = src[i];
  __syncthreads();
  small_step_body<NT, REG, PAR>(&sctrl, gram, ns, mode, smem);
  __syncthreads();
  double* back = reinterpret_cast<double*>(ctrl);
  for (int i = threadIdx.x; i < W; i += blockDim.x) back[i] = dst[i];
}

__global__ void __launch_bounds__(ST) k_small_dense(const double* __restrict__ a, int s, int mode, double* evals,
                                                    double* evecs) {
  extern __shared__ double smem[];
  __shared__ double red[ST / 32];
  __shared__ double rc[SMAX / 2 + 1], rs[SMAX / 2 + 1];
  __shared__ int ra[SMAX / 2 + 1], rb[SMAX / 2 + 1], order[SMAX];
  __shared__ int sflag;
  const int ld = SMAX;
  double* A = smem;
  double* V = smem + SMAX * SMAX;
  for (int t = threadIdx.x; t < s * s; t += blockDim.x) A[(t / s) * ld + t % s] = a[t];
  __syncthreads();
  if (mode == SM_RR_PLAIN) {
    cta_identity(V, s, ld);
    __syncthreads();
    cta_jacobi(A, V, s, ld, red, rc, rs, ra, rb);
    if (threadIdx.x == 0) {
      sort_eigs(A, s, ld, order);
      for (int q = 0; q < s; ++q) evals[q] = A[order[q] * ld + order[q]];
    }
    __syncthreads();
    for (int t = threadIdx.x; t < s * s; t += blockDim.x) {
      const int i = t / s, q = t % s;
      evecs[t] = V[i * ld + order[q]];
    }
  } else {
    const bool ok = cta_cholesky(A, s, ld, 0.0, &sflag);
    if (ok) {
      cta_identity(V, s, ld);
      __syncthreads();
      cta_trsm_left_lowerT(A, V, s, s, ld);
      for (int t = threadIdx.x; t < s * s; t += blockDim.x) evecs[t] = V[(t / s) * ld + t % s];
    }
    if (threadIdx.x == 0) evals[0] = ok ? 1.0 : 0.0;
  }
}

}  // namespace

// SPECTRAL_INIT_SMALL_STEP=cta keeps the multi-warp small step for every
// width (the single-warp version is the default up to 16 columns); read on
// every call, so one process can compare both.
// SPECTRAL_INIT_SMALL_STEP = warp (a single warp running the shared-memory
// routines, up to 16 columns) | reg (a single warp, register-resident
// Rayleigh-Ritz, up to 16 columns); default: the 128-thread CTA, measured
// fastest at n = 1M (FP64 solve 103 ms against 107 / 123 ms).  Read on every
// launch, so one process can compare them.
int small_step_variant() {
  const char* e = std::getenv("SPECTRAL_INIT_SMALL_STEP");
  if (e == nullptr) return 1;
  const std::string v(e);
  return v == "warp" ? 0 : (v == "reg" ? 2 : (v == "serial" ? 3 : 1));
}

void small_step_dev(const Exec& ex, LobpcgCtrl* ctrl, const double* gram, int ns, int mode, int m) {
  const int LDS = 3 * MAXM;
  const size_t smem = sizeof(double) * 5 * LDS * LDS;
  static std::atomic<bool> attr_set[128];
  if (ex.device >= 0 && ex.device < 128 && !attr_set[ex.device]) {
    SI_CUDA(cudaFuncSetAttribute(k_small_step<ST>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 static_cast<int>(smem)));
    SI_CUDA(cudaFuncSetAttribute(k_small_step<ST_WIDE>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 static_cast<int>(smem)));
    SI_CUDA(cudaFuncSetAttribute(k_small_step<ST, false, true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 static_cast<int>(smem)));
    SI_CUDA(cudaFuncSetAttribute(k_small_step<ST_WIDE, false, true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 static_cast<int>(smem)));
    SI_CUDA(cudaFuncSetAttribute(k_small_step<32>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 static_cast<int>(smem)));
    SI_CUDA(cudaFuncSetAttribute(k_small_step<32, true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 static_cast<int>(smem)));
    attr_set[ex.device] = true;
  }
  // the Rayleigh-Ritz problem has up to ns * m rows: up to 16 fit one warp's
  // registers; wider blocks get a CTA, the widest the most threads
  // (SPECTRAL_INIT_SMALL_STEP: unset, the CTA with the parallel Rayleigh-Ritz;
  // serial, the CTA with one-thread-per-column triangular solves; warp / reg,
  // one warp)
  const int variant = small_step_variant();
  const bool par = variant != 3;
  if (ns * m > 24) {
    if (par) k_small_step<ST_WIDE, false, true><<<1, ST_WIDE, smem, ex.stream>>>(ctrl, gram, ns, mode);
    else k_small_step<ST_WIDE><<<1, ST_WIDE, smem, ex.stream>>>(ctrl, gram, ns, mode);
  } else if (ns * m > WRR || variant == 1 || variant == 3) {
    if (par) k_small_step<ST, false, true><<<1, ST, smem, ex.stream>>>(ctrl, gram, ns, mode);
    else k_small_step<ST><<<1, ST, smem, ex.stream>>>(ctrl, gram, ns, mode);
  } else if (variant == 2)
    k_small_step<32, true><<<1, 32, smem, ex.stream>>>(ctrl, gram, ns, mode);
  else
    k_small_step<32><<<1, 32, smem, ex.stream>>>(ctrl, gram, ns, mode);
  SI_LAUNCH_CHECK();
}

void small_dense_dev(const Exec& ex, const double* a, int s, int mode, double* evals, double* evecs) {
  SI_REQUIRE(s >= 1 && s <= SMAX, SI_INVALID_ARGUMENT, "small_dense: size out of range");
  const size_t smem = sizeof(double) * 2 * SMAX * SMAX;
  static std::atomic<bool> attr_set[128];
  if (ex.device >= 0 && ex.device < 128 && !attr_set[ex.device]) {
    SI_CUDA(cudaFuncSetAttribute(k_small_dense, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem)));
    attr_set[ex.device] = true;
  }
  k_small_dense<<<1, ST, smem, ex.stream>>>(a, s, mode, evals, evecs);
  SI_LAUNCH_CHECK();
}

}  // namespace si
