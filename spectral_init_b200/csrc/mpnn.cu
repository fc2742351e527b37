// Learned warm start: a 3-layer message-passing network that predicts the
// starting block of LOBPCG, with its forward pass, backward pass and Adam
// update on the device.
//
// Network (hidden width 64, bf16 weights and activations, f32 accumulation):
//   H0    = [s, p1..p4, 0 ...]                      per-node features, [n x 64]
//           s = sqrt(d) scaled to unit RMS, p_j = Chebyshev-filtered random
//           probes (degree 8 on [0.1, 2], the starting filter of the solver),
//           unit RMS
//   A_l   = [H_l | Ahat H_l]                        [n x 128], Ahat = D^-1/2 W D^-1/2
//   H_l+1 = ReLU(A_l W_l + b_l)                     l = 0, 1, 2 (W_l: 128 x 64)
//   Y     = A_3 W_out + b_out                       [n x 16], first k columns used
// Loss (subspace projection against target eigenvectors V, n x k, orthonormal):
//   L = 1 - tr(G^-1 M) / k,  G = Y^T Y,  C = V^T Y,  M = C^T C
//   dL/dY = -(2/k) (V C G^-1 - Y G^-1 M G^-1)
// The dense layers run on the tcgen05 GEMM (umma_gemm.cu); message passing
// is a warp-per-row CSR product over bf16 rows (128 B per neighbour).
// Backpropagation through Ahat uses Ahat^T = Ahat (symmetric graphs).
#include <algorithm>
#include <cmath>
#include <numeric>
#include <vector>

#include "mpnn.h"

namespace si {

namespace {

constexpr int kT = 256;

int grid_for_rows(const Exec& ex, int64_t items, int per_sm = 8) {
  const int64_t need = (items + kT - 1) / kT;
  return static_cast<int>(std::max<int64_t>(1, std::min<int64_t>(need, int64_t(ex.sms) * per_sm)));
}

// ---- features ------------------------------------------------------------------
// A0 row i: [s_i * cs, p_i1 * c1, .., p_i4 * c4, 0 .. 0 | right half untouched]
__global__ void k_features(int64_t n, const double* __restrict__ sqrt_deg, double s_scale,
                           const float* __restrict__ probes, int pld, const double* __restrict__ p_scale,
                           const float* __restrict__ given, __nv_bfloat16* __restrict__ a0) {
  const int64_t total = n * kMpnnHidden;
  const int64_t stride = static_cast<int64_t>(gridDim.x) * blockDim.x;
  for (int64_t e = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; e < total; e += stride) {
    const int64_t i = e / kMpnnHidden;
    const int c = static_cast<int>(e % kMpnnHidden);
    float v = 0.0f;
    if (c < kMpnnFeatures) {
      if (given != nullptr) {
        v = given[i * kMpnnFeatures + c];
      } else if (c == 0) {
        v = static_cast<float>(sqrt_deg[i] * s_scale);
      } else {
        v = static_cast<float>(static_cast<double>(probes[i * pld + (c - 1)]) * p_scale[c - 1]);
      }
    }
    a0[i * kMpnnCat + c] = __float2bfloat16_rn(v);
  }
}

// ---- message passing: A[:, 64:128] = Ahat A[:, 0:64] (Ahat = -offdiag(L)) -------------
__global__ void __launch_bounds__(kT) k_mp_forward(int64_t n, const uint64_t* __restrict__ indptr,
                                                   const uint32_t* __restrict__ indices,
                                                   const float* __restrict__ vals, __nv_bfloat16* __restrict__ a) {
  const int lane = threadIdx.x & 31;
  const int64_t warps = static_cast<int64_t>(gridDim.x) * (kT / 32);
  for (int64_t i = blockIdx.x * static_cast<int64_t>(kT / 32) + (threadIdx.x >> 5); i < n; i += warps) {
    const uint64_t e0 = indptr[i], e1 = indptr[i + 1];
    float2 acc = make_float2(0.f, 0.f);
    uint64_t e = e0;
    for (; e + 4 <= e1; e += 4) {
      uint32_t j[4];
      float w[4];
      __nv_bfloat162 h[4];
#pragma unroll
      for (int u = 0; u < 4; ++u) {
        j[u] = __ldg(indices + e + u);
        w[u] = __ldg(vals + e + u);
      }
#pragma unroll
      for (int u = 0; u < 4; ++u)
        h[u] = *reinterpret_cast<const __nv_bfloat162*>(a + static_cast<int64_t>(j[u]) * kMpnnCat + 2 * lane);
#pragma unroll
      for (int u = 0; u < 4; ++u) {
        const float2 f = __bfloat1622float2(h[u]);
        acc.x -= w[u] * f.x;
        acc.y -= w[u] * f.y;
      }
    }
    for (; e < e1; ++e) {
      const uint32_t j = __ldg(indices + e);
      const float w = __ldg(vals + e);
      const float2 f = __bfloat1622float2(
          *reinterpret_cast<const __nv_bfloat162*>(a + static_cast<int64_t>(j) * kMpnnCat + 2 * lane));
      acc.x -= w * f.x;
      acc.y -= w * f.y;
    }
    *reinterpret_cast<__nv_bfloat162*>(a + i * kMpnnCat + kMpnnHidden + 2 * lane) =
        __floats2bfloat162_rn(acc.x, acc.y);
  }
}

// ---- backward through [H | Ahat H] and the ReLU of H:
//   dH = dA[:, 0:64] + Ahat dA[:, 64:128];  dZ = dH * (H > 0)  (bf16)
__global__ void __launch_bounds__(kT) k_mp_backward(int64_t n, const uint64_t* __restrict__ indptr,
                                                    const uint32_t* __restrict__ indices,
                                                    const float* __restrict__ vals, const float* __restrict__ da,
                                                    const __nv_bfloat16* __restrict__ h,
                                                    __nv_bfloat16* __restrict__ dz) {
  const int lane = threadIdx.x & 31;
  const int64_t warps = static_cast<int64_t>(gridDim.x) * (kT / 32);
  for (int64_t i = blockIdx.x * static_cast<int64_t>(kT / 32) + (threadIdx.x >> 5); i < n; i += warps) {
    const uint64_t e0 = indptr[i], e1 = indptr[i + 1];
    float2 acc = *reinterpret_cast<const float2*>(da + i * kMpnnCat + 2 * lane);
    uint64_t e = e0;
    for (; e + 4 <= e1; e += 4) {
      uint32_t j[4];
      float w[4];
      float2 g[4];
#pragma unroll
      for (int u = 0; u < 4; ++u) {
        j[u] = __ldg(indices + e + u);
        w[u] = __ldg(vals + e + u);
      }
#pragma unroll
      for (int u = 0; u < 4; ++u)
        g[u] = *reinterpret_cast<const float2*>(da + static_cast<int64_t>(j[u]) * kMpnnCat + kMpnnHidden + 2 * lane);
#pragma unroll
      for (int u = 0; u < 4; ++u) {
        acc.x -= w[u] * g[u].x;
        acc.y -= w[u] * g[u].y;
      }
    }
    for (; e < e1; ++e) {
      const uint32_t j = __ldg(indices + e);
      const float w = __ldg(vals + e);
      const float2 g =
          *reinterpret_cast<const float2*>(da + static_cast<int64_t>(j) * kMpnnCat + kMpnnHidden + 2 * lane);
      acc.x -= w * g.x;
      acc.y -= w * g.y;
    }
    const float2 hv = __bfloat1622float2(*reinterpret_cast<const __nv_bfloat162*>(h + i * kMpnnCat + 2 * lane));
    const float gx = hv.x > 0.0f ? acc.x : 0.0f;
    const float gy = hv.y > 0.0f ? acc.y : 0.0f;
    *reinterpret_cast<__nv_bfloat162*>(dz + i * kMpnnHidden + 2 * lane) = __floats2bfloat162_rn(gx, gy);
  }
}

// ---- transpose [n x c] (pitch pin) -> [c x npad] (pitch npad), zero padded ----------
__global__ void k_transpose_bf16(int64_t n, int c, const __nv_bfloat16* __restrict__ in, int64_t pin,
                                 __nv_bfloat16* __restrict__ out, int64_t npad) {
  __shared__ __nv_bfloat16 tile[32][34];
  const int64_t r0 = static_cast<int64_t>(blockIdx.x) * 32;
  const int c0 = blockIdx.y * 32;
  for (int k = threadIdx.y; k < 32; k += blockDim.y) {
    const int64_t r = r0 + k;
    const int cc = c0 + threadIdx.x;
    tile[k][threadIdx.x] = (r < n && cc < c) ? in[r * pin + cc] : __float2bfloat16_rn(0.0f);
  }
  __syncthreads();
  for (int k = threadIdx.y; k < 32; k += blockDim.y) {
    const int cc = c0 + k;
    const int64_t r = r0 + threadIdx.x;
    if (cc < c && r < npad) out[static_cast<int64_t>(cc) * npad + r] = tile[threadIdx.x][k];
  }
}

// ---- row sums of a [rows x npad] bf16 matrix (bias gradients), one CTA per row ------
__global__ void k_row_sums(const __nv_bfloat16* __restrict__ m, int64_t npad, float* __restrict__ out) {
  __shared__ double red[kT / 32];
  const __nv_bfloat16* row = m + static_cast<int64_t>(blockIdx.x) * npad;
  double s = 0.0;
  for (int64_t i = threadIdx.x; i < npad; i += kT) s += __bfloat162float(row[i]);
  s = warp_sum(s);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = s;
  __syncthreads();
  if (threadIdx.x < 32) {
    double t = threadIdx.x < kT / 32 ? red[threadIdx.x] : 0.0;
    t = warp_sum(t);
    if (threadIdx.x == 0) out[blockIdx.x] = static_cast<float>(t);
  }
}

// ---- loss statistics: G = Y^T Y, C = V^T Y over the first k columns (f64) -----------
// partial layout: [entry][cta], entries = 2 k^2; the last CTA adds in CTA order.
__global__ void k_loss_stats(int64_t n, int k, const float* __restrict__ y, const double* __restrict__ v, int vld,
                             double* __restrict__ partial, unsigned* __restrict__ ticket, double* __restrict__ stats) {
  extern __shared__ double sh_stats[];  // [2 k^2] per warp
  __shared__ bool last;
  const int ne = 2 * k * k;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  double* mine = sh_stats + warp * ne;
  const int64_t wstride = static_cast<int64_t>(gridDim.x) * (blockDim.x >> 5);
  for (int e = lane; e < ne; e += 32) {
    const bool gpart = e < k * k;
    const int ee = gpart ? e : e - k * k;
    const int a = ee / k, b = ee % k;
    double s = 0.0;
    for (int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x >> 5) + warp; i < n; i += wstride) {
      const double yb = y[i * kMpnnOut + b];
      const double xa = gpart ? static_cast<double>(y[i * kMpnnOut + a]) : v[i * vld + a];
      s += xa * yb;
    }
    mine[e] = s;
  }
  __syncthreads();
  for (int e = threadIdx.x; e < ne; e += blockDim.x) {
    double s = 0.0;
    for (int w = 0; w < static_cast<int>(blockDim.x >> 5); ++w) s += sh_stats[w * ne + e];
    partial[static_cast<int64_t>(e) * gridDim.x + blockIdx.x] = s;
  }
  __threadfence();
  __syncthreads();
  if (threadIdx.x == 0) last = atomicAdd(ticket, 1u) == gridDim.x - 1;
  __syncthreads();
  if (!last) return;
  __threadfence();
  for (int e = threadIdx.x; e < ne; e += blockDim.x) {
    double s = 0.0;
    for (int b = 0; b < static_cast<int>(gridDim.x); ++b)
      s += __ldcg(&partial[static_cast<int64_t>(e) * gridDim.x + b]);
    stats[e] = s;
  }
  if (threadIdx.x == 0) *ticket = 0u;
}

// ---- small k x k algebra of the loss (one thread) ------------------------------------
// coef = [P1 = C G^-1 | P2 = G^-1 M G^-1] (row-major k x k each), out[0] = loss,
// out[1] = 1 when G was not positive definite.
__global__ void k_loss_small(int k, const double* __restrict__ stats, double* __restrict__ coef,
                             double* __restrict__ out) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  double G[kMpnnOut * kMpnnOut], Cm[kMpnnOut * kMpnnOut], L[kMpnnOut * kMpnnOut], Gi[kMpnnOut * kMpnnOut];
  for (int e = 0; e < k * k; ++e) {
    G[e] = stats[e];
    Cm[e] = stats[k * k + e];
  }
  // Cholesky G = L L^T with a tiny relative ridge
  double tr = 0.0;
  for (int a = 0; a < k; ++a) tr += G[a * k + a];
  const double ridge = 1e-12 * (tr > 0.0 ? tr : 1.0);
  bool bad = false;
  for (int j = 0; j < k; ++j) {
    double d = G[j * k + j] + ridge;
    for (int p = 0; p < j; ++p) d -= L[j * k + p] * L[j * k + p];
    if (!(d > 0.0)) {
      bad = true;
      d = ridge;
    }
    L[j * k + j] = sqrt(d);
    for (int i = j + 1; i < k; ++i) {
      double s = G[i * k + j];
      for (int p = 0; p < j; ++p) s -= L[i * k + p] * L[j * k + p];
      L[i * k + j] = s / L[j * k + j];
    }
    for (int i = 0; i < j; ++i) L[i * k + j] = 0.0;
  }
  // Gi = G^-1 column by column
  for (int c = 0; c < k; ++c) {
    double z[kMpnnOut];
    for (int i = 0; i < k; ++i) {
      double s = (i == c) ? 1.0 : 0.0;
      for (int p = 0; p < i; ++p) s -= L[i * k + p] * z[p];
      z[i] = s / L[i * k + i];
    }
    for (int i = k - 1; i >= 0; --i) {
      double s = z[i];
      for (int p = i + 1; p < k; ++p) s -= L[p * k + i] * Gi[p * k + c];
      Gi[i * k + c] = s / L[i * k + i];
    }
  }
  // M = C^T C ; P1 = C Gi ; T = Gi M ; P2 = T Gi ; f = tr(Gi M)
  double M[kMpnnOut * kMpnnOut], T[kMpnnOut * kMpnnOut];
  for (int a = 0; a < k; ++a)
    for (int b = 0; b < k; ++b) {
      double s = 0.0;
      for (int p = 0; p < k; ++p) s += Cm[p * k + a] * Cm[p * k + b];
      M[a * k + b] = s;
    }
  for (int a = 0; a < k; ++a)
    for (int b = 0; b < k; ++b) {
      double s1 = 0.0, s2 = 0.0;
      for (int p = 0; p < k; ++p) {
        s1 += Cm[a * k + p] * Gi[p * k + b];
        s2 += Gi[a * k + p] * M[p * k + b];
      }
      coef[a * k + b] = s1;
      T[a * k + b] = s2;
    }
  double f = 0.0;
  for (int a = 0; a < k; ++a) f += T[a * k + a];
  for (int a = 0; a < k; ++a)
    for (int b = 0; b < k; ++b) {
      double s = 0.0;
      for (int p = 0; p < k; ++p) s += T[a * k + p] * Gi[p * k + b];
      coef[k * k + a * k + b] = s;
    }
  out[0] = 1.0 - f / k;
  out[1] = bad ? 1.0 : 0.0;
}

// dY[i, c] = -(2/k) (sum_a V[i,a] P1[a,c] - sum_a Y[i,a] P2[a,c]) for c < k, 0 beyond.
__global__ void k_loss_grad(int64_t n, int k, const float* __restrict__ y, const double* __restrict__ v, int vld,
                            const double* __restrict__ coef, __nv_bfloat16* __restrict__ dy) {
  __shared__ double P[2 * kMpnnOut * kMpnnOut];
  for (int e = threadIdx.x; e < 2 * k * k; e += blockDim.x) P[e] = coef[e];
  __syncthreads();
  const double sc = -2.0 / k;
  const int64_t total = n * kMpnnOut;
  const int64_t stride = static_cast<int64_t>(gridDim.x) * blockDim.x;
  for (int64_t e = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; e < total; e += stride) {
    const int64_t i = e / kMpnnOut;
    const int c = static_cast<int>(e % kMpnnOut);
    double g = 0.0;
    if (c < k) {
      for (int a = 0; a < k; ++a)
        g += v[i * vld + a] * P[a * k + c] - static_cast<double>(y[i * kMpnnOut + a]) * P[k * k + a * k + c];
      g *= sc;
    }
    dy[e] = __float2bfloat16_rn(static_cast<float>(g));
  }
}

// ---- parameters -------------------------------------------------------------------------
// flat layout: for l in 0..2: Wt_l [64 x 128], b_l [64]; then Wt_out [16 x 128], b_out [16]
__host__ __device__ constexpr int64_t off_wt(int l) {
  return static_cast<int64_t>(l) * (kMpnnHidden * kMpnnCat + kMpnnHidden);
}
__host__ __device__ constexpr int64_t off_b(int l) { return off_wt(l) + kMpnnHidden * kMpnnCat; }
__host__ __device__ constexpr int64_t off_wt_out() { return off_wt(kMpnnLayers); }
__host__ __device__ constexpr int64_t off_b_out() { return off_wt_out() + kMpnnOut * kMpnnCat; }

// bf16 copies: wt (forward operand, [N x 128] per layer) and w (backward operand,
// [128 x N] per layer: the transpose).
__global__ void k_params_to_bf16(const float* __restrict__ p, __nv_bfloat16* __restrict__ wt,
                                 __nv_bfloat16* __restrict__ w) {
  const int64_t per = kMpnnHidden * kMpnnCat;
  const int64_t total = kMpnnLayers * per + kMpnnOut * kMpnnCat;
  const int64_t stride = static_cast<int64_t>(gridDim.x) * blockDim.x;
  for (int64_t e = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; e < total; e += stride) {
    int l, N;
    int64_t r, src;
    if (e < kMpnnLayers * per) {
      l = static_cast<int>(e / per);
      r = e % per;
      N = kMpnnHidden;
      src = off_wt(l) + r;
    } else {
      l = kMpnnLayers;
      r = e - kMpnnLayers * per;
      N = kMpnnOut;
      src = off_wt_out() + r;
    }
    const int j = static_cast<int>(r / kMpnnCat);  // output unit
    const int i = static_cast<int>(r % kMpnnCat);  // input feature
    const __nv_bfloat16 b = __float2bfloat16_rn(p[src]);
    const int64_t base = static_cast<int64_t>(l) * per;
    wt[base + r] = b;
    w[base + static_cast<int64_t>(i) * N + j] = b;
  }
}

// gradient assembly: gw_l [128 x N] (W layout, from the GEMM) -> flat Wt layout
__global__ void k_assemble_grad(const float* __restrict__ gw, const float* __restrict__ gb, int l, int N,
                                float* __restrict__ grad) {
  const int total = N * kMpnnCat + N;
  const int64_t wo = l < kMpnnLayers ? off_wt(l) : off_wt_out();
  const int64_t bo = l < kMpnnLayers ? off_b(l) : off_b_out();
  for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < total; e += gridDim.x * blockDim.x) {
    if (e < N * kMpnnCat) {
      const int j = e / kMpnnCat, i = e % kMpnnCat;
      grad[wo + e] = gw[static_cast<int64_t>(i) * N + j];
    } else {
      grad[bo + (e - N * kMpnnCat)] = gb[e - N * kMpnnCat];
    }
  }
}

__global__ void k_adam(int64_t count, float* __restrict__ p, const float* __restrict__ g, float* __restrict__ m,
                       float* __restrict__ v, float lr, float b1, float b2, float eps, float c1, float c2) {
  const int64_t stride = static_cast<int64_t>(gridDim.x) * blockDim.x;
  for (int64_t e = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; e < count; e += stride) {
    const float gg = g[e];
    const float mm = b1 * m[e] + (1.0f - b1) * gg;
    const float vv = b2 * v[e] + (1.0f - b2) * gg * gg;
    m[e] = mm;
    v[e] = vv;
    p[e] -= lr * (mm / c1) / (sqrtf(vv / c2) + eps);
  }
}

__global__ void k_init_params(int64_t count, float* __restrict__ p, uint64_t seed) {
  const int64_t stride = static_cast<int64_t>(gridDim.x) * blockDim.x;
  for (int64_t e = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; e < count; e += stride) {
    bool bias = false;
    for (int l = 0; l <= kMpnnLayers; ++l) {
      const int64_t bo = l < kMpnnLayers ? off_b(l) : off_b_out();
      const int N = l < kMpnnLayers ? kMpnnHidden : kMpnnOut;
      if (e >= bo && e < bo + N) bias = true;
    }
    if (bias) {
      p[e] = 0.0f;
    } else {
      double z0, z1;
      philox_normal2(seed, 0x6d706e6eull, static_cast<uint64_t>(e), z0, z1);
      p[e] = static_cast<float>(z0) * sqrtf(2.0f / kMpnnCat);  // He initialisation over the 128 inputs
    }
  }
}

// Chebyshev filter T_8 of (L - c)/e on x (f32 [n x 4]): the solver's start filter.
void cheb_filter(const Exec& ex, const OpDev& op, float* x, float* b0, float* b1, float* b2, int64_t n) {
  const double a = 0.1, b = 2.0;
  const double c = (a + b) / 2.0, e = (b - a) / 2.0;
  const double scale = 2.0 / e, shift = scale * c;
  Epilogue<float> ep1;
  ep1.alpha = 1.0 / e;
  ep1.beta = -c / e;
  ep1.z1 = x;
  spmm_dev<float>(ex, op, x, b0, 4, 4, ep1, nullptr, true);
  float* bufs[3] = {b0, b1, b2};
  const float* yprev = x;
  float* y = b0;
  int nxt = 1;
  for (int d = 2; d <= 8; ++d) {
    float* out = bufs[nxt];
    Epilogue<float> ep;
    ep.alpha = scale;
    ep.beta = -shift;
    ep.z1 = y;
    ep.gamma = -1.0;
    ep.z2 = yprev;
    spmm_dev<float>(ex, op, y, out, 4, 4, ep, nullptr, true);
    yprev = y;
    y = out;
    nxt = (nxt + 1) % 3;
  }
  SI_CUDA(cudaMemcpyAsync(x, y, sizeof(float) * n * 4, cudaMemcpyDeviceToDevice, ex.stream));
}

}  // namespace

// ---------------------------------------------------------------------------------------------
int64_t mpnn_param_count() { return off_b_out() + kMpnnOut; }

void MpnnModel::init(const Exec& ex, uint64_t seed) {
  const int64_t P = mpnn_param_count();
  params.alloc(P, ex.stream);
  grad.alloc(P, ex.stream);
  m1.alloc(P, ex.stream);
  m2.alloc(P, ex.stream);
  grad.zero();
  m1.zero();
  m2.zero();
  wt.alloc(kMpnnLayers * kMpnnHidden * kMpnnCat + kMpnnOut * kMpnnCat, ex.stream);
  w.alloc(wt.size(), ex.stream);
  k_init_params<<<grid_for_rows(ex, P), kT, 0, ex.stream>>>(P, params.get(), seed);
  SI_LAUNCH_CHECK();
  step = 0;
  sync_weights(ex);
}

void MpnnModel::sync_weights(const Exec& ex) {
  k_params_to_bf16<<<grid_for_rows(ex, static_cast<int64_t>(wt.size())), kT, 0, ex.stream>>>(params.get(), wt.get(),
                                                                                               w.get());
  SI_LAUNCH_CHECK();
}

void MpnnModel::set(const Exec& ex, const float* host) {
  SI_CUDA(cudaMemcpyAsync(params.get(), host, sizeof(float) * params.size(), cudaMemcpyHostToDevice, ex.stream));
  m1.zero();
  m2.zero();
  step = 0;
  sync_weights(ex);
  SI_CUDA(cudaStreamSynchronize(ex.stream));
}

void MpnnModel::get(const Exec& ex, float* host) const {
  SI_CUDA(cudaMemcpyAsync(host, params.get(), sizeof(float) * params.size(), cudaMemcpyDeviceToHost, ex.stream));
  SI_CUDA(cudaStreamSynchronize(ex.stream));
}

void MpnnActs::ensure(const Exec& ex, int64_t n_) {
  if (n == n_ && y.size() > 0) return;
  n = n_;
  npad = (n + 7) / 8 * 8;
  for (int l = 0; l <= kMpnnLayers; ++l) a[l].alloc(static_cast<size_t>(n) * kMpnnCat, ex.stream);
  y.alloc(static_cast<size_t>(n) * kMpnnOut, ex.stream);
}

void mpnn_features(const Exec& ex, const OpDev& op, const double* sqrt_deg, uint64_t seed, const float* given,
                   MpnnActs& acts) {
  const int64_t n = op.n;
  acts.ensure(ex, n);
  DevBuf<float> probes, b0, b1, b2;
  DevBuf<double> pscale(4, ex.stream);
  double s_scale = 1.0;
  if (given == nullptr) {
    SI_REQUIRE(sqrt_deg != nullptr && op.v32 != nullptr, SI_INVALID_ARGUMENT,
               "warm start: features need sqrt_deg and f32 operator values");
    probes.alloc(static_cast<size_t>(n) * 4, ex.stream);
    b0.alloc(probes.size(), ex.stream);
    b1.alloc(probes.size(), ex.stream);
    b2.alloc(probes.size(), ex.stream);
    fill_normal_dev<float>(ex, probes.get(), n, 4, 4, seed, 7);
    cheb_filter(ex, op, probes.get(), b0.get(), b1.get(), b2.get(), n);
    GramWork gw;
    DevBuf<double> norms(4, ex.stream), dn(1, ex.stream);
    column_residual_norms_dev<float>(ex, gw, probes.get(), nullptr, nullptr, 4, 4, n, norms.get());
    column_residual_norms_dev<double>(ex, gw, sqrt_deg, nullptr, nullptr, 1, 1, n, dn.get());
    double hn[5];
    SI_CUDA(cudaMemcpyAsync(hn, norms.get(), sizeof(double) * 4, cudaMemcpyDeviceToHost, ex.stream));
    SI_CUDA(cudaMemcpyAsync(hn + 4, dn.get(), sizeof(double), cudaMemcpyDeviceToHost, ex.stream));
    SI_CUDA(cudaStreamSynchronize(ex.stream));
    const double rn = std::sqrt(static_cast<double>(n));
    double ps[4];
    for (int j = 0; j < 4; ++j) ps[j] = hn[j] > 0.0 ? rn / hn[j] : 0.0;
    s_scale = hn[4] > 0.0 ? rn / hn[4] : 0.0;
    SI_CUDA(cudaMemcpyAsync(pscale.get(), ps, sizeof(ps), cudaMemcpyHostToDevice, ex.stream));
  }
  k_features<<<grid_for_rows(ex, n * kMpnnHidden), kT, 0, ex.stream>>>(n, sqrt_deg, s_scale, probes.get(), 4,
                                                                      pscale.get(), given, acts.a[0].get());
  SI_LAUNCH_CHECK();
  SI_CUDA(cudaStreamSynchronize(ex.stream));
}

void mpnn_forward(const Exec& ex, const MpnnModel& model, const OpDev& op, MpnnActs& acts, GemmWorkspace& ws) {
  const int64_t n = op.n;
  const int gmp = grid_for_rows(ex, n * 32, 16);
  for (int l = 0; l <= kMpnnLayers; ++l) {
    k_mp_forward<<<gmp, kT, 0, ex.stream>>>(n, op.indptr, op.indices, op.v32, acts.a[l].get());
    SI_LAUNCH_CHECK();
    GemmEpilogue ep;
    if (l < kMpnnLayers) {
      ep.mode = GEMM_BIAS_RELU_BF16;
      ep.out_bf16 = acts.a[l + 1].get();
      ep.ldo = kMpnnCat;
      ep.bias = model.params.get() + off_b(l);
      gemm_bf16_nt(ex, n, kMpnnHidden, kMpnnCat, acts.a[l].get(), kMpnnCat,
                   model.wt.get() + static_cast<int64_t>(l) * kMpnnHidden * kMpnnCat, kMpnnCat, ep, 1, ws);
    } else {
      ep.mode = GEMM_BIAS_F32;
      ep.out_f32 = acts.y.get();
      ep.ldo = kMpnnOut;
      ep.bias = model.params.get() + off_b_out();
      gemm_bf16_nt(ex, n, kMpnnOut, kMpnnCat, acts.a[l].get(), kMpnnCat,
                   model.wt.get() + static_cast<int64_t>(kMpnnLayers) * kMpnnHidden * kMpnnCat, kMpnnCat, ep, 1,
                   ws);
    }
  }
}

double mpnn_loss_backward(const Exec& ex, MpnnModel& model, const OpDev& op, MpnnActs& acts, const double* target,
                          int vld, int k, GemmWorkspace& ws) {
  const int64_t n = op.n;
  const int64_t npad = acts.npad;
  SI_REQUIRE(k >= 1 && k <= kMpnnOut, SI_INVALID_ARGUMENT, "warm start: k must be in [1, 16]");
  // ---- loss and dL/dY
  const int ne = 2 * k * k;
  const int sgrid = std::max(1, std::min(ex.sms * 2, static_cast<int>((n + 255) / 256)));
  DevBuf<double> partial(static_cast<size_t>(ne) * sgrid, ex.stream), stats(ne, ex.stream),
      coef(2 * k * k, ex.stream), lout(2, ex.stream);
  DevBuf<unsigned> ticket(1, ex.stream);
  ticket.zero();
  const int sthreads = 256;
  k_loss_stats<<<sgrid, sthreads, sizeof(double) * ne * (sthreads / 32), ex.stream>>>(
      n, k, acts.y.get(), target, vld, partial.get(), ticket.get(), stats.get());
  SI_LAUNCH_CHECK();
  k_loss_small<<<1, 32, 0, ex.stream>>>(k, stats.get(), coef.get(), lout.get());
  SI_LAUNCH_CHECK();
  DevBuf<__nv_bfloat16> dy(static_cast<size_t>(n) * kMpnnOut, ex.stream),
      dyt(static_cast<size_t>(kMpnnOut) * npad, ex.stream);
  k_loss_grad<<<grid_for_rows(ex, n * kMpnnOut), kT, 0, ex.stream>>>(n, k, acts.y.get(), target, vld, coef.get(),
                                                                    dy.get());
  SI_LAUNCH_CHECK();

  DevBuf<__nv_bfloat16> at(static_cast<size_t>(kMpnnCat) * npad, ex.stream);
  DevBuf<float> da(static_cast<size_t>(n) * kMpnnCat, ex.stream), gw(kMpnnCat * kMpnnHidden, ex.stream),
      gb(kMpnnHidden, ex.stream);
  DevBuf<__nv_bfloat16> dz(static_cast<size_t>(n) * kMpnnHidden, ex.stream),
      dzt(static_cast<size_t>(kMpnnHidden) * npad, ex.stream);
  const dim3 tblk(32, 8);
  auto transpose = [&](const __nv_bfloat16* in, int c, int64_t pin, __nv_bfloat16* out) {
    const dim3 grid(static_cast<unsigned>((npad + 31) / 32), static_cast<unsigned>((c + 31) / 32));
    k_transpose_bf16<<<grid, tblk, 0, ex.stream>>>(n, c, in, pin, out, npad);
    SI_LAUNCH_CHECK();
  };
  // weight gradients reduce over all n rows: split K so every SM gets a slice of at least 1024 rows
  const int ksplit = static_cast<int>(std::max<int64_t>(1, std::min<int64_t>(ex.sms, (npad + 1023) / 1024)));

  // ---- output layer: dW_out = A_3^T dY, db_out = colsum(dY), dA_3 = dY W_out^T
  transpose(dy.get(), kMpnnOut, kMpnnOut, dyt.get());
  transpose(acts.a[kMpnnLayers].get(), kMpnnCat, kMpnnCat, at.get());
  {
    GemmEpilogue ep;
    ep.mode = GEMM_STORE_F32;
    ep.out_f32 = gw.get();
    ep.ldo = kMpnnOut;
    gemm_bf16_nt(ex, kMpnnCat, kMpnnOut, npad, at.get(), npad, dyt.get(), npad, ep, ksplit, ws);
    k_row_sums<<<kMpnnOut, kT, 0, ex.stream>>>(dyt.get(), npad, gb.get());
    SI_LAUNCH_CHECK();
    k_assemble_grad<<<16, kT, 0, ex.stream>>>(gw.get(), gb.get(), kMpnnLayers, kMpnnOut, model.grad.get());
    SI_LAUNCH_CHECK();
    GemmEpilogue ed;
    ed.mode = GEMM_STORE_F32;
    ed.out_f32 = da.get();
    ed.ldo = kMpnnCat;
    gemm_bf16_nt(ex, n, kMpnnCat, kMpnnOut, dy.get(), kMpnnOut,
                 model.w.get() + static_cast<int64_t>(kMpnnLayers) * kMpnnHidden * kMpnnCat, kMpnnOut, ed, 1, ws);
  }
  const int gmp = grid_for_rows(ex, n * 32, 16);
  for (int l = kMpnnLayers - 1; l >= 0; --l) {
    // dZ_l from dA_{l+1} through the message passing and the ReLU of H_{l+1}
    k_mp_backward<<<gmp, kT, 0, ex.stream>>>(n, op.indptr, op.indices, op.v32, da.get(), acts.a[l + 1].get(),
                                             dz.get());
    SI_LAUNCH_CHECK();
    transpose(dz.get(), kMpnnHidden, kMpnnHidden, dzt.get());
    transpose(acts.a[l].get(), kMpnnCat, kMpnnCat, at.get());
    GemmEpilogue ep;
    ep.mode = GEMM_STORE_F32;
    ep.out_f32 = gw.get();
    ep.ldo = kMpnnHidden;
    gemm_bf16_nt(ex, kMpnnCat, kMpnnHidden, npad, at.get(), npad, dzt.get(), npad, ep, ksplit, ws);
    k_row_sums<<<kMpnnHidden, kT, 0, ex.stream>>>(dzt.get(), npad, gb.get());
    SI_LAUNCH_CHECK();
    k_assemble_grad<<<32, kT, 0, ex.stream>>>(gw.get(), gb.get(), l, kMpnnHidden, model.grad.get());
    SI_LAUNCH_CHECK();
    if (l > 0) {
      GemmEpilogue ed;
      ed.mode = GEMM_STORE_F32;
      ed.out_f32 = da.get();
      ed.ldo = kMpnnCat;
      gemm_bf16_nt(ex, n, kMpnnCat, kMpnnHidden, dz.get(), kMpnnHidden,
                   model.w.get() + static_cast<int64_t>(l) * kMpnnHidden * kMpnnCat, kMpnnHidden, ed, 1, ws);
    }
  }
  double h[2];
  SI_CUDA(cudaMemcpyAsync(h, lout.get(), sizeof(h), cudaMemcpyDeviceToHost, ex.stream));
  gemm_check(ex, ws);  // synchronises
  SI_REQUIRE(h[1] == 0.0, SI_CONVERGENCE_FAILURE, "warm start: predicted block is rank deficient");
  return h[0];
}

void mpnn_adam(const Exec& ex, MpnnModel& model, float lr) {
  ++model.step;
  const float b1 = 0.9f, b2 = 0.999f;
  const float c1 = 1.0f - std::pow(b1, static_cast<float>(model.step));
  const float c2 = 1.0f - std::pow(b2, static_cast<float>(model.step));
  const int64_t P = mpnn_param_count();
  k_adam<<<grid_for_rows(ex, P), kT, 0, ex.stream>>>(P, model.params.get(), model.grad.get(), model.m1.get(),
                                                      model.m2.get(), lr, b1, b2, 1e-8f, c1, c2);
  SI_LAUNCH_CHECK();
  model.sync_weights(ex);
}

}  // namespace si
