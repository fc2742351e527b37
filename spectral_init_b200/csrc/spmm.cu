// CSR SpMM over row-major blocks of vectors: the LinearOperator::apply of the
// crate (src/operator.rs:176-223) re-designed for sm_100a.
//
// Layout: the operator is CSR (u64 indptr, u32 indices, f64 or f32 values)
// with an optional implicit diagonal coefficient; x and y are row-major
// [n x ld] blocks, ld in {4, 8, 16} for the vectorised kernels.
//
// Mapping: G lanes (4..32, chosen from the mean row length) own one row.
// Each lane walks the row's entries with stride G, so the index/value
// streams are read coalesced and with the evict-first L2 policy (they are
// touched once per SpMM), while the gathered x rows are 32-byte (f64, ld=4)
// or 16/32-byte (f32) vector loads that stay cached.  The per-lane partial
// sums are combined by a transposing butterfly: at every step a lane keeps
// half of its columns and trades the other half, so ld columns cost ld
// shuffles instead of ld*log2(G), and each lane ends owning distinct output
// columns that it finishes with the fused epilogue
//   y = alpha * (diag * x_i + sum_j v_ij x_j) + beta z1 + gamma z2 + delta z3.
// Accumulation is always f64 (also for f32 data).
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdio>
#include <cstdlib>
#include <string>
#include <atomic>
#include <map>
#include <mutex>
#include <tuple>
#include <type_traits>
#include <vector>

#include "si_internal.h"
#include "umma.cuh"
#include "umma_gemm.h"

namespace si {
namespace {

template <class T>
__device__ __forceinline__ T ld_stream(const T* p) {
  return __ldcs(p);
}

// Vector gather of one x row of LD elements into f64 registers.  The 4-wide
// rows bypass L1 (.cg): the rows a warp gathers are scattered over the block,
// so an L1 allocation is rarely reused and costs L1 fill bandwidth.
template <class XT, int LD>
struct RowLoad;

template <int LD>
struct RowLoad<double, LD> {
  __device__ __forceinline__ static void run(const double* p, double (&v)[LD]) {
#pragma unroll
    for (int q = 0; q < LD / 4; ++q) {
      double a, b, c, d;
      asm volatile("ld.global.cg.v4.f64 {%0,%1,%2,%3}, [%4];"
                   : "=d"(a), "=d"(b), "=d"(c), "=d"(d)
                   : "l"(p + 4 * q));
      v[4 * q + 0] = a;
      v[4 * q + 1] = b;
      v[4 * q + 2] = c;
      v[4 * q + 3] = d;
    }
  }
};

template <>
struct RowLoad<float, 4> {
  __device__ __forceinline__ static void run(const float* p, double (&v)[4]) {
    float4 t = __ldcg(reinterpret_cast<const float4*>(p));
    v[0] = t.x;
    v[1] = t.y;
    v[2] = t.z;
    v[3] = t.w;
  }
};

template <int LD>
struct RowLoadF32x8 {
  __device__ __forceinline__ static void run(const float* p, double (&v)[LD]) {
#pragma unroll
    for (int q = 0; q < LD / 8; ++q) {
      float a[8];
      asm volatile("ld.global.nc.v8.f32 {%0,%1,%2,%3,%4,%5,%6,%7}, [%8];"
                   : "=f"(a[0]), "=f"(a[1]), "=f"(a[2]), "=f"(a[3]), "=f"(a[4]), "=f"(a[5]), "=f"(a[6]),
                     "=f"(a[7])
                   : "l"(p + 8 * q));
#pragma unroll
      for (int t = 0; t < 8; ++t) v[8 * q + t] = a[t];
    }
  }
};
template <>
struct RowLoad<float, 8> : RowLoadF32x8<8> {};
template <>
struct RowLoad<float, 16> : RowLoadF32x8<16> {};

// Transposing butterfly over a group of G lanes.  On return the lane holds
// W = max(LD/G, 1) column sums starting at the returned base column.
template <int LD, int G>
struct GroupReduce {
  static constexpr int W = (LD >= G) ? LD / G : 1;
  // first output column owned by lane `sub` after run()
  __device__ __forceinline__ static int base_of(int sub) {
    int base = 0;
    int width = LD;
#pragma unroll
    for (int o = G / 2; o >= 1; o >>= 1) {
      if (width > W) {
        if (sub & o) base += width / 2;
        width /= 2;
      }
    }
    return base;
  }
  __device__ __forceinline__ static int run(double (&v)[LD], int sub, unsigned mask) {
    int base = 0;
    int width = LD;
#pragma unroll
    for (int o = G / 2; o >= 1; o >>= 1) {
      if (width > W) {
        const int h = width / 2;
        const bool upper = (sub & o) != 0;
#pragma unroll
        for (int c = 0; c < LD / 2; ++c) {
          if (c < h) {
            const double send = upper ? v[c] : v[c + h];
            const double keep = upper ? v[c + h] : v[c];
            v[c] = keep + __shfl_xor_sync(mask, send, o, G);
          }
        }
        if (upper) base += h;
        width = h;
      } else {
#pragma unroll
        for (int c = 0; c < W; ++c) v[c] += __shfl_xor_sync(mask, v[c], o, G);
      }
    }
    return base;
  }
};

// Where a row's index/value streams are read from.
template <class VT>
struct GlobalStream {
  const uint32_t* idx;
  const VT* val;
  __device__ __forceinline__ uint32_t j(uint64_t k) const { return ld_stream(idx + k); }
  __device__ __forceinline__ double v(uint64_t k) const { return static_cast<double>(ld_stream(val + k)); }
};
template <class VT>
struct SharedStream {  // entries [base, base + count) staged in shared memory
  const uint32_t* idx;
  const VT* val;
  uint64_t base;
  __device__ __forceinline__ uint32_t j(uint64_t k) const { return idx[k - base]; }
  __device__ __forceinline__ double v(uint64_t k) const { return static_cast<double>(val[k - base]); }
};

// One row of y = epilogue(A x) by a group of G lanes.  U entries per lane per
// pass: all index/value reads of a pass are issued before its gathers.  The
// own-row epilogue terms are loaded first so they overlap the gathers.
template <class VT, class XT, int LD, int G, class Src>
__device__ __forceinline__ void spmm_row(int64_t row, uint64_t s, uint64_t e, const Src& src, double diag,
                                         const XT* __restrict__ x, XT* __restrict__ y, const Epilogue<XT>& ep,
                                         int sub, unsigned mask, bool writer) {
  constexpr int W = GroupReduce<LD, G>::W;
  constexpr int U = (LD >= 16) ? 4 : 8;
  const int obase = GroupReduce<LD, G>::base_of(sub);
  double own[W], addz[W];
#pragma unroll
  for (int c = 0; c < W; ++c) {
    own[c] = 0.0;
    addz[c] = 0.0;
    if (writer) {
      const int64_t off = row * LD + obase + c;
      own[c] = diag * static_cast<double>(x[off]);
      if (ep.z1) addz[c] = ep.beta * static_cast<double>(ep.z1[off]);
      if (ep.z2) addz[c] = fma(ep.gamma, static_cast<double>(ep.z2[off]), addz[c]);
      if (ep.z3) addz[c] = fma(ep.delta, static_cast<double>(ep.z3[off]), addz[c]);
    }
  }
  double acc[LD];
#pragma unroll
  for (int c = 0; c < LD; ++c) acc[c] = 0.0;
  for (uint64_t b0 = s + sub; b0 < e; b0 += static_cast<uint64_t>(G) * U) {
    uint32_t jj[U];
    double vv[U];
#pragma unroll
    for (int u = 0; u < U; ++u) {
      const uint64_t k = b0 + static_cast<uint64_t>(u) * G;
      const bool ok = k < e;
      jj[u] = ok ? src.j(k) : 0u;
      vv[u] = ok ? src.v(k) : 0.0;
    }
#pragma unroll
    for (int u = 0; u < U; ++u) {
      if (b0 + static_cast<uint64_t>(u) * G < e) {
        double xr[LD];
        RowLoad<XT, LD>::run(x + static_cast<int64_t>(jj[u]) * LD, xr);
#pragma unroll
        for (int c = 0; c < LD; ++c) acc[c] = fma(vv[u], xr[c], acc[c]);
      }
    }
  }
  const int base = GroupReduce<LD, G>::run(acc, sub, mask);
  if (writer) {
#pragma unroll
    for (int c = 0; c < W; ++c) {
      const int64_t off = row * LD + base + c;
      y[off] = static_cast<XT>(fma(ep.alpha, own[c] + acc[c], addz[c]));
    }
  }
}

template <int G>
__device__ __forceinline__ unsigned group_mask(int lane) {
  return (G == 32) ? 0xffffffffu : (((1u << G) - 1u) << (lane & ~(G - 1)));
}

template <int LD, int G>
__device__ __forceinline__ bool group_writer(int sub) {
  return (LD >= G) || ((sub & ((G / (LD < G ? LD : G)) - 1)) == 0);
}

// Direct kernel: rows in grid-stride order, streams read from global memory;
// the next row's bounds are fetched while the current row is in flight.
template <class VT, class XT, int LD, int G>
__global__ void __launch_bounds__(256) k_spmm_vec(int64_t n, const uint64_t* __restrict__ indptr,
                                                  const uint32_t* __restrict__ indices,
                                                  const VT* __restrict__ vals, double diag,
                                                  const XT* __restrict__ x, XT* __restrict__ y,
                                                  Epilogue<XT> ep, const int* __restrict__ stop) {
  if (stop != nullptr && *stop != 0) return;
  const int lane = threadIdx.x & 31;
  const int sub = lane & (G - 1);
  const unsigned mask = group_mask<G>(lane);
  const bool writer = group_writer<LD, G>(sub);
  const int64_t group = (static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x) / G;
  const int64_t ngroups = static_cast<int64_t>(gridDim.x) * blockDim.x / G;
  const GlobalStream<VT> src{indices, vals};
  int64_t row = group;
  uint64_t s = 0, e = 0;
  if (row < n) {
    s = __ldg(indptr + row);
    e = __ldg(indptr + row + 1);
  }
  for (; row < n; row += ngroups) {
    const int64_t nrow = row + ngroups;
    uint64_t ns = 0, ne = 0;
    if (nrow < n) {
      ns = __ldg(indptr + nrow);
      ne = __ldg(indptr + nrow + 1);
    }
    spmm_row<VT, XT, LD, G>(row, s, e, src, diag, x, y, ep, sub, mask, writer);
    s = ns;
    e = ne;
  }
}

// Tiled kernel: persistent CTAs walk row blocks of ~kSpmmBlockNnz entries.
// A block's row pointers, column indices and values are staged into shared
// memory with cp.async (every warp request a full contiguous 128-byte line)
// while the previous block is computed from shared memory, so the only global
// loads of the compute phase are the x-row gathers (L2 resident).  Blocks
// that do not fit (a row longer than the staging capacity) are computed
// straight from global memory.
__device__ __forceinline__ void cp_async_4(void* smem, const void* gmem) {
  const unsigned s = static_cast<unsigned>(__cvta_generic_to_shared(smem));
  asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"(s), "l"(gmem));
}
__device__ __forceinline__ void cp_async_8(void* smem, const void* gmem) {
  const unsigned s = static_cast<unsigned>(__cvta_generic_to_shared(smem));
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(s), "l"(gmem));
}
__device__ __forceinline__ void cp_async_commit_grp() { asm volatile("cp.async.commit_group;\n" ::); }
template <int N>
__device__ __forceinline__ void cp_async_wait_grp() {
  asm volatile("cp.async.wait_group %0;\n" ::"n"(N));
}

template <class VT>
struct TileSmem {
  uint32_t idx[2][kSpmmBlockCap];
  VT val[2][kSpmmBlockCap];
  uint64_t ptr[2][kSpmmBlockRows + 1];
};

struct BlockInfo {
  int64_t r0 = 0, r1 = 0;
  uint64_t p0 = 0, p1 = 0;
  __device__ bool fits() const {
    return (r1 - r0) <= kSpmmBlockRows && (p1 - p0) <= static_cast<uint64_t>(kSpmmBlockCap);
  }
};

template <class VT, class XT, int LD, int G>
__global__ void __launch_bounds__(256) k_spmm_tiled(int64_t n, const uint64_t* __restrict__ indptr,
                                                    const uint32_t* __restrict__ indices,
                                                    const VT* __restrict__ vals, const int64_t* __restrict__ rblk,
                                                    const uint64_t* __restrict__ bptr, int64_t nblk, double diag,
                                                    const XT* __restrict__ x, XT* __restrict__ y, Epilogue<XT> ep,
                                                    const int* __restrict__ stop) {
  if (stop != nullptr && *stop != 0) return;
  extern __shared__ __align__(16) unsigned char tile_raw[];
  TileSmem<VT>& sm = *reinterpret_cast<TileSmem<VT>*>(tile_raw);
  const int lane = threadIdx.x & 31;
  const int sub = lane & (G - 1);
  const unsigned mask = group_mask<G>(lane);
  const bool writer = group_writer<LD, G>(sub);
  const int group = threadIdx.x / G;
  constexpr int NG = 256 / G;

  // block bounds: four independent loads (row range and its entry range)
  auto info = [&](int64_t b) {
    BlockInfo bi;
    if (b < nblk) {
      bi.r0 = rblk[b];
      bi.r1 = rblk[b + 1];
      bi.p0 = bptr[b];
      bi.p1 = bptr[b + 1];
    }
    return bi;
  };
  auto stage = [&](const BlockInfo& bi, int buf) {
    const int ne = static_cast<int>(bi.p1 - bi.p0);
    const int nr = static_cast<int>(bi.r1 - bi.r0);
    for (int t = threadIdx.x; t < ne; t += 256) {
      cp_async_4(&sm.idx[buf][t], indices + bi.p0 + t);
      if constexpr (sizeof(VT) == 8) cp_async_8(&sm.val[buf][t], vals + bi.p0 + t);
      else cp_async_4(&sm.val[buf][t], vals + bi.p0 + t);
    }
    for (int t = threadIdx.x; t <= nr; t += 256) cp_async_8(&sm.ptr[buf][t], indptr + bi.r0 + t);
  };

  int64_t b = blockIdx.x;
  const int64_t step = gridDim.x;
  int buf = 0;
  BlockInfo cur = info(b);
  if (b < nblk && cur.fits()) stage(cur, 0);
  cp_async_commit_grp();
  BlockInfo nxt = info(b + step);
  for (; b < nblk; b += step) {
    if (b + step < nblk && nxt.fits()) stage(nxt, buf ^ 1);
    cp_async_commit_grp();
    const BlockInfo after = info(b + 2 * step);  // in flight during this block's compute
    cp_async_wait_grp<1>();
    __syncthreads();
    if (cur.fits()) {
      const int nr = static_cast<int>(cur.r1 - cur.r0);
      const SharedStream<VT> src{sm.idx[buf], sm.val[buf], cur.p0};
      for (int rr = group; rr < nr; rr += NG)
        spmm_row<VT, XT, LD, G>(cur.r0 + rr, sm.ptr[buf][rr], sm.ptr[buf][rr + 1], src, diag, x, y, ep, sub, mask,
                                writer);
    } else {
      const GlobalStream<VT> src{indices, vals};
      for (int64_t rr = group; rr < cur.r1 - cur.r0; rr += NG)
        spmm_row<VT, XT, LD, G>(cur.r0 + rr, indptr[cur.r0 + rr], indptr[cur.r0 + rr + 1], src, diag, x, y, ep, sub,
                                mask, writer);
    }
    __syncthreads();
    buf ^= 1;
    cur = nxt;
    nxt = after;
  }
  cp_async_wait_grp<0>();
}

__global__ void k_block_ptrs(int64_t nblk, const int64_t* __restrict__ rblk, const uint64_t* __restrict__ indptr,
                             uint64_t* __restrict__ out) {
  const int64_t stride = static_cast<int64_t>(gridDim.x) * blockDim.x;
  for (int64_t b = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; b <= nblk; b += stride)
    out[b] = indptr[rblk[b]];
}

// row_blocks[b] = first row whose start offset is >= b * per
__global__ void k_row_blocks(int64_t n, const uint64_t* __restrict__ indptr, int64_t nblk, int64_t per,
                             int64_t* out) {
  const int64_t stride = static_cast<int64_t>(gridDim.x) * blockDim.x;
  for (int64_t b = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; b <= nblk; b += stride) {
    if (b == nblk) {
      out[b] = n;
      continue;
    }
    const uint64_t target = static_cast<uint64_t>(b) * static_cast<uint64_t>(per);
    int64_t lo = 0, hi = n;  // first r in [0, n] with indptr[r] >= target
    while (lo < hi) {
      const int64_t mid = lo + (hi - lo) / 2;
      if (indptr[mid] >= target) hi = mid; else lo = mid + 1;
    }
    out[b] = lo;
  }
}

// ---------------------------------------------------------------------------
// Panel SpMM: the x rows a run of rows gathers from are staged once in shared
// memory.  Graph orders in which each node's neighbours sit near it (kNN
// graphs of clustered data in cluster order, locality orders) give each block
// of ~kPanelBlockNnz entries a contiguous window of W x rows that holds most
// of its column indices; the block's gathers then hit shared memory (several
// entries per clock per SM) instead of issuing one scattered L2 request each,
// which is what bounds the direct kernels.  Entries outside the window fall
// back to a global gather.

// Window plan: for each panel block, the start w0 of the W-row window that
// holds the most of its column indices (histogram over bins of `bin` rows,
// best run of W / bin bins, ties to the lowest start), clamped to [0, n - W].
constexpr int kPanelBins = 4096;
constexpr int kPlanThreads = 256;

__global__ void __launch_bounds__(kPlanThreads) k_panel_windows(int64_t n, const uint64_t* __restrict__ indptr,
                                                                const uint32_t* __restrict__ indices,
                                                                const int64_t* __restrict__ prow, int64_t nblk, int W,
                                                                int bin, int nbins, int64_t* __restrict__ w0) {
  __shared__ int hist[kPanelBins];
  __shared__ long long best_key[kPlanThreads / 32];
  const int tid = threadIdx.x;
  const int wb = max(W / bin, 1);  // window length in bins
  const int nstart = max(nbins - wb + 1, 1);
  for (int64_t b = blockIdx.x; b < nblk; b += gridDim.x) {
    for (int i = tid; i < nbins; i += kPlanThreads) hist[i] = 0;
    __syncthreads();
    const uint64_t p0 = indptr[prow[b]], p1 = indptr[prow[b + 1]];
    for (uint64_t q = p0 + tid; q < p1; q += kPlanThreads) {
      const int bi = static_cast<int>(__ldg(indices + q) / static_cast<uint32_t>(bin));
      atomicAdd(&hist[min(bi, nbins - 1)], 1);
    }
    __syncthreads();
    // each thread scans a contiguous range of starts with a sliding sum;
    // key = count * 2^32 + (2^32 - 1 - start): max picks the most entries, then the lowest start
    const int per = (nstart + kPlanThreads - 1) / kPlanThreads;
    const int s0 = tid * per, s1 = min(s0 + per, nstart);
    long long key = -1;
    if (s0 < s1) {
      int sum = 0;
      for (int i = s0; i < min(s0 + wb, nbins); ++i) sum += hist[i];
      for (int st = s0; st < s1; ++st) {
        if (st > s0) sum += (st + wb - 1 < nbins ? hist[st + wb - 1] : 0) - hist[st - 1];
        const long long k = (static_cast<long long>(sum) << 32) | static_cast<long long>(0xffffffffu - st);
        key = max(key, k);
      }
    }
#pragma unroll
    for (int o = 16; o >= 1; o >>= 1) key = max(key, __shfl_xor_sync(0xffffffffu, key, o));
    if ((tid & 31) == 0) best_key[tid >> 5] = key;
    __syncthreads();
    if (tid == 0) {
      long long k = best_key[0];
      for (int w = 1; w < kPlanThreads / 32; ++w) k = max(k, best_key[w]);
      const int64_t st = static_cast<int64_t>(0xffffffffu - static_cast<unsigned>(k & 0xffffffffLL));
      int64_t start = st * bin;
      start = min(start, max(n - static_cast<int64_t>(W), int64_t(0)));
      // a block whose best window holds less than half of its entries gains
      // little from one: marked -1, it is computed with global gathers only
      const long long inside = k >> 32;
      w0[b] = (2 * inside < static_cast<long long>(p1 - p0)) ? int64_t(-1) : max(start, int64_t(0));
    }
    __syncthreads();
  }
}

// x row of LD elements from the shared-memory window (16-byte vector loads).
template <class XT, int LD>
__device__ __forceinline__ void smem_row(const XT* p, double (&v)[LD]) {
  if constexpr (std::is_same<XT, float>::value) {
#pragma unroll
    for (int q = 0; q < LD / 4; ++q) {
      const float4 t = reinterpret_cast<const float4*>(p)[q];
      v[4 * q + 0] = t.x;
      v[4 * q + 1] = t.y;
      v[4 * q + 2] = t.z;
      v[4 * q + 3] = t.w;
    }
  } else {
#pragma unroll
    for (int q = 0; q < LD / 2; ++q) {
      const double2 t = reinterpret_cast<const double2*>(p)[q];
      v[2 * q + 0] = t.x;
      v[2 * q + 1] = t.y;
    }
  }
}

// One row by a group of G lanes, gathers from the window [w, w + wn) when the
// column falls inside it (global memory otherwise).  The row's streams are
// addressed from its start with 32-bit offsets (the kernel is used only for
// operators with fewer than 2^31 entries), so the per-entry work is two
// streaming loads, one 16/32-byte gather and the LD fused multiply-adds; the
// own-row epilogue loads are issued before the gathers.
template <class VT, class XT, int LD, int G>
__device__ __forceinline__ void spmm_row_panel(int64_t row, uint64_t s, uint64_t e, const uint32_t* __restrict__ idx,
                                               const VT* __restrict__ val, double diag, const XT* __restrict__ x,
                                               const XT* panel, uint32_t w, uint32_t wn, XT* __restrict__ y,
                                               const Epilogue<XT>& ep, int sub, unsigned mask, bool writer) {
  constexpr int W = GroupReduce<LD, G>::W;
  constexpr int U = (LD >= 16) ? 4 : 8;
  const int obase = GroupReduce<LD, G>::base_of(sub);
  double own[W], addz[W];
#pragma unroll
  for (int c = 0; c < W; ++c) {
    own[c] = 0.0;
    addz[c] = 0.0;
    if (writer) {
      const int64_t off = row * LD + obase + c;
      own[c] = diag * static_cast<double>(x[off]);
      if (ep.z1) addz[c] = ep.beta * static_cast<double>(ep.z1[off]);
      if (ep.z2) addz[c] = fma(ep.gamma, static_cast<double>(ep.z2[off]), addz[c]);
      if (ep.z3) addz[c] = fma(ep.delta, static_cast<double>(ep.z3[off]), addz[c]);
    }
  }
  const uint32_t* __restrict__ ip = idx + s;
  const VT* __restrict__ vp = val + s;
  const int len = static_cast<int>(e - s);
  double acc[LD];
#pragma unroll
  for (int c = 0; c < LD; ++c) acc[c] = 0.0;
  for (int t0 = sub; t0 < len; t0 += G * U) {
    uint32_t jj[U];
    double vv[U];
#pragma unroll
    for (int u = 0; u < U; ++u) {
      const int t = t0 + u * G;
      const bool ok = t < len;
      jj[u] = ok ? ld_stream(ip + t) : 0u;
      vv[u] = ok ? static_cast<double>(ld_stream(vp + t)) : 0.0;
    }
#pragma unroll
    for (int u = 0; u < U; ++u) {
      if (t0 + u * G < len) {
        double xr[LD];
        const uint32_t d = jj[u] - w;
        if (d < wn) smem_row<XT, LD>(panel + static_cast<size_t>(d) * LD, xr);
        else RowLoad<XT, LD>::run(x + static_cast<size_t>(jj[u]) * LD, xr);
#pragma unroll
        for (int c = 0; c < LD; ++c) acc[c] = fma(vv[u], xr[c], acc[c]);
      }
    }
  }
  const int base = GroupReduce<LD, G>::run(acc, sub, mask);
  if (writer) {
#pragma unroll
    for (int c = 0; c < W; ++c) {
      const int64_t off = row * LD + base + c;
      y[off] = static_cast<XT>(fma(ep.alpha, own[c] + acc[c], addz[c]));
    }
  }
}

template <class XT, int LD>
constexpr int panel_threads() {
  return LD * sizeof(XT) <= 16 ? 1024 : 512;
}

template <class XT, int LD>
constexpr int panel_rows() {
  return (kPanelBytes / (LD * static_cast<int>(sizeof(XT)))) / 64 * 64;
}

// Persistent CTAs (one per SM): CTA c walks panel blocks [c*nblk/grid,
// (c+1)*nblk/grid); consecutive blocks with the same window form one run whose
// rows are spread over the CTA's row groups; the window is reloaded (between
// two CTA barriers) only when a run's window differs from the one held.
template <class VT, class XT, int LD, int G, int NT>
__global__ void __launch_bounds__(NT, 1) k_spmm_panel(int64_t n, const uint64_t* __restrict__ indptr,
                                                      const uint32_t* __restrict__ indices,
                                                      const VT* __restrict__ vals, const int64_t* __restrict__ prow,
                                                      const int64_t* __restrict__ pw0, int64_t nblk, double diag,
                                                      const XT* __restrict__ x, XT* __restrict__ y, Epilogue<XT> ep,
                                                      const int* __restrict__ stop) {
  if (stop != nullptr && *stop != 0) return;
  constexpr int WR = panel_rows<XT, LD>();
  extern __shared__ __align__(16) unsigned char panel_raw[];
  XT* panel = reinterpret_cast<XT*>(panel_raw);
  const int tid = threadIdx.x;
  const int lane = tid & 31;
  const int sub = lane & (G - 1);
  const unsigned mask = group_mask<G>(lane);
  const bool writer = group_writer<LD, G>(sub);
  const int group = tid / G;
  constexpr int NG = NT / G;
  const int64_t b_lo = nblk * blockIdx.x / gridDim.x;
  const int64_t b_hi = nblk * (blockIdx.x + 1) / gridDim.x;
  // a block whose planned window lies within WR/8 rows of the one held keeps
  // the held window (it covers nearly the same columns): reloads only happen
  // when the window really moves
  constexpr int64_t kSlack = WR / 8;
  int64_t held = -1;
  for (int64_t b = b_lo; b < b_hi;) {
    int64_t w = pw0[b];
    if (w < 0) {  // no useful window: left to the second phase
      ++b;
      continue;
    }
    if (held >= 0 && llabs(w - held) <= kSlack) w = held;
    int64_t be = b + 1;
    while (be < b_hi && pw0[be] >= 0 && llabs(pw0[be] - w) <= kSlack) ++be;
    const int64_t r0 = prow[b], r1 = prow[be];
    const uint32_t wn = static_cast<uint32_t>(min(static_cast<int64_t>(WR), n - w));
    if (w != held) {
      __syncthreads();  // every row of the previous run is done with the old window
      constexpr int VEC = 16 / sizeof(XT);
      const int64_t nvec = static_cast<int64_t>(wn) * LD / VEC;
      const uint4* src = reinterpret_cast<const uint4*>(x + w * LD);
      uint4* dst = reinterpret_cast<uint4*>(panel);
      for (int64_t i = tid; i < nvec; i += NT) dst[i] = __ldcg(src + i);
      __syncthreads();
      held = w;
    }
    for (int64_t row = r0 + group; row < r1; row += NG)
      spmm_row_panel<VT, XT, LD, G>(row, indptr[row], indptr[row + 1], indices, vals, diag, x, panel,
                                    static_cast<uint32_t>(w), wn, y, ep, sub, mask, writer);
    b = be;
  }
  // second phase: blocks without a window (rows whose columns scatter over
  // the whole graph), spread over all CTAs, global gathers only
  for (int64_t b = blockIdx.x; b < nblk; b += gridDim.x) {
    if (pw0[b] >= 0) continue;
    const int64_t r0 = prow[b], r1 = prow[b + 1];
    for (int64_t row = r0 + group; row < r1; row += NG)
      spmm_row_panel<VT, XT, LD, G>(row, indptr[row], indptr[row + 1], indices, vals, diag, x, panel, 0u, 0u, y,
                                    ep, sub, mask, writer);
  }
}

// Generic kernel: any row stride ld, first k columns, four columns per pass.
template <class VT, class XT, int G>
__global__ void __launch_bounds__(256) k_spmm_generic(int64_t n, const uint64_t* __restrict__ indptr,
                                                      const uint32_t* __restrict__ indices,
                                                      const VT* __restrict__ vals, double diag,
                                                      const XT* __restrict__ x, XT* __restrict__ y, int ld,
                                                      int k, Epilogue<XT> ep, const int* __restrict__ stop) {
  if (stop != nullptr && *stop != 0) return;
  const int lane = threadIdx.x & 31;
  const int sub = lane & (G - 1);
  const unsigned mask = (G == 32) ? 0xffffffffu : (((1u << G) - 1u) << (lane & ~(G - 1)));
  const int64_t group = (static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x) / G;
  const int64_t ngroups = static_cast<int64_t>(gridDim.x) * blockDim.x / G;
  for (int64_t row = group; row < n; row += ngroups) {
    const uint64_t s = indptr[row];
    const uint64_t e = indptr[row + 1];
    for (int c0 = 0; c0 < k; c0 += 4) {
      double acc[4] = {0.0, 0.0, 0.0, 0.0};
      for (uint64_t q = s + sub; q < e; q += G) {
        const int64_t j = ld_stream(indices + q);
        const double v = static_cast<double>(ld_stream(vals + q));
#pragma unroll
        for (int c = 0; c < 4; ++c)
          if (c0 + c < k) acc[c] = fma(v, static_cast<double>(__ldg(x + j * ld + c0 + c)), acc[c]);
      }
#pragma unroll
      for (int c = 0; c < 4; ++c)
#pragma unroll
        for (int o = G / 2; o >= 1; o >>= 1) acc[c] += __shfl_xor_sync(mask, acc[c], o, G);
      if (sub < 4 && c0 + sub < k) {
        double a = acc[0];
#pragma unroll
        for (int c = 1; c < 4; ++c)
          if (sub == c) a = acc[c];
        const int64_t off = row * ld + c0 + sub;
        double r = fma(diag, static_cast<double>(x[off]), a);
        r *= ep.alpha;
        if (ep.z1) r = fma(ep.beta, static_cast<double>(ep.z1[off]), r);
        if (ep.z2) r = fma(ep.gamma, static_cast<double>(ep.z2[off]), r);
        if (ep.z3) r = fma(ep.delta, static_cast<double>(ep.z3[off]), r);
        y[off] = static_cast<XT>(r);
      }
    }
  }
}

// TMA-gather kernel (f32 values, 4-wide f32 rows): the x rows of a block's
// entries are fetched by tile::gather4 copies (four rows per instruction,
// through the TMA unit instead of per-lane loads) into a double-buffered
// shared-memory staging area, while the previous block is computed from it.
// A block (about kGatherBlockNnz entries, at most kGatherCap) is gathered
// into 128-byte slots of four 16-byte rows.  Waits give up after one second
// and record an error instead of hanging; blocks that do not fit the staging
// area use plain gathers.
constexpr int kGatherSlots = kGatherCap / 4;

template <int G>
__device__ __forceinline__ void gather_row(int64_t row, uint64_t s, uint64_t e, uint64_t p0, const float* slots,
                                           const float* __restrict__ vals, double diag, const float* __restrict__ x,
                                           float* __restrict__ y, const Epilogue<float>& ep, int sub, unsigned mask,
                                           bool writer) {
  constexpr int LD = 4;
  constexpr int W = GroupReduce<LD, G>::W;
  const int obase = GroupReduce<LD, G>::base_of(sub);
  double own[W], addz[W];
#pragma unroll
  for (int c = 0; c < W; ++c) {
    own[c] = 0.0;
    addz[c] = 0.0;
    if (writer) {
      const int64_t off = row * LD + obase + c;
      own[c] = diag * static_cast<double>(x[off]);
      if (ep.z1) addz[c] = ep.beta * static_cast<double>(ep.z1[off]);
      if (ep.z2) addz[c] = fma(ep.gamma, static_cast<double>(ep.z2[off]), addz[c]);
      if (ep.z3) addz[c] = fma(ep.delta, static_cast<double>(ep.z3[off]), addz[c]);
    }
  }
  double acc[LD] = {0.0, 0.0, 0.0, 0.0};
  for (uint64_t k = s + sub; k < e; k += G) {
    const uint64_t q = k - p0;  // entry within the block: slot q / 4, row q % 4 of the slot
    const float4 xr = *reinterpret_cast<const float4*>(slots + (q >> 2) * 32 + (q & 3) * 4);
    const double v = static_cast<double>(__ldcs(vals + k));
    acc[0] = fma(v, static_cast<double>(xr.x), acc[0]);
    acc[1] = fma(v, static_cast<double>(xr.y), acc[1]);
    acc[2] = fma(v, static_cast<double>(xr.z), acc[2]);
    acc[3] = fma(v, static_cast<double>(xr.w), acc[3]);
  }
  const int base = GroupReduce<LD, G>::run(acc, sub, mask);
  if (writer) {
#pragma unroll
    for (int c = 0; c < W; ++c) {
      const int64_t off = row * LD + base + c;
      y[off] = static_cast<float>(fma(ep.alpha, own[c] + acc[c], addz[c]));
    }
  }
}

template <int G>
__global__ void __launch_bounds__(256) k_spmm_gather(const __grid_constant__ CUtensorMap xmap, int64_t n,
                                                     const uint64_t* __restrict__ indptr,
                                                     const uint32_t* __restrict__ indices,
                                                     const float* __restrict__ vals, const int64_t* __restrict__ rblk,
                                                     const uint64_t* __restrict__ bptr, int64_t nblk, double diag,
                                                     const float* __restrict__ x, float* __restrict__ y,
                                                     Epilogue<float> ep, const int* __restrict__ stop, int* err) {
  if (stop != nullptr && *stop != 0) return;
  __shared__ __align__(128) float slots[2][kGatherSlots][32];
  __shared__ __align__(8) uint64_t mbar[2];
  __shared__ int s_bad;
  const int tid = threadIdx.x;
  const int lane = tid & 31;
  const int sub = lane & (G - 1);
  const unsigned mask = group_mask<G>(lane);
  const bool writer = group_writer<4, G>(sub);
  const int group = tid / G;
  constexpr int NG = 256 / G;
  if (tid == 0) {
    umma::mbar_init(&mbar[0], 1);
    umma::mbar_init(&mbar[1], 1);
    umma::fence_mbar_init();
    umma::tma_prefetch_desc(&xmap);
    s_bad = 0;
  }
  __syncthreads();
  uint32_t phase[2] = {0u, 0u};
  auto info = [&](int64_t b) {
    BlockInfo bi;
    if (b < nblk) {
      bi.r0 = rblk[b];
      bi.r1 = rblk[b + 1];
      bi.p0 = bptr[b];
      bi.p1 = bptr[b + 1];
    }
    return bi;
  };
  auto staged = [](const BlockInfo& bi) { return bi.p1 > bi.p0 && (bi.p1 - bi.p0) <= kGatherCap; };
  // all threads: one thread posts the byte count, then every thread issues its gathers
  auto issue = [&](const BlockInfo& bi, int st) {
    const int ne = static_cast<int>(bi.p1 - bi.p0);
    const int ng = (ne + 3) / 4;
    if (tid == 0) umma::mbar_arrive_expect_tx(&mbar[st], static_cast<uint32_t>(ng) * 64u);
    __syncthreads();
    const int32_t pad = static_cast<int32_t>(__ldg(indices + bi.p0));  // a valid row for the unused tail
    for (int g = tid; g < ng; g += 256) {
      int32_t r[4];
#pragma unroll
      for (int q = 0; q < 4; ++q) {
        const uint64_t k = bi.p0 + 4 * g + q;
        r[q] = k < bi.p1 ? static_cast<int32_t>(__ldg(indices + k)) : pad;
      }
      umma::tma_gather4(&slots[st][g][0], &xmap, &mbar[st], 0, r[0], r[1], r[2], r[3]);
    }
  };
  const int64_t step = gridDim.x;
  int64_t b = blockIdx.x;
  int st = 0;
  bool pending[2] = {false, false};  // a stage with copies not yet waited for
  bool tma_on = true;                // cleared (uniformly) after a wait gave up
  BlockInfo cur = info(b);
  bool cur_staged = b < nblk && staged(cur);
  if (cur_staged) {
    issue(cur, 0);
    pending[0] = true;
  }
  for (; b < nblk; b += step) {
    const BlockInfo nxt = info(b + step);
    const bool nxt_staged = tma_on && b + step < nblk && staged(nxt);
    if (nxt_staged) {
      issue(nxt, st ^ 1);
      pending[st ^ 1] = true;
    }
    if (cur_staged) {
      if (umma::mbar_wait(&mbar[st], phase[st])) {
        phase[st] ^= 1u;
        pending[st] = false;
      } else {
        s_bad = 1;
      }
    }
    __syncthreads();
    if (s_bad) tma_on = false;
    if (cur_staged && tma_on) {
      for (int64_t rr = cur.r0 + group; rr < cur.r1; rr += NG)
        gather_row<G>(rr, indptr[rr], indptr[rr + 1], cur.p0, &slots[st][0][0], vals, diag, x, y, ep, sub, mask,
                      writer);
    } else {
      const GlobalStream<float> src{indices, vals};
      for (int64_t rr = cur.r0 + group; rr < cur.r1; rr += NG)
        spmm_row<float, float, 4, G>(rr, indptr[rr], indptr[rr + 1], src, diag, x, y, ep, sub, mask, writer);
    }
    __syncthreads();
    st ^= 1;
    cur = nxt;
    cur_staged = nxt_staged;
  }
  if (s_bad) {
    // a wait gave up (those blocks were computed with plain gathers): let the
    // copies still in flight land, within the same limit, before exit
    for (int s2 = 0; s2 < 2; ++s2)
      if (pending[s2]) umma::mbar_wait(&mbar[s2], phase[s2]);
    if (tid == 0) atomicExch(err, 1);
    __syncthreads();
  }
}

CUtensorMap x_rows_map(const float* x, int64_t n) {
  SI_REQUIRE(reinterpret_cast<uintptr_t>(x) % 16 == 0, SI_INVALID_ARGUMENT, "spmm: x not 16-byte aligned");
  SI_REQUIRE(n < (int64_t(1) << 31), SI_INVALID_ARGUMENT, "spmm: too many rows for the gather path");
  CUtensorMap map;
  const cuuint64_t dims[2] = {4, static_cast<cuuint64_t>(n)};
  const cuuint64_t strides[1] = {16};
  const cuuint32_t box[2] = {4, 1};
  const cuuint32_t estr[2] = {1, 1};
  const CUresult r = tensor_map_encoder()(&map, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 2, const_cast<float*>(x), dims,
                                          strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
                                          CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_NONE,
                                          CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  SI_REQUIRE(r == CUDA_SUCCESS, SI_CUDA_ERROR, "cuTensorMapEncodeTiled (x rows) failed");
  return map;
}

// error flag of the gather kernel, one per device (set only by a timed-out wait)
int* gather_err(const Exec& ex) {
  static std::mutex mu;
  static int* flags[128] = {};
  std::lock_guard<std::mutex> lk(mu);
  const int dev = (ex.device >= 0 && ex.device < 128) ? ex.device : 0;
  if (flags[dev] == nullptr) {
    SI_CUDA(cudaMalloc(reinterpret_cast<void**>(&flags[dev]), sizeof(int)));
    SI_CUDA(cudaMemset(flags[dev], 0, sizeof(int)));
  }
  return flags[dev];
}

template <int G>
void launch_gather(const Exec& ex, const OpDev& op, const float* vals, const float* x, float* y,
                   const Epilogue<float>& ep, const int* stop) {
  const CUtensorMap map = x_rows_map(x, op.n);
  int per_sm = 0;
  static std::atomic<int> resident[128];
  const int dev = (ex.device >= 0 && ex.device < 128) ? ex.device : 0;
  if (resident[dev] == 0) {
    SI_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_spmm_gather<G>, 256, 0));
    resident[dev] = std::max(per_sm, 1);
  }
  const int grid = static_cast<int>(
      std::max<int64_t>(1, std::min<int64_t>(op.n_gather_blocks, int64_t(ex.sms) * resident[dev])));
  k_spmm_gather<G><<<grid, 256, 0, ex.stream>>>(map, op.n, op.indptr, op.indices, vals, op.gather_blocks,
                                                op.gather_ptr, op.n_gather_blocks, op.diag, x, y, ep, stop,
                                                gather_err(ex));
  SI_LAUNCH_CHECK();
}

template <class VT, class XT, int LD, int G>
void launch_vec(const Exec& ex, const OpDev& op, const VT* vals, const XT* x, XT* y, const Epilogue<XT>& ep,
                const int* stop) {
  const int threads = 256;
  const int64_t need = (op.n * G + threads - 1) / threads;
  const int grid = static_cast<int>(std::max<int64_t>(1, std::min<int64_t>(need, int64_t(ex.sms) * 8)));
  k_spmm_vec<VT, XT, LD, G><<<grid, threads, 0, ex.stream>>>(op.n, op.indptr, op.indices, vals, op.diag, x, y,
                                                              ep, stop);
  SI_LAUNCH_CHECK();
}

template <class VT, class XT, int G>
void launch_generic(const Exec& ex, const OpDev& op, const VT* vals, const XT* x, XT* y, int ld, int k,
                    const Epilogue<XT>& ep, const int* stop) {
  const int threads = 256;
  const int64_t need = (op.n * G + threads - 1) / threads;
  const int grid = static_cast<int>(std::max<int64_t>(1, std::min<int64_t>(need, int64_t(ex.sms) * 8)));
  k_spmm_generic<VT, XT, G><<<grid, threads, 0, ex.stream>>>(op.n, op.indptr, op.indices, vals, op.diag, x, y,
                                                              ld, k, ep, stop);
  SI_LAUNCH_CHECK();
}

template <class VT, class XT, int LD, int G>
void launch_tiled(const Exec& ex, const OpDev& op, const VT* vals, const XT* x, XT* y, const Epilogue<XT>& ep,
                  const int* stop) {
  const int smem = static_cast<int>(sizeof(TileSmem<VT>));
  static std::atomic<int> resident[128];  // per device: resident CTAs per SM (0 = not set up)
  const int dev = (ex.device >= 0 && ex.device < 128) ? ex.device : 0;
  if (resident[dev] == 0) {
    SI_CUDA(cudaFuncSetAttribute(k_spmm_tiled<VT, XT, LD, G>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
    int per_sm = 0;
    SI_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_spmm_tiled<VT, XT, LD, G>, 256, smem));
    resident[dev] = std::max(per_sm, 1);
  }
  const int grid = static_cast<int>(
      std::max<int64_t>(1, std::min<int64_t>(op.n_blocks, int64_t(ex.sms) * resident[dev])));
  k_spmm_tiled<VT, XT, LD, G><<<grid, 256, smem, ex.stream>>>(op.n, op.indptr, op.indices, vals, op.row_blocks,
                                                               op.block_ptr, op.n_blocks, op.diag, x, y, ep, stop);
  SI_LAUNCH_CHECK();
}

// Windows of the panel SpMM for window size W (built on first use, outside
// stream capture; null when the operator has no panel partition or when the
// windows would have to be built inside a capture).
const int64_t* panel_windows(const Exec& ex, const OpDev& op, int W) {
  if (op.panels == nullptr || op.panels->n_pblocks <= 0 || W <= 0) return nullptr;
  for (const PanelWindows& pw : op.panels->windows)
    if (pw.W == W) return pw.w0.get();
  cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
  SI_CUDA(cudaStreamIsCapturing(ex.stream, &cs));
  if (cs != cudaStreamCaptureStatusNone) return nullptr;
  int64_t bin = std::max<int64_t>(1, (W + 7) / 8);
  int64_t nbins = (op.n + bin - 1) / bin;
  if (nbins > kPanelBins) {
    bin = (op.n + kPanelBins - 1) / kPanelBins;
    nbins = (op.n + bin - 1) / bin;
  }
  PanelWindows pw;
  pw.W = W;
  const int64_t nb = op.panels->n_pblocks;
  pw.w0.alloc(static_cast<size_t>(nb), ex.stream);
  const int grid = static_cast<int>(std::max<int64_t>(1, std::min<int64_t>(nb, int64_t(ex.sms) * 8)));
  k_panel_windows<<<grid, kPlanThreads, 0, ex.stream>>>(op.n, op.indptr, op.indices, op.panels->pstarts.get(), nb, W,
                                                        static_cast<int>(bin), static_cast<int>(std::max<int64_t>(nbins, 1)),
                                                        pw.w0.get());
  SI_LAUNCH_CHECK();
  op.panels->windows.push_back(std::move(pw));
  return op.panels->windows.back().w0.get();
}

template <class VT, class XT, int LD>
bool launch_panel(const Exec& ex, const OpDev& op, const VT* vals, const XT* x, XT* y, const Epilogue<XT>& ep,
                  const int* stop) {
  constexpr int WR = panel_rows<XT, LD>();
  constexpr int NT = panel_threads<XT, LD>();
  constexpr int G = 4;
  if (op.nnz >= (int64_t(1) << 31)) return false;  // 32-bit offsets within a row
  const int64_t* w0 = panel_windows(ex, op, WR);
  if (w0 == nullptr) return false;
  const int smem = WR * LD * static_cast<int>(sizeof(XT));
  static std::atomic<int> ready[128];
  const int dev = (ex.device >= 0 && ex.device < 128) ? ex.device : 0;
  if (ready[dev] == 0) {
    SI_CUDA(cudaFuncSetAttribute(k_spmm_panel<VT, XT, LD, G, NT>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
    ready[dev] = 1;
  }
  const int grid = static_cast<int>(std::max<int64_t>(1, std::min<int64_t>(op.panels->n_pblocks, int64_t(ex.sms))));
  k_spmm_panel<VT, XT, LD, G, NT><<<grid, NT, smem, ex.stream>>>(op.n, op.indptr, op.indices, vals,
                                                                  op.panels->pstarts.get(), w0, op.panels->n_pblocks,
                                                                  op.diag, x, y, ep, stop);
  SI_LAUNCH_CHECK();
  return true;
}

// ---------------------------------------------------------------------------
// Sliced SpMM.  One lane owns one row of a 32-row slice of the sliced-ELL copy
// (SellLayout), so a warp's index and value loads are two coalesced 128-byte
// requests per 32 entries, no lane waits on another's row bounds, and the row
// sum needs no cross-lane reduction.  Rows are sorted by length inside
// 4096-row windows, so a slice is about as wide as its average row; rows far
// longer than the mean (hubs of kNN graphs) would make their slice that wide
// and are instead read from the CSR arrays by a whole warp each.  Persistent
// CTAs own contiguous slice ranges (balanced by slot count) and an equal share
// of the long rows; inside a CTA warps take long rows first, then slices, from
// shared counters.  With L1-cached gathers the x rows of a CTA's neighbourhood
// stay in the SM's L1 for graphs whose node order keeps neighbours near (kNN
// graphs of clustered data, locality orders).

// Counting sort of each window of kSellSortRows rows by length (longest
// first), short rows only; the window's long rows go to its segment of
// `long_tmp` and their count to long_cnt[window].  Positions past the
// window's short rows are empty lanes.
__global__ void __launch_bounds__(kSellSortThreads) k_sell_sort(int64_t n, const uint64_t* __restrict__ indptr,
                                                                 int long_min, uint32_t* __restrict__ perm,
                                                                 uint32_t* __restrict__ plen,
                                                                 uint32_t* __restrict__ long_tmp,
                                                                 uint64_t* __restrict__ long_cnt) {
  constexpr int R = kSellSortRows / kSellSortThreads;
  __shared__ int hist[kSellMaxShort + 1];  // bin long_min - 1 - len: longest first
  __shared__ int n_long, n_short;
  const int nb = long_min;  // lengths 0 .. long_min - 1
  for (int i = threadIdx.x; i < nb; i += blockDim.x) hist[i] = 0;
  if (threadIdx.x == 0) n_long = 0;
  __syncthreads();
  const int64_t w0 = static_cast<int64_t>(blockIdx.x) * kSellSortRows;
  int lens[R];
#pragma unroll
  for (int q = 0; q < R; ++q) {
    const int64_t row = w0 + threadIdx.x + q * kSellSortThreads;
    lens[q] = -1;
    if (row < n) {
      const uint64_t len = indptr[row + 1] - indptr[row];
      if (len >= static_cast<uint64_t>(long_min)) {
        const int p = atomicAdd(&n_long, 1);
        long_tmp[w0 + p] = static_cast<uint32_t>(row);
      } else {
        lens[q] = static_cast<int>(len);
        atomicAdd(&hist[nb - 1 - lens[q]], 1);
      }
    }
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    int run = 0;
    for (int i = 0; i < nb; ++i) {
      const int c = hist[i];
      hist[i] = run;
      run += c;
    }
    n_short = run;
    long_cnt[blockIdx.x] = static_cast<uint64_t>(n_long);
  }
  __syncthreads();
#pragma unroll
  for (int q = 0; q < R; ++q) {
    if (lens[q] >= 0) {
      const int p = atomicAdd(&hist[nb - 1 - lens[q]], 1);
      perm[w0 + p] = static_cast<uint32_t>(w0 + threadIdx.x + q * kSellSortThreads);
      plen[w0 + p] = static_cast<uint32_t>(lens[q]);
    }
  }
  for (int i = n_short + threadIdx.x; i < kSellSortRows; i += blockDim.x) {
    perm[w0 + i] = 0xffffffffu;
    plen[w0 + i] = 0u;
  }
}

// Long rows of every window into one list (window order).
__global__ void k_sell_long_compact(int64_t n_win, const uint32_t* __restrict__ long_tmp,
                                    const uint64_t* __restrict__ long_ptr, uint32_t* __restrict__ long_rows) {
  for (int64_t w = blockIdx.x; w < n_win; w += gridDim.x) {
    const uint64_t b = long_ptr[w];
    const int c = static_cast<int>(long_ptr[w + 1] - b);
    for (int i = threadIdx.x; i < c; i += blockDim.x) long_rows[b + i] = long_tmp[w * kSellSortRows + i];
  }
}

// Slots of each slice (32 x its first, longest row), one more zero entry for
// the scan.
__global__ void k_sell_widths(int64_t n_slices, const uint32_t* __restrict__ plen, uint64_t* __restrict__ cnt) {
  for (int64_t s = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; s <= n_slices;
       s += static_cast<int64_t>(gridDim.x) * blockDim.x)
    cnt[s] = s < n_slices ? 32ull * plen[s * 32] : 0ull;
}

// Copy of the index and value streams into slots: one warp a slice.
__global__ void k_sell_fill(int64_t n_slices, const uint64_t* __restrict__ slice_ptr,
                            const uint32_t* __restrict__ perm, const uint32_t* __restrict__ plen,
                            const uint64_t* __restrict__ indptr, const uint32_t* __restrict__ indices,
                            const float* __restrict__ v32, const double* __restrict__ v64,
                            uint32_t* __restrict__ sidx, float* __restrict__ s32, double* __restrict__ s64) {
  const int lane = threadIdx.x & 31;
  const int64_t warps = static_cast<int64_t>(gridDim.x) * (blockDim.x / 32);
  for (int64_t s = (static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x) / 32; s < n_slices; s += warps) {
    const uint64_t base = slice_ptr[s];
    const uint64_t w = (slice_ptr[s + 1] - base) / 32;
    const uint32_t row = perm[s * 32 + lane];
    const uint64_t len = plen[s * 32 + lane];
    const uint64_t src = row != 0xffffffffu ? indptr[row] : 0;
    for (uint64_t j = 0; j < w; ++j) {
      const uint64_t slot = base + 32 * j + lane;
      const bool ok = j < len;
      sidx[slot] = ok ? indices[src + j] : 0u;
      if (s32 != nullptr) s32[slot] = ok ? v32[src + j] : 0.0f;
      if (s64 != nullptr) s64[slot] = ok ? v64[src + j] : 0.0;
    }
  }
}

// x row gather for the sliced kernel: L1-cached (.nc; measured faster on
// every operator tried) or L2-only (.cg).
template <class XT, int LD, bool L1>
struct SellRowLoad;
template <int LD, bool L1>
struct SellRowLoad<double, LD, L1> {
  __device__ __forceinline__ static void run(const double* p, double (&v)[LD]) {
#pragma unroll
    for (int q = 0; q < LD / 4; ++q) {
      double a, b, c, d;
      if constexpr (L1)
        asm volatile("ld.global.nc.v4.f64 {%0,%1,%2,%3}, [%4];" : "=d"(a), "=d"(b), "=d"(c), "=d"(d) : "l"(p + 4 * q));
      else
        asm volatile("ld.global.cg.v4.f64 {%0,%1,%2,%3}, [%4];" : "=d"(a), "=d"(b), "=d"(c), "=d"(d) : "l"(p + 4 * q));
      v[4 * q + 0] = a;
      v[4 * q + 1] = b;
      v[4 * q + 2] = c;
      v[4 * q + 3] = d;
    }
  }
};
template <int LD, bool L1>
struct SellRowLoad<float, LD, L1> {
  __device__ __forceinline__ static void run(const float* p, double (&v)[LD]) {
#pragma unroll
    for (int q = 0; q < LD / 4; ++q) {
      const float4* a = reinterpret_cast<const float4*>(p + 4 * q);
      const float4 t = L1 ? __ldg(a) : __ldcg(a);
      v[4 * q + 0] = t.x;
      v[4 * q + 1] = t.y;
      v[4 * q + 2] = t.z;
      v[4 * q + 3] = t.w;
    }
  }
};

// First slice whose slot offset is >= target (n_slices when none).
__device__ __forceinline__ int64_t sell_bound(const uint64_t* __restrict__ slice_ptr, int64_t n_slices,
                                              uint64_t target) {
  int64_t lo = 0, hi = n_slices;
  while (lo < hi) {
    const int64_t mid = (lo + hi) / 2;
    if (slice_ptr[mid] < target) lo = mid + 1;
    else hi = mid;
  }
  return lo;
}

struct SellArgs {
  int64_t n_slices, n_long;
  const uint64_t* slice_ptr;
  const uint32_t* perm;
  const uint32_t* plen;
  const uint32_t* sidx;
  const uint32_t* long_rows;
  const uint64_t* indptr;  // CSR arrays, for the long rows
  const uint32_t* indices;
};

// Bulk prefetch of [p, p + bytes) into L2 (p and bytes multiples of 16).
__device__ __forceinline__ void l2_prefetch_bulk(const void* p, uint32_t bytes) {
  asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"(p), "r"(bytes) : "memory");
}

template <class VT, class XT, int LD, int U, int NT, bool L1, bool PF, bool PIPE>
__global__ void __launch_bounds__(NT, 1) k_spmm_sell(SellArgs a, const VT* __restrict__ sval,
                                                     const VT* __restrict__ vals, double diag,
                                                     const XT* __restrict__ x, XT* __restrict__ y, Epilogue<XT> ep,
                                                     const int* __restrict__ stop) {
  if (stop != nullptr && *stop != 0) return;
  __shared__ long long next_long, next_slice;
  const int lane = threadIdx.x & 31;
  const uint64_t total = a.slice_ptr[a.n_slices];
  const int64_t s_lo = blockIdx.x == 0 ? 0 : sell_bound(a.slice_ptr, a.n_slices, total * blockIdx.x / gridDim.x);
  const int64_t s_hi =
      blockIdx.x + 1 == gridDim.x ? a.n_slices : sell_bound(a.slice_ptr, a.n_slices, total * (blockIdx.x + 1) / gridDim.x);
  const int64_t l_lo = a.n_long * blockIdx.x / gridDim.x;
  const int64_t l_hi = a.n_long * (blockIdx.x + 1) / gridDim.x;
  if (threadIdx.x == 0) {
    next_long = l_lo;
    next_slice = s_lo;
  }
  __syncthreads();
  // long rows: a warp each, straight from the CSR arrays
  const GlobalStream<VT> src{a.indices, vals};
  const bool writer = group_writer<LD, 32>(lane);
  for (;;) {
    long long i = 0;
    if (lane == 0) i = atomicAdd(reinterpret_cast<unsigned long long*>(&next_long), 1ull);
    i = __shfl_sync(0xffffffffu, i, 0);
    if (i >= l_hi) break;
    const int64_t row = a.long_rows[i];
    spmm_row<VT, XT, LD, 32>(row, a.indptr[row], a.indptr[row + 1], src, diag, x, y, ep, lane, 0xffffffffu, writer);
  }
  // slices: a lane a row
  constexpr int NW = NT / 32;
  for (;;) {
    long long s = 0;
    if (lane == 0) s = atomicAdd(reinterpret_cast<unsigned long long*>(&next_slice), 1ull);
    s = __shfl_sync(0xffffffffu, s, 0);
    if (s >= s_hi) break;
    if (PF && lane == 0 && s + NW < s_hi) {
      // the slice a warp of this CTA takes about NW slices from now: its
      // index and value streams into L2 while this slice is computed
      const uint64_t pb = a.slice_ptr[s + NW];
      const uint64_t pc = a.slice_ptr[s + NW + 1] - pb;
      if (pc > 0) {
        l2_prefetch_bulk(a.sidx + pb, static_cast<uint32_t>(pc * sizeof(uint32_t)));
        l2_prefetch_bulk(sval + pb, static_cast<uint32_t>(pc * sizeof(VT)));
      }
    }
    const uint64_t base = a.slice_ptr[s];
    const int w = static_cast<int>((a.slice_ptr[s + 1] - base) / 32);
    const uint32_t row = a.perm[s * 32 + lane];
    const int len = static_cast<int>(a.plen[s * 32 + lane]);
    const uint32_t* __restrict__ ip = a.sidx + base + lane;
    const VT* __restrict__ vp = sval + base + lane;
    double acc[LD];
#pragma unroll
    for (int c = 0; c < LD; ++c) acc[c] = 0.0;
    if constexpr (PIPE) {
      // the next U positions' indices and values are loaded before this U's
      // gathers, so the stream latency overlaps the gather latency
      uint32_t jj[U];
      VT vr[U];
#pragma unroll
      for (int u = 0; u < U; ++u) {
        const bool ok = u < w;
        jj[u] = ok ? ld_stream(ip + 32 * u) : 0u;
        vr[u] = ok ? ld_stream(vp + 32 * u) : VT(0);
      }
      for (int j0 = 0; j0 < w; j0 += U) {
        ip += 32 * U;
        vp += 32 * U;
        uint32_t nj[U];
        VT nv[U];
#pragma unroll
        for (int u = 0; u < U; ++u) {
          const bool ok = j0 + U + u < w;
          nj[u] = ok ? ld_stream(ip + 32 * u) : 0u;
          nv[u] = ok ? ld_stream(vp + 32 * u) : VT(0);
        }
#pragma unroll
        for (int u = 0; u < U; ++u) {
          if (j0 + u < len) {
            double xr[LD];
            SellRowLoad<XT, LD, L1>::run(x + static_cast<size_t>(jj[u]) * LD, xr);
            const double v = static_cast<double>(vr[u]);
#pragma unroll
            for (int c = 0; c < LD; ++c) acc[c] = fma(v, xr[c], acc[c]);
          }
        }
#pragma unroll
        for (int u = 0; u < U; ++u) {
          jj[u] = nj[u];
          vr[u] = nv[u];
        }
      }
    } else {
      for (int j0 = 0; j0 < w; j0 += U, ip += 32 * U, vp += 32 * U) {
        uint32_t jj[U];
        double vv[U];
#pragma unroll
        for (int u = 0; u < U; ++u) {
          const bool ok = j0 + u < w;
          jj[u] = ok ? ld_stream(ip + 32 * u) : 0u;
          vv[u] = ok ? static_cast<double>(ld_stream(vp + 32 * u)) : 0.0;
        }
#pragma unroll
        for (int u = 0; u < U; ++u) {
          if (j0 + u < len) {
            double xr[LD];
            SellRowLoad<XT, LD, L1>::run(x + static_cast<size_t>(jj[u]) * LD, xr);
#pragma unroll
            for (int c = 0; c < LD; ++c) acc[c] = fma(vv[u], xr[c], acc[c]);
          }
        }
      }
    }
    if (row != 0xffffffffu) {
      const size_t off = static_cast<size_t>(row) * LD;
#pragma unroll
      for (int c = 0; c < LD; ++c) {
        const double own = diag * static_cast<double>(x[off + c]);
        double addz = 0.0;
        if (ep.z1) addz = ep.beta * static_cast<double>(ep.z1[off + c]);
        if (ep.z2) addz = fma(ep.gamma, static_cast<double>(ep.z2[off + c]), addz);
        if (ep.z3) addz = fma(ep.delta, static_cast<double>(ep.z3[off + c]), addz);
        y[off + c] = static_cast<XT>(fma(ep.alpha, own + acc[c], addz));
      }
    }
  }
}

// The sliced-ELL copy of the operator (built on first use, outside stream
// capture, for owners that allow it; null when not available).
const SellLayout* sell_layout(const Exec& ex, const OpDev& op) {
  if (op.panels == nullptr || !op.panels->sell_ok || op.panels->sell_failed) return nullptr;
  if (op.panels->sell) return op.panels->sell.get();
  if (op.n <= 0 || op.n >= int64_t(0xffffffff) - kSellSortRows || op.nnz >= (int64_t(1) << 32)) return nullptr;
  cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
  SI_CUDA(cudaStreamIsCapturing(ex.stream, &cs));
  if (cs != cudaStreamCaptureStatusNone) return nullptr;
  auto L = std::make_unique<SellLayout>();
  // rows of 4x the mean length or more (at least 128, at most kSellMaxShort+1) are long
  const double mean = static_cast<double>(op.nnz) / static_cast<double>(op.n);
  L->long_min = static_cast<int>(std::min<double>(kSellMaxShort + 1, std::max(128.0, std::ceil(4.0 * mean))));
  const int64_t n_win = (op.n + kSellSortRows - 1) / kSellSortRows;
  const int64_t n_pad = n_win * kSellSortRows;
  L->n_slices = n_pad / 32;
  L->perm.alloc(static_cast<size_t>(n_pad), ex.stream);
  L->plen.alloc(static_cast<size_t>(n_pad), ex.stream);
  DevBuf<uint32_t> long_tmp(static_cast<size_t>(n_pad), ex.stream);
  DevBuf<uint64_t> long_cnt(static_cast<size_t>(n_win + 1), ex.stream);
  long_cnt.zero();
  k_sell_sort<<<static_cast<unsigned>(n_win), kSellSortThreads, 0, ex.stream>>>(
      op.n, op.indptr, L->long_min, L->perm.get(), L->plen.get(), long_tmp.get(), long_cnt.get());
  SI_LAUNCH_CHECK();
  DevBuf<uint64_t> long_ptr(static_cast<size_t>(n_win + 1), ex.stream);
  L->n_long = static_cast<int64_t>(exclusive_scan_u64(ex, long_cnt.get(), long_ptr.get(), n_win));
  L->long_rows.alloc(static_cast<size_t>(std::max<int64_t>(L->n_long, 1)), ex.stream);
  if (L->n_long > 0) {
    const int gl = static_cast<int>(std::max<int64_t>(1, std::min<int64_t>(n_win, int64_t(ex.sms) * 8)));
    k_sell_long_compact<<<gl, 256, 0, ex.stream>>>(n_win, long_tmp.get(), long_ptr.get(), L->long_rows.get());
    SI_LAUNCH_CHECK();
  }
  DevBuf<uint64_t> cnt(static_cast<size_t>(L->n_slices + 1), ex.stream);
  const int g1 = static_cast<int>(std::max<int64_t>(1, std::min<int64_t>((L->n_slices + 256) / 256, int64_t(ex.sms) * 8)));
  k_sell_widths<<<g1, 256, 0, ex.stream>>>(L->n_slices, L->plen.get(), cnt.get());
  SI_LAUNCH_CHECK();
  L->slice_ptr.alloc(static_cast<size_t>(L->n_slices + 1), ex.stream);
  L->slots = exclusive_scan_u64(ex, cnt.get(), L->slice_ptr.get(), L->n_slices);
  // the copy must fit beside the solver's work buffers: at most a quarter of
  // the free memory
  const size_t per_slot = 4 + (op.v32 ? 4 : 0) + (op.v64 ? 8 : 0);
  size_t free_b = 0, total_b = 0;
  SI_CUDA(cudaMemGetInfo(&free_b, &total_b));
  if (L->slots * per_slot > free_b / 4) {
    op.panels->sell_failed = true;
    return nullptr;
  }
  L->idx.alloc(static_cast<size_t>(std::max<uint64_t>(L->slots, 1)), ex.stream);
  if (op.v32) L->v32.alloc(static_cast<size_t>(std::max<uint64_t>(L->slots, 1)), ex.stream);
  if (op.v64) L->v64.alloc(static_cast<size_t>(std::max<uint64_t>(L->slots, 1)), ex.stream);
  const int g2 = static_cast<int>(std::max<int64_t>(1, std::min<int64_t>((L->n_slices + 7) / 8, int64_t(ex.sms) * 16)));
  k_sell_fill<<<g2, 256, 0, ex.stream>>>(L->n_slices, L->slice_ptr.get(), L->perm.get(), L->plen.get(), op.indptr,
                                          op.indices, op.v32, op.v64, L->idx.get(), L->v32.get(), L->v64.get());
  SI_LAUNCH_CHECK();
  op.panels->sell = std::move(L);
  return op.panels->sell.get();
}

template <class XT, int LD>
constexpr int sell_threads() {
  return (LD * sizeof(XT) <= 16) ? 1024 : 512;
}
template <class XT, int LD>
constexpr int sell_unroll() {
  return (LD * sizeof(XT) <= 32) ? 4 : (LD * sizeof(XT) <= 64 ? 2 : 1);
}

template <class VT, class XT, int LD, bool L1, bool PF, bool PIPE>
bool launch_sell(const Exec& ex, const OpDev& op, const VT* vals, const XT* x, XT* y, const Epilogue<XT>& ep,
                 const int* stop) {
  const SellLayout* L = sell_layout(ex, op);
  if (L == nullptr) return false;
  const VT* sval;
  if constexpr (std::is_same<VT, float>::value) {
    if (vals != op.v32) return false;
    sval = L->v32.get();
  } else {
    if (vals != op.v64) return false;
    sval = L->v64.get();
  }
  if (sval == nullptr) return false;
  constexpr int NT = sell_threads<XT, LD>();
  constexpr int U = sell_unroll<XT, LD>();
  static std::atomic<int> resident[128];
  const int dev = (ex.device >= 0 && ex.device < 128) ? ex.device : 0;
  if (resident[dev] == 0) {
    SI_CUDA(cudaFuncSetAttribute(k_spmm_sell<VT, XT, LD, U, NT, L1, PF, PIPE>,
                                 cudaFuncAttributePreferredSharedMemoryCarveout, 0));
    int per_sm = 0;
    SI_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_spmm_sell<VT, XT, LD, U, NT, L1, PF, PIPE>, NT, 0));
    resident[dev] = std::max(per_sm, 1);
  }
  const int grid = static_cast<int>(std::max<int64_t>(1, std::min<int64_t>(L->n_slices, int64_t(ex.sms) * resident[dev])));
  const SellArgs args{L->n_slices, L->n_long, L->slice_ptr.get(), L->perm.get(), L->plen.get(),
                      L->idx.get(), L->long_rows.get(), op.indptr, op.indices};
  k_spmm_sell<VT, XT, LD, U, NT, L1, PF, PIPE><<<grid, NT, 0, ex.stream>>>(args, sval, vals, op.diag, x, y, ep, stop);
  SI_LAUNCH_CHECK();
  return true;
}

// choice < 100: direct kernel with `choice` lanes per row; 100 + g: tiled kernel
template <class VT, class XT, int LD>
void launch_lanes(int g, const Exec& ex, const OpDev& op, const VT* vals, const XT* x, XT* y, const Epilogue<XT>& ep,
                  const int* stop) {
  if (g == 300) {
    if (launch_panel<VT, XT, LD>(ex, op, vals, x, y, ep, stop)) return;
    g = spmm_group_lanes(op);  // no windows (inside a capture before first use): direct kernel
  }
  if (g >= 400 && g <= 403) {
    bool ok = false;
    switch (g) {
      case 400: ok = launch_sell<VT, XT, LD, true, false, false>(ex, op, vals, x, y, ep, stop); break;
      case 401: ok = launch_sell<VT, XT, LD, true, true, false>(ex, op, vals, x, y, ep, stop); break;
      case 402: ok = launch_sell<VT, XT, LD, true, false, true>(ex, op, vals, x, y, ep, stop); break;
      default: ok = launch_sell<VT, XT, LD, true, true, true>(ex, op, vals, x, y, ep, stop); break;
    }
    if (ok) return;
    g = spmm_group_lanes(op);  // no sliced copy: direct kernel
  }
  switch (g) {
    case 4: launch_vec<VT, XT, LD, 4>(ex, op, vals, x, y, ep, stop); break;
    case 8: launch_vec<VT, XT, LD, 8>(ex, op, vals, x, y, ep, stop); break;
    case 16: launch_vec<VT, XT, LD, 16>(ex, op, vals, x, y, ep, stop); break;
    case 104: launch_tiled<VT, XT, LD, 4>(ex, op, vals, x, y, ep, stop); break;
    case 108: launch_tiled<VT, XT, LD, 8>(ex, op, vals, x, y, ep, stop); break;
    case 204:
    case 208:
      if constexpr (std::is_same<VT, float>::value && std::is_same<XT, float>::value && LD == 4) {
        if (g == 204) launch_gather<4>(ex, op, vals, x, y, ep, stop);
        else launch_gather<8>(ex, op, vals, x, y, ep, stop);
      } else {
        launch_vec<VT, XT, LD, 8>(ex, op, vals, x, y, ep, stop);
      }
      break;
    default: launch_vec<VT, XT, LD, 32>(ex, op, vals, x, y, ep, stop); break;
  }
}

// Autotuner: lanes per row for one operator / block width / precision.  The
// first call on a (device, operator, ld, value type, block type) times every
// candidate with CUDA events on the caller's stream (the kernel is
// idempotent: y never aliases its inputs) and caches the fastest; under
// stream capture it uses the cached choice or the degree heuristic.
struct TuneKey {
  int device;
  const void* indptr;
  const void* indices;
  int64_t n, nnz;
  int ld, vbytes, xbytes, tiled, panel, sell;
  bool operator<(const TuneKey& o) const {
    return std::tie(device, indptr, indices, n, nnz, ld, vbytes, xbytes, tiled, panel, sell) <
           std::tie(o.device, o.indptr, o.indices, o.n, o.nnz, o.ld, o.vbytes, o.xbytes, o.tiled, o.panel, o.sell);
  }
};
std::mutex g_tune_mu;
std::map<TuneKey, int> g_tune;
constexpr int64_t kTuneMinNnz = int64_t(1) << 22;  // operators the autotuner times

// Tuning file (SPECTRAL_INIT_SPMM_TUNE_FILE): choices keyed by the operator's
// shape rather than its addresses, one line "n nnz ld vbytes xbytes tiled
// panel sell choice" each.  A present file is read once and its choices are
// used instead of timing; a choice timed by this process is appended.  This
// lets a profiled run replay the kernels a plain run picked (timings taken
// under a profiler are not representative) and later processes skip tuning.
using ShapeKey = std::tuple<int64_t, int64_t, int, int, int, int, int, int>;
ShapeKey shape_key(const TuneKey& k) {
  return ShapeKey{k.n, k.nnz, k.ld, k.vbytes, k.xbytes, k.tiled, k.panel, k.sell};
}
std::map<ShapeKey, int>& tune_file_choices() {  // caller holds g_tune_mu
  static std::map<ShapeKey, int> m;
  static bool loaded = false;
  if (!loaded) {
    loaded = true;
    const char* path = std::getenv("SPECTRAL_INIT_SPMM_TUNE_FILE");
    if (path != nullptr && *path != '\0') {
      if (FILE* f = std::fopen(path, "r")) {
        long long n, nnz;
        int ld, vb, xb, t, p, sl, c;
        while (std::fscanf(f, "%lld %lld %d %d %d %d %d %d %d", &n, &nnz, &ld, &vb, &xb, &t, &p, &sl, &c) == 9)
          m[ShapeKey{n, nnz, ld, vb, xb, t, p, sl}] = c;
        std::fclose(f);
      }
    }
  }
  return m;
}
void tune_file_append(const TuneKey& k, int choice) {  // caller holds g_tune_mu
  const char* path = std::getenv("SPECTRAL_INIT_SPMM_TUNE_FILE");
  if (path == nullptr || *path == '\0') return;
  if (FILE* f = std::fopen(path, "a")) {
    std::fprintf(f, "%lld %lld %d %d %d %d %d %d %d\n", static_cast<long long>(k.n), static_cast<long long>(k.nnz),
                 k.ld, k.vbytes, k.xbytes, k.tiled, k.panel, k.sell, choice);
    std::fclose(f);
  }
  tune_file_choices()[shape_key(k)] = choice;
}

// Kernel override for tuning and tests: SPECTRAL_INIT_SPMM_KERNEL = vec4 | vec8 |
// vec16 | vec32 | tiled4 | tiled8 | gather4 | gather8 | panel | sell | sell_pf | sell_pipe |
// sell_pf_pipe (unset or "auto": the
// autotuner).  A choice the operator or the types cannot use is ignored.
template <class VT, class XT, int LD>
int forced_choice(const OpDev& op, bool tiled) {
  // SPECTRAL_INIT_SPMM_KERNEL_F32 / _F64 override it for one value type
  const char* env = std::getenv(std::is_same<VT, float>::value ? "SPECTRAL_INIT_SPMM_KERNEL_F32"
                                                                : "SPECTRAL_INIT_SPMM_KERNEL_F64");
  if (env == nullptr) env = std::getenv("SPECTRAL_INIT_SPMM_KERNEL");
  if (env == nullptr) return 0;
  const std::string v(env);
  static const std::pair<const char*, int> names[] = {{"vec4", 4},     {"vec8", 8},       {"vec16", 16},
                                                      {"vec32", 32},   {"tiled4", 104},   {"tiled8", 108},
                                                      {"gather4", 204}, {"gather8", 208},
                                                      {"panel", 300},  {"sell", 400},    {"sell_pf", 401},
                                                      {"sell_pipe", 402}, {"sell_pf_pipe", 403}};
  for (const auto& nm : names) {
    if (v != nm.first) continue;
    const int c = nm.second;
    if (c > 100 && c < 200 && !tiled) return 0;
    if (c == 300 && (op.panels == nullptr || op.panels->n_pblocks <= 0)) return 0;
    if (c >= 400 && (op.panels == nullptr || !op.panels->sell_ok)) return 0;
    if (c > 200 && c < 300 && !(std::is_same<VT, float>::value && std::is_same<XT, float>::value && LD == 4 &&
                     op.gather_blocks != nullptr && op.n_gather_blocks > 0))
      return 0;
    return c;
  }
  return 0;
}

template <class VT, class XT, int LD>
void dispatch_g(const Exec& ex, const OpDev& op, const VT* vals, const XT* x, XT* y, const Epilogue<XT>& ep,
                const int* stop) {
  const bool tiled = op.row_blocks != nullptr && op.n_blocks > 0;
  const bool panel = op.panels != nullptr && op.panels->n_pblocks > 0;
  const bool sell = op.panels != nullptr && op.panels->sell_ok;
  const TuneKey key{ex.device, op.indptr, op.indices, op.n, op.nnz, LD, static_cast<int>(sizeof(VT)),
                    static_cast<int>(sizeof(XT)), tiled ? 1 : 0, panel ? 1 : 0, sell ? 1 : 0};
  int g = forced_choice<VT, XT, LD>(op, tiled);
  if (g != 0) {
    launch_lanes<VT, XT, LD>(g, ex, op, vals, x, y, ep, stop);
    return;
  }
  {
    std::lock_guard<std::mutex> lk(g_tune_mu);
    auto it = g_tune.find(key);
    if (it != g_tune.end()) {
      g = it->second;
    } else {
      auto& file = tune_file_choices();
      auto ft = file.find(shape_key(key));
      if (ft != file.end()) {
        g = ft->second;
        g_tune[key] = g;
      }
    }
  }
  if (g == 0) {
    bool timed = false;
    cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
    SI_CUDA(cudaStreamIsCapturing(ex.stream, &cs));
    // below ~4 M stored entries timing the candidates (and building the
    // sliced copy for them) costs more than a better kernel saves over a solve:
    // measured on 502 components of 20 to 100 k nodes, the CSR vector kernel
    // alone finished the workload in 1.17 s, the tuned run in 1.20 / 1.44 s
    const bool tiny = op.n < 20000;
    const bool small = op.nnz < kTuneMinNnz;
    if (cs != cudaStreamCaptureStatusNone || tiny) {
      g = tiled ? 104 : spmm_group_lanes(op);
    } else if (small) {
      g = spmm_group_lanes(op);
    } else {
      timed = true;
      cudaEvent_t e0, e1;
      SI_CUDA(cudaEventCreate(&e0));
      SI_CUDA(cudaEventCreate(&e1));
      float best = 1e30f;
      std::vector<int> cands = {4, 8, 16, 32};
      if (tiled) {
        cands.push_back(104);
        cands.push_back(108);
      }
      if (std::is_same<VT, float>::value && std::is_same<XT, float>::value && LD == 4 &&
          op.gather_blocks != nullptr && op.n_gather_blocks > 0) {
        cands.push_back(204);
        cands.push_back(208);
      }
      if (op.panels != nullptr && op.panels->n_pblocks > 0) cands.push_back(300);
      if (sell)
        for (int c = 400; c <= 403; ++c) cands.push_back(c);
      for (int cand : cands) {
        launch_lanes<VT, XT, LD>(cand, ex, op, vals, x, y, ep, nullptr);
        SI_CUDA(cudaEventRecord(e0, ex.stream));
        for (int r = 0; r < 3; ++r) launch_lanes<VT, XT, LD>(cand, ex, op, vals, x, y, ep, nullptr);
        SI_CUDA(cudaEventRecord(e1, ex.stream));
        SI_CUDA(cudaEventSynchronize(e1));
        float ms = 0.f;
        SI_CUDA(cudaEventElapsedTime(&ms, e0, e1));
        if (ms < best) {
          best = ms;
          g = cand;
        }
      }
      cudaEventDestroy(e0);
      cudaEventDestroy(e1);
    }
    std::lock_guard<std::mutex> lk(g_tune_mu);
    g_tune[key] = g;
    if (timed) tune_file_append(key, g);
  }
  launch_lanes<VT, XT, LD>(g, ex, op, vals, x, y, ep, stop);
}

template <class VT, class XT>
void dispatch(const Exec& ex, const OpDev& op, const VT* vals, const XT* x, XT* y, int ld, int k,
              const Epilogue<XT>& ep, const int* stop) {
  // vector gathers need the row start aligned to the vector width (32 B for
  // f64 and for 8-wide f32, 16 B for 4-wide f32); otherwise use the generic path
  const uintptr_t a = reinterpret_cast<uintptr_t>(x);
  const bool aligned = (sizeof(XT) == 4 && ld == 4) ? (a % 16 == 0) : (a % 32 == 0);
  if (aligned && ld == 4) return dispatch_g<VT, XT, 4>(ex, op, vals, x, y, ep, stop);
  if (aligned && ld == 8) return dispatch_g<VT, XT, 8>(ex, op, vals, x, y, ep, stop);
  if (aligned && ld == 16) return dispatch_g<VT, XT, 16>(ex, op, vals, x, y, ep, stop);
  switch (spmm_group_lanes(op)) {
    case 4: return launch_generic<VT, XT, 4>(ex, op, vals, x, y, ld, k, ep, stop);
    case 8: return launch_generic<VT, XT, 8>(ex, op, vals, x, y, ld, k, ep, stop);
    case 16: return launch_generic<VT, XT, 16>(ex, op, vals, x, y, ld, k, ep, stop);
    default: return launch_generic<VT, XT, 32>(ex, op, vals, x, y, ld, k, ep, stop);
  }
}

}  // namespace

void make_row_blocks(const Exec& ex, const OpDev& op, RowBlocks& rb) {
  auto build = [&](int64_t per, int64_t& nb, DevBuf<int64_t>& starts, DevBuf<uint64_t>& ptrs) {
    nb = std::max<int64_t>(1, (op.nnz + per - 1) / per);
    starts.alloc(nb + 1, ex.stream);
    const int grid = static_cast<int>(std::min<int64_t>((nb + 256) / 256, int64_t(ex.sms) * 8));
    k_row_blocks<<<std::max(grid, 1), 256, 0, ex.stream>>>(op.n, op.indptr, nb, per, starts.get());
    SI_LAUNCH_CHECK();
    ptrs.alloc(nb + 1, ex.stream);
    k_block_ptrs<<<std::max(grid, 1), 256, 0, ex.stream>>>(nb, starts.get(), op.indptr, ptrs.get());
    SI_LAUNCH_CHECK();
  };
  build(kSpmmBlockNnz, rb.n_blocks, rb.starts, rb.ptrs);
  build(kGatherBlockNnz, rb.n_gblocks, rb.gstarts, rb.gptrs);
  build(kPanelBlockNnz, rb.n_pblocks, rb.pstarts, rb.pptrs);
  rb.windows.clear();
  rb.sell.reset();
  rb.sell_failed = false;
}

int spmm_group_lanes(const OpDev& op) {
  // a lane covers up to 8 entries per pass: fewest lanes that keep most rows
  // to one pass (more rows in flight per SM beats wider groups)
  const double mean = op.n > 0 ? static_cast<double>(op.nnz) / static_cast<double>(op.n) : 0.0;
  if (mean <= 28.0) return 4;
  if (mean <= 56.0) return 8;
  if (mean <= 112.0) return 16;
  return 32;
}

template <class XT>
void spmm_dev(const Exec& ex, const OpDev& op, const XT* x, XT* y, int ld, int k, const Epilogue<XT>& ep,
              const int* stop, bool use_f32_values) {
  if (op.n == 0) return;
  SI_REQUIRE(k >= 1 && k <= ld, SI_INVALID_ARGUMENT, "spmm: need 1 <= k <= ld");
  SI_REQUIRE(x != y, SI_INVALID_ARGUMENT, "spmm: x and y must not alias");
  if (use_f32_values) {
    SI_REQUIRE(op.v32 != nullptr, SI_INVALID_ARGUMENT, "spmm: f32 values requested but absent");
    dispatch<float, XT>(ex, op, op.v32, x, y, ld, k, ep, stop);
  } else {
    SI_REQUIRE(op.v64 != nullptr, SI_INVALID_ARGUMENT, "spmm: f64 values absent");
    dispatch<double, XT>(ex, op, op.v64, x, y, ld, k, ep, stop);
  }
}

template void spmm_dev<double>(const Exec&, const OpDev&, const double*, double*, int, int,
                               const Epilogue<double>&, const int*, bool);
template void spmm_dev<float>(const Exec&, const OpDev&, const float*, float*, int, int,
                              const Epilogue<float>&, const int*, bool);

}  // namespace si
