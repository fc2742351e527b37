// Connected components on the device (find_components, src/components.rs:7-44).
//
// Lock-free union-find: every edge hooks the larger of its two roots under
// the smaller one with atomicCAS, so parent[x] <= x always holds and the final
// root of a component is its smallest node.  Numbering components by the rank
// of their root therefore reproduces the crate's BFS labels (components are
// numbered in the order of their smallest node) for symmetric graphs.  Every
// loop is bounded: a failed CAS means some root was hooked to a strictly
// smaller node, and root chains only shrink.
#include <cub/cub.cuh>

#include "si_internal.h"

namespace si {
namespace {

__device__ __forceinline__ uint32_t find_root(uint32_t* parent, uint32_t x) {
  // path halving; parents only ever decrease, so the benign races are safe
  for (int guard = 0; guard < (1 << 30); ++guard) {
    const uint32_t p = parent[x];
    if (p == x) return x;
    const uint32_t gp = parent[p];
    if (gp != p) parent[x] = gp;
    x = gp;
  }
  return x;
}

__global__ void k_init_parent(int64_t n, uint32_t* parent) {
  const int64_t stride = static_cast<int64_t>(gridDim.x) * blockDim.x;
  for (int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; i < n; i += stride)
    parent[i] = static_cast<uint32_t>(i);
}

// One thread per row; hooks every edge (i, j).
__global__ void k_hook(int64_t n, const uint64_t* __restrict__ indptr, const uint32_t* __restrict__ indices,
                       uint32_t* parent) {
  const int64_t stride = static_cast<int64_t>(gridDim.x) * blockDim.x;
  for (int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; i < n; i += stride) {
    for (uint64_t k = indptr[i]; k < indptr[i + 1]; ++k) {
      const uint32_t j = indices[k];
      if (j == static_cast<uint32_t>(i)) continue;
      uint32_t ri = find_root(parent, static_cast<uint32_t>(i));
      uint32_t rj = find_root(parent, j);
      for (int guard = 0; guard < (1 << 30) && ri != rj; ++guard) {
        const uint32_t hi = ri > rj ? ri : rj;
        const uint32_t lo = ri > rj ? rj : ri;
        const uint32_t old = atomicCAS(parent + hi, hi, lo);
        if (old == hi) break;
        ri = find_root(parent, old);
        rj = find_root(parent, lo);
      }
    }
  }
}

__global__ void k_compress(int64_t n, uint32_t* parent, uint32_t* is_root) {
  const int64_t stride = static_cast<int64_t>(gridDim.x) * blockDim.x;
  for (int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; i < n; i += stride) {
    const uint32_t r = find_root(parent, static_cast<uint32_t>(i));
    parent[i] = r;
    is_root[i] = (r == static_cast<uint32_t>(i)) ? 1u : 0u;
  }
}

__global__ void k_label(int64_t n, const uint32_t* __restrict__ parent, const uint32_t* __restrict__ rank,
                        uint32_t* __restrict__ labels) {
  const int64_t stride = static_cast<int64_t>(gridDim.x) * blockDim.x;
  for (int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; i < n; i += stride)
    labels[i] = rank[parent[i]];
}

}  // namespace

int64_t find_components_dev(const Exec& ex, const GraphDev& g, uint32_t* labels) {
  if (g.n == 0) return 0;
  const int threads = 256;
  const int grid = static_cast<int>(std::max<int64_t>(1, std::min<int64_t>((g.n + threads - 1) / threads,
                                                                           int64_t(ex.sms) * 16)));
  DevBuf<uint32_t> parent(g.n, ex.stream), is_root(g.n + 1, ex.stream), rank(g.n + 1, ex.stream);
  k_init_parent<<<grid, threads, 0, ex.stream>>>(g.n, parent.get());
  SI_LAUNCH_CHECK();
  k_hook<<<grid, threads, 0, ex.stream>>>(g.n, g.indptr, g.indices, parent.get());
  SI_LAUNCH_CHECK();
  SI_CUDA(cudaMemsetAsync(is_root.get() + g.n, 0, sizeof(uint32_t), ex.stream));
  k_compress<<<grid, threads, 0, ex.stream>>>(g.n, parent.get(), is_root.get());
  SI_LAUNCH_CHECK();
  size_t tmp_bytes = 0;
  SI_CUDA(cub::DeviceScan::ExclusiveSum(nullptr, tmp_bytes, is_root.get(), rank.get(), g.n + 1, ex.stream));
  DevBuf<unsigned char> tmp(tmp_bytes, ex.stream);
  SI_CUDA(cub::DeviceScan::ExclusiveSum(tmp.get(), tmp_bytes, is_root.get(), rank.get(), g.n + 1, ex.stream));
  k_label<<<grid, threads, 0, ex.stream>>>(g.n, parent.get(), rank.get(), labels);
  SI_LAUNCH_CHECK();
  uint32_t total = 0;
  SI_CUDA(cudaMemcpyAsync(&total, rank.get() + g.n, sizeof(uint32_t), cudaMemcpyDeviceToHost, ex.stream));
  SI_CUDA(cudaStreamSynchronize(ex.stream));
  return static_cast<int64_t>(total);
}

}  // namespace si
