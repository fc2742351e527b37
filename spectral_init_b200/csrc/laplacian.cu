// Graph preparation on the device: CSR validation, degrees (compute_degrees,
// src/laplacian.rs:29-49) and the normalised Laplacian
// (build_normalized_laplacian, src/laplacian.rs:60-88).
//
// Degrees, PythonCompat: the crate scatters deg[col] += w in f32 in CSR order
// (src/laplacian.rs:8-16), i.e. column j sums its entries in increasing row
// order.  For a symmetric graph with sorted rows that is exactly the
// sequential f32 sum of row j in increasing column order, so one thread per
// row reproduces the bits without atomics.  Non-symmetric input takes a
// stable radix sort by column and then the same sequential per-column sum.
// RustNative: sequential f64 sum of each row.
//
// Laplacian values are evaluated as ((-inv_i) * w_ij) * inv_j in f64 -- the
// crate's expression and association -- so they match it bit for bit.
#include <cub/cub.cuh>

#include "si_internal.h"

namespace si {
namespace {

enum : unsigned {
  ERR_ENDS = 1u,        // indptr[0] != 0 or indptr[n] != nnz
  ERR_MONOTONE = 2u,    // indptr decreasing or past nnz
  ERR_RANGE = 4u,       // column index >= n
  ERR_ORDER = 8u,       // columns not strictly increasing within a row
  ERR_NONFINITE = 16u,  // NaN / Inf weight
};

__global__ void k_validate(int64_t n, int64_t nnz, const uint64_t* __restrict__ indptr,
                           const uint32_t* __restrict__ indices, const float* __restrict__ data,
                           unsigned* err) {
  const int64_t stride = static_cast<int64_t>(gridDim.x) * blockDim.x;
  unsigned local = 0;
  for (int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; i < n; i += stride) {
    const uint64_t s = indptr[i], e = indptr[i + 1];
    if (e < s || e > static_cast<uint64_t>(nnz)) {
      local |= ERR_MONOTONE;
      continue;
    }
    int64_t prev = -1;
    for (uint64_t k = s; k < e; ++k) {
      const uint32_t c = indices[k];
      if (c >= static_cast<uint64_t>(n)) {
        local |= ERR_RANGE;
        break;
      }
      if (static_cast<int64_t>(c) <= prev) local |= ERR_ORDER;
      prev = c;
      if (data != nullptr && !isfinite(data[k])) local |= ERR_NONFINITE;
    }
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    if (indptr[0] != 0 || indptr[n] != static_cast<uint64_t>(nnz)) local |= ERR_ENDS;
  }
  if (local) atomicOr(err, local);
}

// For every stored (i, j, w): is (j, i) stored with the same bits?
__global__ void k_symmetric(int64_t n, const uint64_t* __restrict__ indptr, const uint32_t* __restrict__ indices,
                            const float* __restrict__ data, unsigned* asym) {
  const int64_t stride = static_cast<int64_t>(gridDim.x) * blockDim.x;
  for (int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; i < n; i += stride) {
    const uint64_t s = indptr[i], e = indptr[i + 1];
    for (uint64_t k = s; k < e; ++k) {
      const uint32_t j = indices[k];
      uint64_t lo = indptr[j], hi = indptr[j + 1];
      bool found = false;
      while (lo < hi) {
        const uint64_t mid = lo + (hi - lo) / 2;
        const uint32_t c = indices[mid];
        if (c == static_cast<uint32_t>(i)) {
          found = __float_as_uint(data[mid]) == __float_as_uint(data[k]);
          break;
        }
        if (c < static_cast<uint32_t>(i)) lo = mid + 1; else hi = mid;
      }
      if (!found) {
        atomicOr(asym, 1u);
        return;
      }
    }
  }
}

// Sequential f32 sum of each row (== the crate's column scatter for symmetric graphs).
__global__ void k_rowsum_f32_seq(int64_t n, const uint64_t* __restrict__ indptr, const float* __restrict__ data,
                                 double* __restrict__ deg, double* __restrict__ sqrt_deg) {
  const int64_t stride = static_cast<int64_t>(gridDim.x) * blockDim.x;
  for (int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; i < n; i += stride) {
    float s = 0.0f;
    for (uint64_t k = indptr[i]; k < indptr[i + 1]; ++k) s = __fadd_rn(s, data[k]);
    const double d = static_cast<double>(s);
    deg[i] = d;
    sqrt_deg[i] = sqrt(d);
  }
}

// Sequential f64 sum of each row (RustNative).
__global__ void k_rowsum_f64_seq(int64_t n, const uint64_t* __restrict__ indptr, const float* __restrict__ data,
                                 double* __restrict__ deg, double* __restrict__ sqrt_deg) {
  const int64_t stride = static_cast<int64_t>(gridDim.x) * blockDim.x;
  for (int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; i < n; i += stride) {
    double s = 0.0;
    for (uint64_t k = indptr[i]; k < indptr[i + 1]; ++k) s = __dadd_rn(s, static_cast<double>(data[k]));
    deg[i] = s;
    sqrt_deg[i] = sqrt(s);
  }
}

__global__ void k_iota_u32(int64_t nnz, uint32_t* out) {
  const int64_t stride = static_cast<int64_t>(gridDim.x) * blockDim.x;
  for (int64_t k = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; k < nnz; k += stride)
    out[k] = static_cast<uint32_t>(k);
}

__global__ void k_col_counts(int64_t nnz, const uint32_t* __restrict__ indices, uint64_t* counts) {
  const int64_t stride = static_cast<int64_t>(gridDim.x) * blockDim.x;
  for (int64_t k = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; k < nnz; k += stride)
    atomicAdd(reinterpret_cast<unsigned long long*>(counts + indices[k]), 1ull);
}

// Column sums over entries sorted stably by column (original order kept).
__global__ void k_colsum_sorted(int64_t n, const uint64_t* __restrict__ colptr, const uint32_t* __restrict__ perm,
                                const float* __restrict__ data, double* __restrict__ deg,
                                double* __restrict__ sqrt_deg) {
  const int64_t stride = static_cast<int64_t>(gridDim.x) * blockDim.x;
  for (int64_t j = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; j < n; j += stride) {
    float s = 0.0f;
    for (uint64_t q = colptr[j]; q < colptr[j + 1]; ++q) s = __fadd_rn(s, data[perm[q]]);
    deg[j] = static_cast<double>(s);
    sqrt_deg[j] = sqrt(static_cast<double>(s));
  }
}

__global__ void k_inv_sqrt(int64_t n, const double* __restrict__ sq, double* __restrict__ inv) {
  const int64_t stride = static_cast<int64_t>(gridDim.x) * blockDim.x;
  for (int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; i < n; i += stride) {
    const double s = sq[i];
    inv[i] = s > 0.0 ? 1.0 / s : 0.0;
  }
}

// 8 lanes per row: values[e] = ((-inv_i) * w_e) * inv_j, 0 on the diagonal.
__global__ void k_lap_values(int64_t n, const uint64_t* __restrict__ indptr, const uint32_t* __restrict__ indices,
                             const float* __restrict__ data, const double* __restrict__ inv,
                             double* __restrict__ v64, float* __restrict__ v32) {
  const int sub = threadIdx.x & 7;
  const int64_t groups = static_cast<int64_t>(gridDim.x) * blockDim.x / 8;
  for (int64_t i = (blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x) / 8; i < n; i += groups) {
    const double ni = -inv[i];
    for (uint64_t k = indptr[i] + sub; k < indptr[i + 1]; k += 8) {
      const uint32_t j = indices[k];
      const double v = (j == static_cast<uint32_t>(i)) ? 0.0 : __dmul_rn(__dmul_rn(ni, static_cast<double>(data[k])), inv[j]);
      v64[k] = v;
      if (v32) v32[k] = static_cast<float>(v);
    }
  }
}

// entries per row of the explicit Laplacian: off-diagonal entries + 1
__global__ void k_lap_counts(int64_t n, const uint64_t* __restrict__ indptr, const uint32_t* __restrict__ indices,
                             uint64_t* __restrict__ counts) {
  const int64_t stride = static_cast<int64_t>(gridDim.x) * blockDim.x;
  for (int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; i < n; i += stride) {
    uint64_t c = 1;
    for (uint64_t k = indptr[i]; k < indptr[i + 1]; ++k) c += (indices[k] != static_cast<uint32_t>(i));
    counts[i] = c;
  }
}

__global__ void k_lap_fill(int64_t n, const uint64_t* __restrict__ indptr, const uint32_t* __restrict__ indices,
                           const float* __restrict__ data, const double* __restrict__ inv,
                           const uint64_t* __restrict__ out_ptr, uint32_t* __restrict__ out_idx,
                           double* __restrict__ out_val) {
  const int64_t stride = static_cast<int64_t>(gridDim.x) * blockDim.x;
  for (int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; i < n; i += stride) {
    uint64_t o = out_ptr[i];
    bool diag_done = false;
    const double ni = -inv[i];
    for (uint64_t k = indptr[i]; k < indptr[i + 1]; ++k) {
      const uint32_t j = indices[k];
      if (j == static_cast<uint32_t>(i)) continue;
      if (!diag_done && j > static_cast<uint32_t>(i)) {
        out_idx[o] = static_cast<uint32_t>(i);
        out_val[o] = 1.0;
        ++o;
        diag_done = true;
      }
      out_idx[o] = j;
      out_val[o] = __dmul_rn(__dmul_rn(ni, static_cast<double>(data[k])), inv[j]);
      ++o;
    }
    if (!diag_done) {
      out_idx[o] = static_cast<uint32_t>(i);
      out_val[o] = 1.0;
    }
  }
}

int grid_for(const Exec& ex, int64_t items, int threads = 256) {
  const int64_t need = (items + threads - 1) / threads;
  return static_cast<int>(std::max<int64_t>(1, std::min<int64_t>(need, int64_t(ex.sms) * 16)));
}

}  // namespace

uint64_t exclusive_scan_u64(const Exec& ex, const uint64_t* in, uint64_t* out, int64_t n) {
  // out has n + 1 entries; out[n] = total
  size_t tmp_bytes = 0;
  SI_CUDA(cub::DeviceScan::ExclusiveSum(nullptr, tmp_bytes, in, out, n + 1, ex.stream));
  DevBuf<unsigned char> tmp(tmp_bytes, ex.stream);
  SI_CUDA(cub::DeviceScan::ExclusiveSum(tmp.get(), tmp_bytes, in, out, n + 1, ex.stream));
  uint64_t total = 0;
  SI_CUDA(cudaMemcpyAsync(&total, out + n, sizeof(uint64_t), cudaMemcpyDeviceToHost, ex.stream));
  SI_CUDA(cudaStreamSynchronize(ex.stream));
  return total;
}

void validate_graph(const Exec& ex, const GraphDev& g) {
  SI_REQUIRE(g.n >= 0 && g.nnz >= 0, SI_INVALID_GRAPH, "invalid graph: negative size");
  SI_REQUIRE(g.n < (int64_t(1) << 32), SI_INVALID_GRAPH, "invalid graph: more than 2^32-1 rows");
  SI_REQUIRE(g.indptr != nullptr, SI_INVALID_ARGUMENT, "graph indptr is null");
  // data may be null for structure-only validation (f64 matrices carry their own values)
  SI_REQUIRE(g.nnz == 0 || g.indices != nullptr, SI_INVALID_ARGUMENT, "graph indices are null");
  DevBuf<unsigned> err(1, ex.stream);
  err.zero();
  k_validate<<<grid_for(ex, std::max<int64_t>(g.n, 1)), 256, 0, ex.stream>>>(g.n, g.nnz, g.indptr, g.indices,
                                                                             g.data, err.get());
  SI_LAUNCH_CHECK();
  unsigned h = 0;
  SI_CUDA(cudaMemcpyAsync(&h, err.get(), sizeof(unsigned), cudaMemcpyDeviceToHost, ex.stream));
  SI_CUDA(cudaStreamSynchronize(ex.stream));
  if (h & ERR_ENDS) throw Error(SI_INVALID_GRAPH, "invalid graph: indptr[0] != 0 or indptr[n] != nnz");
  if (h & ERR_MONOTONE) throw Error(SI_INVALID_GRAPH, "invalid graph: indptr is not monotone");
  if (h & ERR_RANGE) throw Error(SI_INVALID_GRAPH, "invalid graph: column index out of range");
  if (h & ERR_ORDER) throw Error(SI_INVALID_GRAPH, "invalid graph: column indices not sorted/unique within a row");
  if (h & ERR_NONFINITE) throw Error(SI_INVALID_GRAPH, "invalid graph: non-finite weight");
}

bool graph_is_symmetric(const Exec& ex, const GraphDev& g) {
  if (g.n == 0) return true;
  DevBuf<unsigned> flag(1, ex.stream);
  flag.zero();
  k_symmetric<<<grid_for(ex, g.n), 256, 0, ex.stream>>>(g.n, g.indptr, g.indices, g.data, flag.get());
  SI_LAUNCH_CHECK();
  unsigned h = 0;
  SI_CUDA(cudaMemcpyAsync(&h, flag.get(), sizeof(unsigned), cudaMemcpyDeviceToHost, ex.stream));
  SI_CUDA(cudaStreamSynchronize(ex.stream));
  return h == 0;
}

void compute_degrees_dev(const Exec& ex, const GraphDev& g, int mode, double* deg, double* sqrt_deg) {
  if (g.n == 0) return;
  if (mode == SI_COMPUTE_RUST_NATIVE) {
    k_rowsum_f64_seq<<<grid_for(ex, g.n), 256, 0, ex.stream>>>(g.n, g.indptr, g.data, deg, sqrt_deg);
    SI_LAUNCH_CHECK();
    return;
  }
  if (graph_is_symmetric(ex, g)) {
    k_rowsum_f32_seq<<<grid_for(ex, g.n), 256, 0, ex.stream>>>(g.n, g.indptr, g.data, deg, sqrt_deg);
    SI_LAUNCH_CHECK();
    return;
  }
  // general graph: stable sort of entry ids by column, then per-column sums
  const int64_t nnz = g.nnz;
  DevBuf<uint32_t> ids(std::max<int64_t>(nnz, 1), ex.stream), ids_sorted(std::max<int64_t>(nnz, 1), ex.stream);
  DevBuf<uint32_t> keys_sorted(std::max<int64_t>(nnz, 1), ex.stream);
  DevBuf<uint64_t> counts(g.n + 1, ex.stream), colptr(g.n + 1, ex.stream);
  counts.zero();
  if (nnz > 0) {
    k_iota_u32<<<grid_for(ex, nnz), 256, 0, ex.stream>>>(nnz, ids.get());
    SI_LAUNCH_CHECK();
    size_t tmp_bytes = 0;
    int end_bit = 1;
    while (end_bit < 32 && (int64_t(1) << end_bit) < g.n) ++end_bit;
    SI_CUDA(cub::DeviceRadixSort::SortPairs(nullptr, tmp_bytes, g.indices, keys_sorted.get(), ids.get(),
                                            ids_sorted.get(), nnz, 0, end_bit, ex.stream));
    DevBuf<unsigned char> tmp(tmp_bytes, ex.stream);
    SI_CUDA(cub::DeviceRadixSort::SortPairs(tmp.get(), tmp_bytes, g.indices, keys_sorted.get(), ids.get(),
                                            ids_sorted.get(), nnz, 0, end_bit, ex.stream));
    k_col_counts<<<grid_for(ex, nnz), 256, 0, ex.stream>>>(nnz, g.indices, counts.get());
    SI_LAUNCH_CHECK();
  }
  exclusive_scan_u64(ex, counts.get(), colptr.get(), g.n);
  k_colsum_sorted<<<grid_for(ex, g.n), 256, 0, ex.stream>>>(g.n, colptr.get(), ids_sorted.get(), g.data, deg,
                                                            sqrt_deg);
  SI_LAUNCH_CHECK();
}

void inv_sqrt_dev(const Exec& ex, const double* sqrt_deg, int64_t n, double* inv) {
  if (n == 0) return;
  k_inv_sqrt<<<grid_for(ex, n), 256, 0, ex.stream>>>(n, sqrt_deg, inv);
  SI_LAUNCH_CHECK();
}

void laplacian_values_dev(const Exec& ex, const GraphDev& g, const double* inv_sqrt_deg, double* v64,
                          float* v32) {
  if (g.n == 0 || g.nnz == 0) return;
  k_lap_values<<<grid_for(ex, g.n * 8), 256, 0, ex.stream>>>(g.n, g.indptr, g.indices, g.data, inv_sqrt_deg,
                                                              v64, v32);
  SI_LAUNCH_CHECK();
}

uint64_t laplacian_csr_nnz_dev(const Exec& ex, const GraphDev& g) {
  if (g.n == 0) return 0;
  DevBuf<uint64_t> counts(g.n + 1, ex.stream), ptr(g.n + 1, ex.stream);
  counts.zero();
  k_lap_counts<<<grid_for(ex, g.n), 256, 0, ex.stream>>>(g.n, g.indptr, g.indices, counts.get());
  SI_LAUNCH_CHECK();
  return exclusive_scan_u64(ex, counts.get(), ptr.get(), g.n);
}

void laplacian_csr_dev(const Exec& ex, const GraphDev& g, const double* inv_sqrt_deg, uint64_t* out_indptr,
                       uint32_t* out_indices, double* out_data) {
  if (g.n == 0) {
    SI_CUDA(cudaMemsetAsync(out_indptr, 0, sizeof(uint64_t), ex.stream));
    return;
  }
  DevBuf<uint64_t> counts(g.n + 1, ex.stream);
  counts.zero();
  k_lap_counts<<<grid_for(ex, g.n), 256, 0, ex.stream>>>(g.n, g.indptr, g.indices, counts.get());
  SI_LAUNCH_CHECK();
  exclusive_scan_u64(ex, counts.get(), out_indptr, g.n);
  k_lap_fill<<<grid_for(ex, g.n), 256, 0, ex.stream>>>(g.n, g.indptr, g.indices, g.data, inv_sqrt_deg, out_indptr,
                                                       out_indices, out_data);
  SI_LAUNCH_CHECK();
}

OpDev op_from_csr64(const uint64_t* indptr, const uint32_t* indices, const double* data, int64_t n, int64_t nnz) {
  OpDev op;
  op.n = n;
  op.nnz = nnz;
  op.indptr = indptr;
  op.indices = indices;
  op.v64 = data;
  op.v32 = nullptr;
  op.diag = 0.0;
  return op;
}

}  // namespace si
