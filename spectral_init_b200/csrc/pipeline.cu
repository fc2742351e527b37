// The spectral_init pipeline on the device (src/lib.rs:198-258) and the
// multi-component layout (src/multi_component.rs:16-312).
//
// Disconnected graphs: nodes are ordered by (component label, node id) with a
// stable radix sort, which lays the graph out block-diagonally; every
// component is then a view into one permuted CSR (its rows are contiguous,
// its column indices are rewritten to component-local ids), so no per-
// component allocation or host copy of the graph is needed.
#include <cub/cub.cuh>

#include <algorithm>
#include <atomic>
#include <exception>
#include <mutex>
#include <thread>
#include <cfloat>
#include <cmath>
#include <numeric>
#include <vector>

#include "pipeline.h"

namespace si {
namespace {

constexpr int kComponentWorkers = 16;  // host threads (one stream each) solving components

__global__ void k_iota_u32p(int64_t n, uint32_t* out) {
  const int64_t stride = static_cast<int64_t>(gridDim.x) * blockDim.x;
  for (int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; i < n; i += stride)
    out[i] = static_cast<uint32_t>(i);
}

// pos[perm[p]] = p
__global__ void k_inverse_perm(int64_t n, const uint32_t* __restrict__ perm, uint32_t* __restrict__ pos) {
  const int64_t stride = static_cast<int64_t>(gridDim.x) * blockDim.x;
  for (int64_t p = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; p < n; p += stride) pos[perm[p]] = static_cast<uint32_t>(p);
}

// entries kept in permuted row p: neighbours in the same component
__global__ void k_perm_counts(int64_t n, const uint32_t* __restrict__ perm, const uint64_t* __restrict__ indptr,
                              const uint32_t* __restrict__ indices, const uint32_t* __restrict__ labels,
                              uint64_t* __restrict__ counts) {
  const int64_t stride = static_cast<int64_t>(gridDim.x) * blockDim.x;
  for (int64_t p = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; p < n; p += stride) {
    const uint32_t u = perm[p];
    const uint32_t lu = labels[u];
    uint64_t c = 0;
    for (uint64_t k = indptr[u]; k < indptr[u + 1]; ++k) c += (labels[indices[k]] == lu);
    counts[p] = c;
  }
}

__global__ void k_perm_fill(int64_t n, const uint32_t* __restrict__ perm, const uint32_t* __restrict__ pos,
                            const uint64_t* __restrict__ indptr, const uint32_t* __restrict__ indices,
                            const float* __restrict__ data, const uint32_t* __restrict__ labels,
                            const uint64_t* __restrict__ comp_off, const uint64_t* __restrict__ out_ptr,
                            uint32_t* __restrict__ out_idx, float* __restrict__ out_val) {
  const int64_t stride = static_cast<int64_t>(gridDim.x) * blockDim.x;
  for (int64_t p = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; p < n; p += stride) {
    const uint32_t u = perm[p];
    const uint32_t lu = labels[u];
    const uint64_t base = comp_off[lu];
    uint64_t o = out_ptr[p];
    for (uint64_t k = indptr[u]; k < indptr[u + 1]; ++k) {
      const uint32_t v = indices[k];
      if (labels[v] != lu) continue;
      out_idx[o] = static_cast<uint32_t>(pos[v] - base);
      out_val[o] = data[k];
      ++o;
    }
  }
}

// dst[i] = src[i] - base for i <= n (component-relative row pointers)
__global__ void k_rebase(int64_t n, const uint64_t* __restrict__ src, uint64_t base, uint64_t* __restrict__ dst) {
  const int64_t stride = static_cast<int64_t>(gridDim.x) * blockDim.x;
  for (int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; i <= n; i += stride)
    dst[i] = src[i] - base;
}

__global__ void k_label_counts(int64_t n, const uint32_t* __restrict__ labels, uint64_t* __restrict__ counts) {
  const int64_t stride = static_cast<int64_t>(gridDim.x) * blockDim.x;
  for (int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; i < n; i += stride)
    atomicAdd(reinterpret_cast<unsigned long long*>(counts + labels[i]), 1ull);
}

// result[perm[off + r], :] = coords[r, :] * s + meta
__global__ void k_place(int64_t sz, int64_t off, const uint32_t* __restrict__ perm, const double* __restrict__ coords,
                        int k, double s, const double* __restrict__ meta, double* __restrict__ result) {
  const int64_t total = sz * k;
  const int64_t stride = static_cast<int64_t>(gridDim.x) * blockDim.x;
  for (int64_t e = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; e < total; e += stride) {
    const int64_t r = e / k;
    const int c = static_cast<int>(e % k);
    const double v = coords != nullptr ? coords[r * k + c] * s : 0.0;
    result[static_cast<int64_t>(perm[off + r]) * k + c] = v + meta[c];
  }
}

// centroid sums: cent[label[i], f] += data[i, f]  (f64)
__global__ void k_centroid_sums(int64_t n, int nf, const float* __restrict__ data, const uint32_t* __restrict__ labels,
                                double* __restrict__ cent) {
  const int64_t total = n * nf;
  const int64_t stride = static_cast<int64_t>(gridDim.x) * blockDim.x;
  for (int64_t e = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; e < total; e += stride) {
    const int64_t i = e / nf;
    const int f = static_cast<int>(e % nf);
    atomicAdd(cent + static_cast<int64_t>(labels[i]) * nf + f, static_cast<double>(data[e]));
  }
}

// ---- meta-embedding on the device (src/multi_component.rs:143-255) -----------
// Every kernel below sums in the order of the crate's loops (features, then
// columns ascending), one thread per output, so the result does not depend on
// the launch shape.

// cent[c, :] /= size_c (the centroid means; empty components stay zero)
__global__ void k_centroid_mean(int64_t ncomp, int nf, const uint64_t* __restrict__ comp_off,
                                double* __restrict__ cent) {
  const int64_t total = ncomp * nf;
  const int64_t stride = static_cast<int64_t>(gridDim.x) * blockDim.x;
  for (int64_t e = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; e < total; e += stride) {
    const int64_t c = e / nf;
    const uint64_t sz = comp_off[c + 1] - comp_off[c];
    if (sz != 0) cent[e] *= 1.0 / static_cast<double>(sz);
  }
}

// aff[i, j] = exp(-||cent_i - cent_j||^2)
__global__ void k_meta_affinity(int64_t ncomp, int nf, const double* __restrict__ cent, double* __restrict__ aff) {
  const int64_t total = ncomp * ncomp;
  const int64_t stride = static_cast<int64_t>(gridDim.x) * blockDim.x;
  for (int64_t e = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; e < total; e += stride) {
    const int64_t i = e / ncomp, j = e % ncomp;
    double d2 = 0.0;
    for (int f = 0; f < nf; ++f) {
      const double dd = cent[i * nf + f] - cent[j * nf + f];
      d2 += dd * dd;
    }
    aff[e] = exp(-d2);
  }
}

// degree of row i without the self affinity: inv_sqrt = d^-1/2 (0 for an
// isolated centroid), sqrt_deg = d^1/2
__global__ void k_meta_degrees(int64_t ncomp, const double* __restrict__ aff, double* __restrict__ inv_sqrt,
                               double* __restrict__ sqrt_deg) {
  const int64_t stride = static_cast<int64_t>(gridDim.x) * blockDim.x;
  for (int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; i < ncomp; i += stride) {
    double s = 0.0;
    for (int64_t j = 0; j < ncomp; ++j)
      if (j != i) s += aff[i * ncomp + j];
    inv_sqrt[i] = s > 0.0 ? 1.0 / sqrt(s) : 0.0;
    sqrt_deg[i] = sqrt(s);
  }
}

// the normalised Laplacian I - D^-1/2 W D^-1/2 as a CSR with every entry of
// each row stored (row i at [i * ncomp, (i + 1) * ncomp))
__global__ void k_meta_laplacian(int64_t ncomp, const double* __restrict__ aff, const double* __restrict__ inv_sqrt,
                                 uint64_t* __restrict__ indptr, uint32_t* __restrict__ indices,
                                 double* __restrict__ values) {
  const int64_t total = ncomp * ncomp;
  const int64_t stride = static_cast<int64_t>(gridDim.x) * blockDim.x;
  for (int64_t e = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; e <= total; e += stride) {
    if (e % ncomp == 0) indptr[e / ncomp] = static_cast<uint64_t>(e);
    if (e == total) continue;
    const int64_t i = e / ncomp, j = e % ncomp;
    indices[e] = static_cast<uint32_t>(j);
    values[e] = (i == j) ? 1.0 : -inv_sqrt[i] * aff[e] * inv_sqrt[j];
  }
}

// meta[i, d] = vecs[i, sel[d]] (the selected eigenvectors, row-major [ncomp x k])
__global__ void k_meta_gather(int64_t ncomp, int dims, const double* __restrict__ vecs, int k,
                              const int* __restrict__ sel, double* __restrict__ meta) {
  const int64_t total = ncomp * dims;
  const int64_t stride = static_cast<int64_t>(gridDim.x) * blockDim.x;
  for (int64_t e = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; e < total; e += stride) {
    const int64_t i = e / dims;
    const int d = static_cast<int>(e % dims);
    meta[e] = vecs[i * k + sel[d]];
  }
}

// x /= d (the meta coordinates over their largest magnitude)
__global__ void k_divide(int64_t count, double d, double* __restrict__ x) {
  const int64_t stride = static_cast<int64_t>(gridDim.x) * blockDim.x;
  for (int64_t e = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; e < count; e += stride) x[e] /= d;
}

// the orthogonal layout (src/multi_component.rs:127-140): component c at
// +e_(c mod dims) for the first dims components, -e_(c mod dims) after
__global__ void k_meta_orthogonal(int64_t ncomp, int dims, double* __restrict__ meta) {
  const int64_t total = ncomp * dims;
  const int64_t stride = static_cast<int64_t>(gridDim.x) * blockDim.x;
  for (int64_t e = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; e < total; e += stride) {
    const int64_t c = e / dims;
    const int d = static_cast<int>(e % dims);
    meta[e] = (d == c % dims) ? (c < dims ? 1.0 : -1.0) : 0.0;
  }
}

// ranges[c] = half the distance to the nearest other (distinct) component
// position, 1 when there is none (src/multi_component.rs:224-255)
__global__ void k_meta_ranges(int64_t ncomp, int dims, const double* __restrict__ meta, double* __restrict__ ranges) {
  const int64_t stride = static_cast<int64_t>(gridDim.x) * blockDim.x;
  for (int64_t c = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; c < ncomp; c += stride) {
    double md = INFINITY;
    for (int64_t i = 0; i < ncomp; ++i) {
      if (i == c) continue;
      double s = 0.0;
      for (int d = 0; d < dims; ++d) {
        const double df = meta[c * dims + d] - meta[i * dims + d];
        s += df * df;
      }
      const double dist = sqrt(s);
      if (dist > 0.0 && dist < md) md = dist;
    }
    ranges[c] = (ncomp > 1 && isfinite(md)) ? md / 2.0 : 1.0;
  }
}


int grid_for(const Exec& ex, int64_t items) {
  return static_cast<int>(std::max<int64_t>(1, std::min<int64_t>((items + 255) / 256, int64_t(ex.sms) * 16)));
}

std::vector<int> selection_order(const std::vector<double>& vals, int nc) {
  SI_REQUIRE(static_cast<int>(vals.size()) > nc, SI_CONVERGENCE_FAILURE,
             "need at least n_components+1 eigenvalues");
  std::vector<int> idx(vals.size());
  std::iota(idx.begin(), idx.end(), 0);
  std::stable_sort(idx.begin(), idx.end(), [&](int a, int b) { return vals[a] < vals[b]; });
  return std::vector<int>(idx.begin() + 1, idx.begin() + 1 + nc);
}

// One connected (sub)graph -> selected, sign-normalised eigenvectors [n x nc] (f64).
void embed_connected(const Exec& ex, const GraphDev& g, int nc, uint64_t seed, const PipelineConfig& pc,
                     DevBuf<double>& coords, SolverStats& st, std::vector<double>& eigvals_out) {
  const int64_t n = g.n;
  DevBuf<double> deg(n, ex.stream), sq(n, ex.stream), inv(n, ex.stream), v64(std::max<int64_t>(g.nnz, 1), ex.stream);
  DevBuf<float> v32;
  compute_degrees_dev(ex, g, pc.compute_mode, deg.get(), sq.get());
  inv_sqrt_dev(ex, sq.get(), n, inv.get());
  const bool mixed = pc.solver.precision == SI_PRECISION_MIXED;
  if (mixed) v32.alloc(std::max<int64_t>(g.nnz, 1), ex.stream);
  laplacian_values_dev(ex, g, inv.get(), v64.get(), mixed ? v32.get() : nullptr);
  OpDev op;
  op.n = n;
  op.nnz = g.nnz;
  op.indptr = g.indptr;
  op.indices = g.indices;
  op.v64 = v64.get();
  op.v32 = mixed ? v32.get() : nullptr;
  op.diag = 1.0;
  EigenResult r;
  SolverConfig sc = pc.solver;
  solve_eigenproblem_dev(ex, op, nc, seed, sq.get(), sc, r, st);
  eigvals_out = r.vals;
  const std::vector<int> order = selection_order(r.vals, nc);
  coords.alloc(static_cast<size_t>(n) * nc, ex.stream);
  gather_columns_dev<double, double>(ex, r.vecs.get(), r.k, coords.get(), nc, n, order);
  GramWork gw;
  normalize_signs_dev(ex, gw, coords.get(), n, nc, nc);
}

}  // namespace

void spectral_init_pipeline(const Exec& ex, const GraphDev& g, int nc, uint64_t seed, const float* data_dev,
                            int64_t n_features, const PipelineConfig& pc, float* out_dev, PipelineReport& rep) {
  const int64_t n = g.n;
  if (n == 0 || nc == 0)
    throw Error(SI_INVALID_GRAPH, "invalid graph: spectral_init requires n > 0 and n_components > 0; got n=" +
                                      std::to_string(n) + ", n_components=" + std::to_string(nc));
  if (n <= nc)
    throw Error(SI_TOO_FEW_NODES, "graph has too few nodes (" + std::to_string(n) + ") for " + std::to_string(nc) +
                                      "-dimensional embedding");
  SI_REQUIRE(nc + 1 <= MAXM, SI_INVALID_ARGUMENT, "n_components must be <= 15");
  validate_graph(ex, g);
  DevBuf<uint32_t> labels(n, ex.stream);
  const int64_t ncomp = find_components_dev(ex, g, labels.get());
  rep.n_components_graph = static_cast<int>(ncomp);
  GramWork gw;
  DevBuf<double> result;
  if (ncomp <= 1) {
    std::vector<double> ev;
    embed_connected(ex, g, nc, seed, pc, result, rep.stats, ev);
    rep.eigvals = ev;
  } else {
    embed_disconnected_dev(ex, g, labels.get(), ncomp, nc, seed, data_dev, n_features, pc, result, rep);
  }
  const double mx = max_abs_dev(ex, gw, result.get(), n, nc, nc);
  if (!(mx > 0.0))
    throw Error(SI_INVALID_GRAPH, "invalid graph: scale_coords: embedding is all-zero; cannot scale to max=10");
  scale_noise_dev(ex, result.get(), n, nc, nc, 10.0 / mx, seed, out_dev, pc.add_noise);
  SI_CUDA(cudaStreamSynchronize(ex.stream));
}

void embed_disconnected_dev(const Exec& ex, const GraphDev& g, const uint32_t* labels, int64_t ncomp, int nc,
                            uint64_t seed, const float* data_dev, int64_t n_features, const PipelineConfig& pc,
                            DevBuf<double>& result, PipelineReport& rep) {
  const int64_t n = g.n;
  // ---- stable order by (label, node) -------------------------------------------
  DevBuf<uint32_t> ids(n, ex.stream), perm(n, ex.stream), lab_sorted(n, ex.stream), pos(n, ex.stream);
  k_iota_u32p<<<grid_for(ex, n), 256, 0, ex.stream>>>(n, ids.get());
  SI_LAUNCH_CHECK();
  {
    size_t tmp_bytes = 0;
    int end_bit = 1;
    while (end_bit < 32 && (int64_t(1) << end_bit) < ncomp) ++end_bit;
    SI_CUDA(cub::DeviceRadixSort::SortPairs(nullptr, tmp_bytes, labels, lab_sorted.get(), ids.get(), perm.get(), n, 0,
                                            end_bit, ex.stream));
    DevBuf<unsigned char> tmp(tmp_bytes, ex.stream);
    SI_CUDA(cub::DeviceRadixSort::SortPairs(tmp.get(), tmp_bytes, labels, lab_sorted.get(), ids.get(), perm.get(), n,
                                            0, end_bit, ex.stream));
  }
  k_inverse_perm<<<grid_for(ex, n), 256, 0, ex.stream>>>(n, perm.get(), pos.get());
  SI_LAUNCH_CHECK();
  DevBuf<uint64_t> csize(ncomp + 1, ex.stream), coff(ncomp + 1, ex.stream);
  csize.zero();
  k_label_counts<<<grid_for(ex, n), 256, 0, ex.stream>>>(n, labels, csize.get());
  SI_LAUNCH_CHECK();
  exclusive_scan_u64(ex, csize.get(), coff.get(), ncomp);
  std::vector<uint64_t> h_off(ncomp + 1);
  SI_CUDA(cudaMemcpyAsync(h_off.data(), coff.get(), sizeof(uint64_t) * (ncomp + 1), cudaMemcpyDeviceToHost, ex.stream));
  // ---- block-diagonal permuted graph with component-local columns ----------------
  DevBuf<uint64_t> cnt(n + 1, ex.stream), pptr(n + 1, ex.stream);
  cnt.zero();
  k_perm_counts<<<grid_for(ex, n), 256, 0, ex.stream>>>(n, perm.get(), g.indptr, g.indices, labels, cnt.get());
  SI_LAUNCH_CHECK();
  const uint64_t pnnz = exclusive_scan_u64(ex, cnt.get(), pptr.get(), n);
  DevBuf<uint32_t> pidx(std::max<uint64_t>(pnnz, 1), ex.stream);
  DevBuf<float> pval(std::max<uint64_t>(pnnz, 1), ex.stream);
  k_perm_fill<<<grid_for(ex, n), 256, 0, ex.stream>>>(n, perm.get(), pos.get(), g.indptr, g.indices, g.data, labels,
                                                      coff.get(), pptr.get(), pidx.get(), pval.get());
  SI_LAUNCH_CHECK();
  std::vector<uint64_t> h_pptr(n + 1);
  SI_CUDA(cudaMemcpyAsync(h_pptr.data(), pptr.get(), sizeof(uint64_t) * (n + 1), cudaMemcpyDeviceToHost, ex.stream));
  SI_CUDA(cudaStreamSynchronize(ex.stream));

  // ---- meta-embedding (src/multi_component.rs:31-51, :127-255), on the device ----
  const int dims = nc;
  DevBuf<double> dmeta_all(static_cast<size_t>(ncomp) * dims, ex.stream);
  if (ncomp > 2 * dims) {
    if (data_dev == nullptr)
      throw Error(SI_INVALID_GRAPH,
                  "invalid graph: data is required for spectral meta-embedding when n_conn_components > 2 * "
                  "n_embedding_dims");
    const int nf = static_cast<int>(n_features);
    DevBuf<double> cent(static_cast<size_t>(ncomp) * nf, ex.stream);
    cent.zero();
    k_centroid_sums<<<grid_for(ex, n * nf), 256, 0, ex.stream>>>(n, nf, data_dev, labels, cent.get());
    SI_LAUNCH_CHECK();
    k_centroid_mean<<<grid_for(ex, ncomp * nf), 256, 0, ex.stream>>>(ncomp, nf, coff.get(), cent.get());
    SI_LAUNCH_CHECK();
    // Gaussian affinity and the normalised Laplacian of the centroid graph
    const int64_t mnnz = ncomp * ncomp;
    DevBuf<double> aff(static_cast<size_t>(mnnz), ex.stream), invm(ncomp, ex.stream), dsq(ncomp, ex.stream);
    k_meta_affinity<<<grid_for(ex, mnnz), 256, 0, ex.stream>>>(ncomp, nf, cent.get(), aff.get());
    SI_LAUNCH_CHECK();
    k_meta_degrees<<<grid_for(ex, ncomp), 256, 0, ex.stream>>>(ncomp, aff.get(), invm.get(), dsq.get());
    SI_LAUNCH_CHECK();
    DevBuf<uint64_t> dlp(ncomp + 1, ex.stream);
    DevBuf<uint32_t> dli(static_cast<size_t>(mnnz), ex.stream);
    DevBuf<double> dlv(static_cast<size_t>(mnnz), ex.stream);
    k_meta_laplacian<<<grid_for(ex, mnnz + 1), 256, 0, ex.stream>>>(ncomp, aff.get(), invm.get(), dlp.get(), dli.get(),
                                                                   dlv.get());
    SI_LAUNCH_CHECK();
    OpDev mop = op_from_csr64(dlp.get(), dli.get(), dlv.get(), ncomp, mnnz);
    EigenResult r;
    SolverStats mst;
    SolverConfig msc = pc.solver;
    msc.precision = SI_PRECISION_FP64;
    msc.force_level = -1;
    solve_eigenproblem_dev(ex, mop, dims, seed, dsq.get(), msc, r, mst);
    const std::vector<int> sel = selection_order(r.vals, dims);
    DevBuf<int> dsel(dims, ex.stream);
    SI_CUDA(cudaMemcpyAsync(dsel.get(), sel.data(), sizeof(int) * dims, cudaMemcpyHostToDevice, ex.stream));
    k_meta_gather<<<grid_for(ex, ncomp * dims), 256, 0, ex.stream>>>(ncomp, dims, r.vecs.get(), r.k, dsel.get(),
                                                                     dmeta_all.get());
    SI_LAUNCH_CHECK();
    GramWork gwm;
    const double mx = max_abs_dev(ex, gwm, dmeta_all.get(), ncomp, dims, dims);
    if (mx == 0.0) throw Error(SI_INVALID_GRAPH, "invalid graph: spectral meta-embedding produced all-zero result");
    k_divide<<<grid_for(ex, ncomp * dims), 256, 0, ex.stream>>>(ncomp * dims, mx, dmeta_all.get());
    SI_LAUNCH_CHECK();
  } else {
    k_meta_orthogonal<<<grid_for(ex, ncomp * dims), 256, 0, ex.stream>>>(ncomp, dims, dmeta_all.get());
    SI_LAUNCH_CHECK();
  }
  // data ranges (src/multi_component.rs:224-255); the host needs them for the scale factors
  std::vector<double> ranges(ncomp, 1.0);
  {
    DevBuf<double> dranges(ncomp, ex.stream);
    k_meta_ranges<<<grid_for(ex, ncomp), 256, 0, ex.stream>>>(ncomp, dims, dmeta_all.get(), dranges.get());
    SI_LAUNCH_CHECK();
    SI_CUDA(cudaMemcpyAsync(ranges.data(), dranges.get(), sizeof(double) * ncomp, cudaMemcpyDeviceToHost, ex.stream));
    SI_CUDA(cudaStreamSynchronize(ex.stream));
  }
  // ---- per component (src/multi_component.rs:261-312) -----------------------------
  // Components are independent: worker threads, each with its own stream,
  // take them largest first, so small components (single-CTA dense solves,
  // latency-bound LOBPCG steps) run side by side on the GPU.  Every worker
  // writes only its components' rows of `result`.
  result.alloc(static_cast<size_t>(n) * dims, ex.stream);
  SI_CUDA(cudaStreamSynchronize(ex.stream));
  std::vector<int64_t> order(ncomp);
  std::iota(order.begin(), order.end(), 0);
  std::stable_sort(order.begin(), order.end(), [&](int64_t a, int64_t b) {
    return (h_off[a + 1] - h_off[a]) > (h_off[b + 1] - h_off[b]);
  });
  std::atomic<int64_t> next{0};
  std::atomic<bool> failed{false};
  std::mutex mu;
  std::exception_ptr first_error;
  auto solve_one = [&](const Exec& wex, GramWork& gw, int64_t c) {
    const int64_t off = static_cast<int64_t>(h_off[c]);
    const int64_t sz = static_cast<int64_t>(h_off[c + 1] - h_off[c]);
    const double* dmeta = dmeta_all.get() + c * dims;  // written on ex.stream, synchronised above
    if (sz < 2 * dims) {
      k_place<<<grid_for(wex, sz * dims), 256, 0, wex.stream>>>(sz, off, perm.get(), nullptr, dims, 0.0, dmeta,
                                                                 result.get());
      SI_LAUNCH_CHECK();
      SI_CUDA(cudaStreamSynchronize(wex.stream));
      return;
    }
    // component view: its rows are contiguous in the permuted CSR; every array
    // handed to the solver is component-relative (indptr rebased to 0)
    const uint64_t ebase = h_pptr[off];
    DevBuf<uint64_t> sub_ptr(sz + 1, wex.stream);
    k_rebase<<<grid_for(wex, sz + 1), 256, 0, wex.stream>>>(sz, pptr.get() + off, ebase, sub_ptr.get());
    SI_LAUNCH_CHECK();
    GraphDev sub;
    sub.n = sz;
    sub.nnz = static_cast<int64_t>(h_pptr[off + sz] - ebase);
    sub.indptr = sub_ptr.get();
    sub.indices = pidx.get() + ebase;
    sub.data = pval.get() + ebase;
    DevBuf<double> coords;
    SolverStats cst;
    std::vector<double> ev;
    embed_connected(wex, sub, dims, seed, pc, coords, cst, ev);
    const double mx = max_abs_dev(wex, gw, coords.get(), sz, dims, dims);
    const double s = mx > 0.0 ? ranges[c] / mx : 1.0;
    k_place<<<grid_for(wex, sz * dims), 256, 0, wex.stream>>>(sz, off, perm.get(), coords.get(), dims, s, dmeta,
                                                               result.get());
    SI_LAUNCH_CHECK();
    SI_CUDA(cudaStreamSynchronize(wex.stream));
    std::lock_guard<std::mutex> lk(mu);
    rep.stats.iterations += cst.iterations;
    rep.stats.spmm_calls += cst.spmm_calls;
    rep.stats.level = std::max(rep.stats.level, cst.level);
    rep.stats.max_residual = std::max(rep.stats.max_residual, cst.max_residual);
  };
  auto worker = [&]() {
    cudaStream_t st = nullptr;
    try {
      SI_CUDA(cudaSetDevice(ex.device));
      SI_CUDA(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
      Exec wex = ex;
      wex.stream = st;
      GramWork gw;
      for (;;) {
        const int64_t i = next.fetch_add(1);
        if (i >= ncomp || failed.load()) break;
        solve_one(wex, gw, order[i]);
      }
    } catch (...) {
      std::lock_guard<std::mutex> lk(mu);
      if (!first_error) first_error = std::current_exception();
      failed.store(true);
    }
    if (st != nullptr) {
      cudaStreamSynchronize(st);
      cudaStreamDestroy(st);
    }
  };
  const int n_workers = static_cast<int>(std::min<int64_t>(kComponentWorkers, ncomp));
  std::vector<std::thread> pool;
  for (int w = 1; w < n_workers; ++w) pool.emplace_back(worker);
  worker();
  for (auto& t : pool) t.join();
  if (first_error) std::rethrow_exception(first_error);
}

}  // namespace si
