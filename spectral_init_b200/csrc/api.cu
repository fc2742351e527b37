// extern "C" boundary of the library (declared in include/spectral_init_gpu.h).
// Every entry point converts internal exceptions into si_status codes plus a
// message for si_last_error(); nothing unwinds across the ABI.
#include <cuda_runtime.h>

#include <cstring>
#include <memory>
#include <mutex>
#include <new>
#include <string>
#include <vector>

#include "mpnn.h"
#include "pipeline.h"

std::atomic<uint64_t> si::g_kernel_launches{0};
thread_local uint64_t si::tl_kernel_launches = 0;

struct si_model {
  int device = 0;
  std::mutex mu;  // one forward pass at a time (components may be solved concurrently)
  si::MpnnModel m;
  si::MpnnActs acts;
  si::GemmWorkspace ws;
};

struct si_ctx {
  int device = 0;
  cudaStream_t stream = nullptr;
  int sms = 148;
  std::string last_error;
  si_model* model = nullptr;  // learned warm start
  si::Exec ex() const {
    si::Exec e;
    e.stream = stream;
    e.sms = sms;
    e.device = device;
    return e;
  }
};

namespace {

template <class F>
si_status guarded(si_ctx* ctx, F&& f) {
  if (ctx == nullptr) return SI_INVALID_ARGUMENT;
  try {
    cudaError_t e = cudaSetDevice(ctx->device);
    if (e != cudaSuccess) throw si::Error(SI_CUDA_ERROR, std::string("cudaSetDevice: ") + cudaGetErrorString(e));
    f();
    ctx->last_error.clear();
    return SI_OK;
  } catch (const si::Error& err) {
    ctx->last_error = err.what();
    return err.code;
  } catch (const std::bad_alloc&) {
    ctx->last_error = "host allocation failed";
    return SI_OUT_OF_MEMORY;
  } catch (const std::exception& err) {
    ctx->last_error = err.what();
    return SI_CUDA_ERROR;
  } catch (...) {
    ctx->last_error = "unknown internal error";
    return SI_CUDA_ERROR;
  }
}

si::GraphDev graph_of(const si_csr_f32* g) {
  SI_REQUIRE(g != nullptr, SI_INVALID_ARGUMENT, "graph is null");
  si::GraphDev d;
  d.n = static_cast<int64_t>(g->n);
  d.nnz = static_cast<int64_t>(g->nnz);
  d.indptr = g->indptr;
  d.indices = g->indices;
  d.data = g->data;
  return d;
}

si::OpDev op_of(const si_operator* op) {
  SI_REQUIRE(op != nullptr, SI_INVALID_ARGUMENT, "operator is null");
  si::OpDev d;
  d.n = static_cast<int64_t>(op->n);
  d.nnz = static_cast<int64_t>(op->nnz);
  d.indptr = op->indptr;
  d.indices = op->indices;
  d.v64 = op->values;
  d.v32 = op->values_f32;
  d.diag = op->diag;
  return d;
}

// Learned start of a solve: features, forward pass, first k predicted columns.
bool learned_block(si_model* model, const si::Exec& ex, const si::OpDev& op, const double* sqrt_deg, int k,
                   uint64_t seed, double* x, int ld) {
  if (op.v32 == nullptr || sqrt_deg == nullptr || k > si::kMpnnOut) return false;
  std::lock_guard<std::mutex> lock(model->mu);
  si::mpnn_features(ex, op, sqrt_deg, seed, nullptr, model->acts);
  si::mpnn_forward(ex, model->m, op, model->acts, model->ws);
  std::vector<int> cols(k);
  for (int c = 0; c < k; ++c) cols[c] = c;
  si::gather_columns_dev<float, double>(ex, model->acts.y.get(), si::kMpnnOut, x, ld, op.n, cols);
  si::gemm_check(ex, model->ws);
  return true;
}

si::SolverConfig solver_cfg(si_ctx* ctx, const si_config* cfg) {
  si_config c;
  if (cfg) c = *cfg; else si_config_default(&c);
  si::SolverConfig s;
  s.block_size = c.block_size;
  s.dense_threshold = c.dense_threshold > 0 ? c.dense_threshold : 2000;
  s.force_level = c.force_level;
  s.rsvd_oversampling = c.rsvd_oversampling;
  s.rsvd_nbiter = c.rsvd_nbiter > 0 ? c.rsvd_nbiter : 2;
  s.max_iterations = c.max_iterations;
  s.precision = c.precision;
  s.tol = c.tol > 0.0 ? c.tol : 1e-5;
  s.mixed_switch_tol = c.mixed_switch_tol;
  s.learned_chebyshev = c.learned_filter != 0;
  SI_REQUIRE(c.precision == SI_PRECISION_FP64 || c.precision == SI_PRECISION_MIXED, SI_INVALID_ARGUMENT,
             "config: unknown precision");
  SI_REQUIRE(c.compute_mode == SI_COMPUTE_PYTHON_COMPAT || c.compute_mode == SI_COMPUTE_RUST_NATIVE,
             SI_INVALID_ARGUMENT, "config: unknown compute_mode");
  SI_REQUIRE(c.warm_start == SI_WARM_START_RANDOM || c.warm_start == SI_WARM_START_LEARNED, SI_INVALID_ARGUMENT,
             "config: unknown warm_start");
  if (c.warm_start == SI_WARM_START_LEARNED) {
    SI_REQUIRE(ctx->model != nullptr, SI_INVALID_ARGUMENT,
               "config: warm_start LEARNED needs a model attached with si_ctx_set_model");
    si_model* model = ctx->model;
    s.learned_start = [model](const si::Exec& ex, const si::OpDev& op, const double* sq, int k, uint64_t seed,
                              double* x, int ld) { return learned_block(model, ex, op, sq, k, seed, x, ld); };
  }
  return s;
}

void fill_report(si_report* rep, const si::SolverStats& st, int ncomp, const std::vector<double>& vals, double ms) {
  if (rep == nullptr) return;
  std::memset(rep, 0, sizeof(*rep));
  rep->level = st.level;
  rep->iterations = st.iterations;
  rep->restarts = st.restarts;
  rep->n_components_graph = ncomp;
  rep->fp32_iterations = st.fp32_iterations;
  rep->spmm_calls = st.spmm_calls;
  rep->learned_start = st.learned_used;
  rep->max_residual = st.max_residual;
  rep->solve_ms = ms;
  for (size_t i = 0; i < vals.size() && i < 16; ++i) rep->eigenvalues[i] = vals[i];
}

// Host explicit CSR (f64, diagonal stored) uploaded to the device.
struct HostCsr64 {
  si::DevBuf<uint64_t> indptr;
  si::DevBuf<uint32_t> indices;
  si::DevBuf<double> data;
  si::OpDev op;
  HostCsr64(const si::Exec& ex, const si_csr_f64* h) {
    SI_REQUIRE(h != nullptr && h->indptr != nullptr, SI_INVALID_ARGUMENT, "matrix is null");
    SI_REQUIRE(h->nnz == 0 || (h->indices != nullptr && h->data != nullptr), SI_INVALID_ARGUMENT,
               "matrix arrays are null");
    const int64_t n = static_cast<int64_t>(h->n), nnz = static_cast<int64_t>(h->nnz);
    indptr.alloc(n + 1, ex.stream);
    indices.alloc(std::max<int64_t>(nnz, 1), ex.stream);
    data.alloc(std::max<int64_t>(nnz, 1), ex.stream);
    SI_CUDA(cudaMemcpyAsync(indptr.get(), h->indptr, sizeof(uint64_t) * (n + 1), cudaMemcpyHostToDevice, ex.stream));
    if (nnz) {
      SI_CUDA(cudaMemcpyAsync(indices.get(), h->indices, sizeof(uint32_t) * nnz, cudaMemcpyHostToDevice, ex.stream));
      SI_CUDA(cudaMemcpyAsync(data.get(), h->data, sizeof(double) * nnz, cudaMemcpyHostToDevice, ex.stream));
    }
    si::GraphDev g;
    g.n = n;
    g.nnz = nnz;
    g.indptr = indptr.get();
    g.indices = indices.get();
    g.data = nullptr;
    si::validate_graph(ex, g);
    op = si::op_from_csr64(indptr.get(), indices.get(), data.get(), n, nnz);
  }
};

si_model* checked_model(si_ctx* ctx, si_model* model) {
  SI_REQUIRE(model != nullptr, SI_INVALID_ARGUMENT, "model is null");
  SI_REQUIRE(model->device == ctx->device, SI_INVALID_ARGUMENT, "model lives on another device");
  return model;
}

}  // namespace

extern "C" {

void si_config_default(si_config* cfg) {
  if (cfg == nullptr) return;
  std::memset(cfg, 0, sizeof(*cfg));
  cfg->compute_mode = SI_COMPUTE_PYTHON_COMPAT;
  cfg->precision = SI_PRECISION_FP64;
  cfg->warm_start = SI_WARM_START_RANDOM;
  cfg->block_size = 0;
  cfg->dense_threshold = 0;
  cfg->force_level = -1;
  cfg->rsvd_oversampling = -1;
  cfg->rsvd_nbiter = 0;
  cfg->max_iterations = 0;
  cfg->tol = 0.0;
  cfg->mixed_switch_tol = 0.0;
}

int32_t si_abi_version(void) { return SI_ABI_VERSION; }

uint64_t si_kernel_launches(void) { return si::g_kernel_launches.load(std::memory_order_relaxed); }

si_status si_ctx_create(int32_t device, si_ctx** out) {
  if (out == nullptr) return SI_INVALID_ARGUMENT;
  *out = nullptr;
  si_ctx* ctx = new (std::nothrow) si_ctx();
  if (ctx == nullptr) return SI_OUT_OF_MEMORY;
  ctx->device = device;
  int count = 0;
  if (cudaGetDeviceCount(&count) != cudaSuccess || device < 0 || device >= count) {
    delete ctx;
    return SI_CUDA_ERROR;
  }
  if (cudaSetDevice(device) != cudaSuccess ||
      cudaStreamCreateWithFlags(&ctx->stream, cudaStreamNonBlocking) != cudaSuccess) {
    delete ctx;
    return SI_CUDA_ERROR;
  }
  cudaDeviceGetAttribute(&ctx->sms, cudaDevAttrMultiProcessorCount, device);
  // keep freed pool memory cached across calls instead of returning it to the driver
  cudaMemPool_t pool;
  if (cudaDeviceGetDefaultMemPool(&pool, device) == cudaSuccess) {
    uint64_t thr = UINT64_MAX;
    cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &thr);
  }
  *out = ctx;
  return SI_OK;
}

void si_ctx_destroy(si_ctx* ctx) {
  if (ctx == nullptr) return;
  cudaSetDevice(ctx->device);
  if (ctx->stream) {
    cudaStreamSynchronize(ctx->stream);
    cudaStreamDestroy(ctx->stream);
  }
  delete ctx;
}

const char* si_last_error(const si_ctx* ctx) { return ctx ? ctx->last_error.c_str() : "null context"; }

si_status si_ctx_synchronize(si_ctx* ctx) {
  return guarded(ctx, [&] { SI_CUDA(cudaStreamSynchronize(ctx->stream)); });
}

void* si_ctx_stream(si_ctx* ctx) { return ctx ? static_cast<void*>(ctx->stream) : nullptr; }

si_status si_spectral_init_device(si_ctx* ctx, const si_csr_f32* graph, uint32_t n_components, uint64_t seed,
                                  const float* data, uint64_t n_features, const si_config* cfg, float* out,
                                  si_report* report) {
  return guarded(ctx, [&] {
    const si::Exec ex = ctx->ex();
    si::GraphDev g = graph_of(graph);
    si::PipelineConfig pc;
    pc.solver = solver_cfg(ctx, cfg);
    pc.compute_mode = cfg ? cfg->compute_mode : SI_COMPUTE_PYTHON_COMPAT;
    SI_REQUIRE(out != nullptr || g.n == 0 || n_components == 0, SI_INVALID_ARGUMENT, "out is null");
    si::PipelineReport rep;
    cudaEvent_t e0, e1;
    SI_CUDA(cudaEventCreate(&e0));
    SI_CUDA(cudaEventCreate(&e1));
    SI_CUDA(cudaEventRecord(e0, ex.stream));
    try {
      si::spectral_init_pipeline(ex, g, static_cast<int>(n_components), seed, data,
                                 static_cast<int64_t>(n_features), pc, out, rep);
    } catch (...) {
      cudaEventDestroy(e0);
      cudaEventDestroy(e1);
      throw;
    }
    SI_CUDA(cudaEventRecord(e1, ex.stream));
    SI_CUDA(cudaEventSynchronize(e1));
    float ms = 0.f;
    cudaEventElapsedTime(&ms, e0, e1);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    fill_report(report, rep.stats, rep.n_components_graph, rep.eigvals, ms);
  });
}

si_status si_spectral_init(si_ctx* ctx, const si_csr_f32* graph, uint32_t n_components, uint64_t seed,
                           const float* data, uint64_t n_features, const si_config* cfg, float* out,
                           si_report* report) {
  return guarded(ctx, [&] {
    const si::Exec ex = ctx->ex();
    SI_REQUIRE(graph != nullptr && graph->indptr != nullptr, SI_INVALID_ARGUMENT, "graph is null");
    const int64_t n = static_cast<int64_t>(graph->n), nnz = static_cast<int64_t>(graph->nnz);
    if (n == 0 || n_components == 0)
      throw si::Error(SI_INVALID_GRAPH, "invalid graph: spectral_init requires n > 0 and n_components > 0; got n=" +
                                            std::to_string(n) + ", n_components=" + std::to_string(n_components));
    if (n <= static_cast<int64_t>(n_components))
      throw si::Error(SI_TOO_FEW_NODES, "graph has too few nodes (" + std::to_string(n) + ") for " +
                                            std::to_string(n_components) + "-dimensional embedding");
    SI_REQUIRE(nnz == 0 || (graph->indices && graph->data), SI_INVALID_ARGUMENT, "graph arrays are null");
    SI_REQUIRE(out != nullptr, SI_INVALID_ARGUMENT, "out is null");
    si::DevBuf<uint64_t> ip(n + 1, ex.stream);
    si::DevBuf<uint32_t> ix(std::max<int64_t>(nnz, 1), ex.stream);
    si::DevBuf<float> dv(std::max<int64_t>(nnz, 1), ex.stream), dd, dout(static_cast<size_t>(n) * n_components, ex.stream);
    SI_CUDA(cudaMemcpyAsync(ip.get(), graph->indptr, sizeof(uint64_t) * (n + 1), cudaMemcpyHostToDevice, ex.stream));
    if (nnz) {
      SI_CUDA(cudaMemcpyAsync(ix.get(), graph->indices, sizeof(uint32_t) * nnz, cudaMemcpyHostToDevice, ex.stream));
      SI_CUDA(cudaMemcpyAsync(dv.get(), graph->data, sizeof(float) * nnz, cudaMemcpyHostToDevice, ex.stream));
    }
    if (data != nullptr && n_features > 0) {
      dd.alloc(static_cast<size_t>(n) * n_features, ex.stream);
      SI_CUDA(cudaMemcpyAsync(dd.get(), data, sizeof(float) * n * n_features, cudaMemcpyHostToDevice, ex.stream));
    }
    si_csr_f32 dg{static_cast<uint64_t>(n), static_cast<uint64_t>(nnz), ip.get(), ix.get(), dv.get()};
    si::GraphDev g = graph_of(&dg);
    si::PipelineConfig pc;
    pc.solver = solver_cfg(ctx, cfg);
    pc.compute_mode = cfg ? cfg->compute_mode : SI_COMPUTE_PYTHON_COMPAT;
    si::PipelineReport rep;
    cudaEvent_t e0, e1;
    SI_CUDA(cudaEventCreate(&e0));
    SI_CUDA(cudaEventCreate(&e1));
    SI_CUDA(cudaEventRecord(e0, ex.stream));
    try {
      si::spectral_init_pipeline(ex, g, static_cast<int>(n_components), seed, dd.get(),
                                 static_cast<int64_t>(n_features), pc, dout.get(), rep);
    } catch (...) {
      cudaEventDestroy(e0);
      cudaEventDestroy(e1);
      throw;
    }
    SI_CUDA(cudaEventRecord(e1, ex.stream));
    SI_CUDA(cudaMemcpyAsync(out, dout.get(), sizeof(float) * n * n_components, cudaMemcpyDeviceToHost, ex.stream));
    SI_CUDA(cudaStreamSynchronize(ex.stream));
    float ms = 0.f;
    cudaEventElapsedTime(&ms, e0, e1);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    fill_report(report, rep.stats, rep.n_components_graph, rep.eigvals, ms);
  });
}

si_status si_compute_degrees(si_ctx* ctx, const si_csr_f32* graph, int32_t compute_mode, double* degrees,
                             double* sqrt_deg) {
  return guarded(ctx, [&] {
    const si::Exec ex = ctx->ex();
    si::GraphDev g = graph_of(graph);
    SI_REQUIRE(compute_mode == SI_COMPUTE_PYTHON_COMPAT || compute_mode == SI_COMPUTE_RUST_NATIVE,
               SI_INVALID_ARGUMENT, "unknown compute_mode");
    SI_REQUIRE(g.n == 0 || (degrees && sqrt_deg), SI_INVALID_ARGUMENT, "output is null");
    si::validate_graph(ex, g);
    si::compute_degrees_dev(ex, g, compute_mode, degrees, sqrt_deg);
    SI_CUDA(cudaStreamSynchronize(ex.stream));
  });
}

si_status si_build_laplacian(si_ctx* ctx, const si_csr_f32* graph, const double* inv_sqrt_deg, double* values,
                             float* values_f32) {
  return guarded(ctx, [&] {
    const si::Exec ex = ctx->ex();
    si::GraphDev g = graph_of(graph);
    SI_REQUIRE(g.nnz == 0 || (values && inv_sqrt_deg), SI_INVALID_ARGUMENT, "null argument");
    si::validate_graph(ex, g);
    si::laplacian_values_dev(ex, g, inv_sqrt_deg, values, values_f32);
    SI_CUDA(cudaStreamSynchronize(ex.stream));
  });
}

si_status si_build_laplacian_csr(si_ctx* ctx, const si_csr_f32* graph, const double* inv_sqrt_deg,
                                 uint64_t* out_indptr, uint32_t* out_indices, double* out_data, uint64_t* out_nnz) {
  return guarded(ctx, [&] {
    const si::Exec ex = ctx->ex();
    si::GraphDev g = graph_of(graph);
    si::validate_graph(ex, g);
    const uint64_t nnz = si::laplacian_csr_nnz_dev(ex, g);
    if (out_nnz) *out_nnz = nnz;
    if (out_indices == nullptr) return;
    SI_REQUIRE(out_indptr && out_data && inv_sqrt_deg, SI_INVALID_ARGUMENT, "null argument");
    si::laplacian_csr_dev(ex, g, inv_sqrt_deg, out_indptr, out_indices, out_data);
    SI_CUDA(cudaStreamSynchronize(ex.stream));
  });
}

si_status si_fuzzy_graph(si_ctx* ctx, const double* points, uint64_t n, uint32_t dims, uint32_t k,
                         int32_t* knn_indices, float* knn_dists, float* sigmas, float* rhos, uint64_t* indptr,
                         uint32_t* indices, float* data, uint64_t capacity, uint64_t* nnz) {
  return guarded(ctx, [&] {
    SI_REQUIRE(points && knn_indices && knn_dists && sigmas && rhos && indptr && indices && data && nnz,
               SI_INVALID_ARGUMENT, "fuzzy graph: null pointer");
    si::fuzzy_graph_dev(ctx->ex(), points, static_cast<int64_t>(n), static_cast<int>(dims), static_cast<int>(k),
                        knn_indices, knn_dists, sigmas, rhos, indptr, indices, data, capacity, nnz);
  });
}

si_status si_find_components(si_ctx* ctx, const si_csr_f32* graph, uint32_t* labels, uint64_t* n_components) {
  return guarded(ctx, [&] {
    const si::Exec ex = ctx->ex();
    si::GraphDev g = graph_of(graph);
    SI_REQUIRE(g.n == 0 || labels, SI_INVALID_ARGUMENT, "labels is null");
    si::validate_graph(ex, g);
    const int64_t nc = si::find_components_dev(ex, g, labels);
    if (n_components) *n_components = static_cast<uint64_t>(nc);
  });
}

si_status si_spmm(si_ctx* ctx, const si_operator* op, const double* x, double* y, uint32_t k) {
  return guarded(ctx, [&] {
    const si::Exec ex = ctx->ex();
    si::OpDev o = op_of(op);
    SI_REQUIRE(k >= 1, SI_INVALID_ARGUMENT, "k must be >= 1");
    si::RowBlocks rb;
    si::make_row_blocks(ex, o, rb);
    rb.attach(o);
    si::Epilogue<double> ep;
    si::spmm_dev<double>(ex, o, x, y, static_cast<int>(k), static_cast<int>(k), ep);
    SI_CUDA(cudaStreamSynchronize(ex.stream));
  });
}

si_status si_spmm_f32(si_ctx* ctx, const si_operator* op, const float* x, float* y, uint32_t k) {
  return guarded(ctx, [&] {
    const si::Exec ex = ctx->ex();
    si::OpDev o = op_of(op);
    SI_REQUIRE(k >= 1, SI_INVALID_ARGUMENT, "k must be >= 1");
    si::RowBlocks rb;
    si::make_row_blocks(ex, o, rb);
    rb.attach(o);
    si::Epilogue<float> ep;
    si::spmm_dev<float>(ex, o, x, y, static_cast<int>(k), static_cast<int>(k), ep, nullptr, true);
    SI_CUDA(cudaStreamSynchronize(ex.stream));
  });
}

struct si_operator_plan {
  int device = 0;
  si::OpDev op;
  si::RowBlocks rb;
};

si_status si_operator_plan_create(si_ctx* ctx, const si_operator* op, si_operator_plan** out) {
  if (out != nullptr) *out = nullptr;
  return guarded(ctx, [&] {
    SI_REQUIRE(out != nullptr, SI_INVALID_ARGUMENT, "plan output pointer is null");
    const si::Exec ex = ctx->ex();
    std::unique_ptr<si_operator_plan> p(new si_operator_plan());
    p->device = ctx->device;
    p->op = op_of(op);
    si::make_row_blocks(ex, p->op, p->rb);
    p->rb.sell_ok = true;
    p->rb.attach(p->op);
    SI_CUDA(cudaStreamSynchronize(ex.stream));
    *out = p.release();
  });
}

void si_operator_plan_destroy(si_operator_plan* plan) {
  if (plan == nullptr) return;
  cudaSetDevice(plan->device);
  cudaDeviceSynchronize();
  delete plan;
}

si_status si_spmm_planned(si_ctx* ctx, const si_operator_plan* plan, const double* x, double* y, uint32_t k) {
  return guarded(ctx, [&] {
    SI_REQUIRE(plan != nullptr, SI_INVALID_ARGUMENT, "plan is null");
    SI_REQUIRE(plan->device == ctx->device, SI_INVALID_ARGUMENT, "plan was prepared on another device");
    SI_REQUIRE(k >= 1, SI_INVALID_ARGUMENT, "k must be >= 1");
    si::Epilogue<double> ep;
    si::spmm_dev<double>(ctx->ex(), plan->op, x, y, static_cast<int>(k), static_cast<int>(k), ep);
  });
}

si_status si_spmm_planned_f32(si_ctx* ctx, const si_operator_plan* plan, const float* x, float* y, uint32_t k) {
  return guarded(ctx, [&] {
    SI_REQUIRE(plan != nullptr, SI_INVALID_ARGUMENT, "plan is null");
    SI_REQUIRE(plan->device == ctx->device, SI_INVALID_ARGUMENT, "plan was prepared on another device");
    SI_REQUIRE(k >= 1, SI_INVALID_ARGUMENT, "k must be >= 1");
    si::Epilogue<float> ep;
    si::spmm_dev<float>(ctx->ex(), plan->op, x, y, static_cast<int>(k), static_cast<int>(k), ep, nullptr, true);
  });
}

si_status si_solve_eigenproblem(si_ctx* ctx, const si_operator* op, uint32_t n_components, uint64_t seed,
                                const double* sqrt_deg, const si_config* cfg, double* eigvals, double* eigvecs,
                                int32_t* level, si_report* report) {
  return guarded(ctx, [&] {
    const si::Exec ex = ctx->ex();
    si::OpDev o = op_of(op);
    SI_REQUIRE(n_components >= 1 && static_cast<int64_t>(n_components) < o.n, SI_INVALID_ARGUMENT,
               "need 1 <= n_components < n");
    si::SolverConfig sc = solver_cfg(ctx, cfg);
    si::EigenResult r;
    si::SolverStats st;
    si::solve_eigenproblem_dev(ex, o, static_cast<int>(n_components), seed, sqrt_deg, sc, r, st);
    if (eigvals) std::memcpy(eigvals, r.vals.data(), sizeof(double) * r.k);
    if (eigvecs)
      SI_CUDA(cudaMemcpyAsync(eigvecs, r.vecs.get(), sizeof(double) * o.n * r.k, cudaMemcpyDeviceToDevice,
                              ex.stream));
    SI_CUDA(cudaStreamSynchronize(ex.stream));
    if (level) *level = st.level;
    fill_report(report, st, 1, r.vals, 0.0);
  });
}

si_status si_solve_eigenproblem_host(si_ctx* ctx, const si_csr_f64* laplacian, uint32_t n_components, uint64_t seed,
                                     const si_config* cfg, double* eigvals, double* eigvecs, int32_t* level,
                                     si_report* report) {
  return guarded(ctx, [&] {
    const si::Exec ex = ctx->ex();
    HostCsr64 L(ex, laplacian);
    const int64_t n = L.op.n;
    SI_REQUIRE(n_components >= 1 && static_cast<int64_t>(n_components) < n, SI_INVALID_ARGUMENT,
               "need 1 <= n_components < n");
    std::vector<double> ones(n, 1.0);
    si::DevBuf<double> sq(n, ex.stream);
    SI_CUDA(cudaMemcpyAsync(sq.get(), ones.data(), sizeof(double) * n, cudaMemcpyHostToDevice, ex.stream));
    si::SolverConfig sc = solver_cfg(ctx, cfg);
    si::EigenResult r;
    si::SolverStats st;
    si::solve_eigenproblem_dev(ex, L.op, static_cast<int>(n_components), seed, sq.get(), sc, r, st);
    if (eigvals) std::memcpy(eigvals, r.vals.data(), sizeof(double) * r.k);
    if (eigvecs)
      SI_CUDA(cudaMemcpyAsync(eigvecs, r.vecs.get(), sizeof(double) * n * r.k, cudaMemcpyDeviceToHost, ex.stream));
    SI_CUDA(cudaStreamSynchronize(ex.stream));
    if (level) *level = st.level;
    fill_report(report, st, 1, r.vals, 0.0);
  });
}

si_status si_lobpcg_solve_host(si_ctx* ctx, const si_csr_f64* op, uint32_t n_components, uint64_t seed,
                               int32_t regularize, const double* sqrt_deg, const si_config* cfg, double* eigvals,
                               double* eigvecs, int32_t* restarts, si_report* report) {
  return guarded(ctx, [&] {
    const si::Exec ex = ctx->ex();
    HostCsr64 L(ex, op);
    const int64_t n = L.op.n;
    SI_REQUIRE(sqrt_deg != nullptr, SI_INVALID_ARGUMENT, "sqrt_deg is null");
    si::DevBuf<double> sq(n, ex.stream);
    SI_CUDA(cudaMemcpyAsync(sq.get(), sqrt_deg, sizeof(double) * n, cudaMemcpyHostToDevice, ex.stream));
    si::SolverConfig sc = solver_cfg(ctx, cfg);
    si::EigenResult r;
    si::SolverStats st;
    const bool ok = si::lobpcg_solve_dev(ex, L.op, static_cast<int>(n_components), seed, regularize != 0, sq.get(),
                                         sc, r, st);
    if (!ok) throw si::Error(SI_CONVERGENCE_FAILURE, "lobpcg_solve returned no result");
    if (eigvals) std::memcpy(eigvals, r.vals.data(), sizeof(double) * r.k);
    if (eigvecs)
      SI_CUDA(cudaMemcpyAsync(eigvecs, r.vecs.get(), sizeof(double) * n * r.k, cudaMemcpyDeviceToHost, ex.stream));
    SI_CUDA(cudaStreamSynchronize(ex.stream));
    if (restarts) *restarts = st.restarts;
    st.level = regularize ? 3 : 1;
    fill_report(report, st, 1, r.vals, 0.0);
  });
}

si_status si_rsvd_solve_host(si_ctx* ctx, const si_csr_f64* laplacian, uint32_t n_components, uint64_t seed,
                             int32_t oversampling, int32_t nbiter, double* eigvals, double* eigvecs) {
  return guarded(ctx, [&] {
    const si::Exec ex = ctx->ex();
    HostCsr64 L(ex, laplacian);
    si::EigenResult r;
    si::SolverStats st;
    si::rsvd_solve_dev(ex, L.op, static_cast<int>(n_components), seed, oversampling, nbiter, r, st);
    if (eigvals) std::memcpy(eigvals, r.vals.data(), sizeof(double) * r.k);
    if (eigvecs)
      SI_CUDA(cudaMemcpyAsync(eigvecs, r.vecs.get(), sizeof(double) * L.op.n * r.k, cudaMemcpyDeviceToHost,
                              ex.stream));
    SI_CUDA(cudaStreamSynchronize(ex.stream));
  });
}

si_status si_dense_evd_host(si_ctx* ctx, const si_csr_f64* laplacian, uint32_t k, double* eigvals, double* eigvecs) {
  return guarded(ctx, [&] {
    const si::Exec ex = ctx->ex();
    HostCsr64 L(ex, laplacian);
    if (static_cast<int64_t>(k) > L.op.n)
      throw si::Error(SI_TOO_FEW_NODES, "graph has too few nodes (" + std::to_string(L.op.n) + ") for " +
                                            std::to_string(k) + "-dimensional embedding");
    si::EigenResult r;
    si::dense_evd_result(ex, L.op, static_cast<int>(k), r);
    if (eigvals) std::memcpy(eigvals, r.vals.data(), sizeof(double) * r.k);
    if (eigvecs)
      SI_CUDA(cudaMemcpyAsync(eigvecs, r.vecs.get(), sizeof(double) * L.op.n * r.k, cudaMemcpyDeviceToHost,
                              ex.stream));
    SI_CUDA(cudaStreamSynchronize(ex.stream));
  });
}

si_status si_normalize_signs(si_ctx* ctx, double* coords, uint64_t n, uint32_t k) {
  return guarded(ctx, [&] {
    const si::Exec ex = ctx->ex();
    si::GramWork gw;
    si::normalize_signs_dev(ex, gw, coords, static_cast<int64_t>(n), static_cast<int>(k), static_cast<int>(k));
    SI_CUDA(cudaStreamSynchronize(ex.stream));
  });
}

// Same result as si_normalize_signs, with every temporary in a static device
// array instead of pool allocations (noalloc.cu explains who needs this).
si_status si_normalize_signs_noalloc(si_ctx* ctx, double* coords, uint64_t n, uint32_t k) {
  return guarded(ctx, [&] {
    const si::Exec ex = ctx->ex();
    if (n > static_cast<uint64_t>(INT64_MAX))
      throw si::Error(SI_INVALID_ARGUMENT, "normalize_signs_noalloc: n does not fit a 64-bit signed index");
    if (k > static_cast<uint32_t>(si::kNoAllocMaxCols))
      throw si::Error(SI_INVALID_ARGUMENT, "normalize_signs_noalloc: k = " + std::to_string(k) +
                                               " columns exceeds the maximum of " +
                                               std::to_string(si::kNoAllocMaxCols) + " held by the static scratch");
    si::normalize_signs_noalloc_dev(ex, coords, static_cast<int64_t>(n), static_cast<int>(k));
    SI_CUDA(cudaStreamSynchronize(ex.stream));
  });
}

uint64_t si_model_param_count(void) { return static_cast<uint64_t>(si::mpnn_param_count()); }

si_status si_model_create(si_ctx* ctx, uint64_t seed, si_model** out) {
  if (out == nullptr) return SI_INVALID_ARGUMENT;
  *out = nullptr;
  return guarded(ctx, [&] {
    si_model* m = new si_model();
    m->device = ctx->device;
    try {
      m->m.init(ctx->ex(), seed);
      SI_CUDA(cudaStreamSynchronize(ctx->stream));
    } catch (...) {
      delete m;
      throw;
    }
    *out = m;
  });
}

void si_model_destroy(si_model* model) {
  if (model == nullptr) return;
  cudaSetDevice(model->device);
  cudaDeviceSynchronize();
  delete model;
}

si_status si_model_set_params(si_ctx* ctx, si_model* model, const float* params) {
  return guarded(ctx, [&] {
    SI_REQUIRE(params != nullptr, SI_INVALID_ARGUMENT, "params is null");
    checked_model(ctx, model)->m.set(ctx->ex(), params);
  });
}

si_status si_model_get_params(si_ctx* ctx, si_model* model, float* params) {
  return guarded(ctx, [&] {
    SI_REQUIRE(params != nullptr, SI_INVALID_ARGUMENT, "params is null");
    checked_model(ctx, model)->m.get(ctx->ex(), params);
  });
}

si_status si_model_train_step(si_ctx* ctx, si_model* model, const si_operator* op, const double* sqrt_deg,
                              const double* target, uint32_t k, uint64_t seed, float lr, double* loss) {
  return guarded(ctx, [&] {
    si_model* m = checked_model(ctx, model);
    const si::Exec ex = ctx->ex();
    si::OpDev o = op_of(op);
    SI_REQUIRE(o.n > 0 && o.v32 != nullptr && target != nullptr && sqrt_deg != nullptr, SI_INVALID_ARGUMENT,
               "train_step: needs a non-empty operator with f32 values, sqrt_deg and target");
    si::mpnn_features(ex, o, sqrt_deg, seed, nullptr, m->acts);
    si::mpnn_forward(ex, m->m, o, m->acts, m->ws);
    const double l = si::mpnn_loss_backward(ex, m->m, o, m->acts, target, static_cast<int>(k), static_cast<int>(k),
                                            m->ws);
    si::mpnn_adam(ex, m->m, lr);
    SI_CUDA(cudaStreamSynchronize(ex.stream));
    if (loss) *loss = l;
  });
}

si_status si_model_gradient(si_ctx* ctx, si_model* model, const si_operator* op, const double* sqrt_deg,
                            const float* features, const double* target, uint32_t k, uint64_t seed, double* loss,
                            float* grad) {
  return guarded(ctx, [&] {
    si_model* m = checked_model(ctx, model);
    const si::Exec ex = ctx->ex();
    si::OpDev o = op_of(op);
    SI_REQUIRE(o.n > 0 && o.v32 != nullptr && target != nullptr, SI_INVALID_ARGUMENT,
               "gradient: needs a non-empty operator with f32 values and a target");
    si::mpnn_features(ex, o, sqrt_deg, seed, features, m->acts);
    si::mpnn_forward(ex, m->m, o, m->acts, m->ws);
    const double l = si::mpnn_loss_backward(ex, m->m, o, m->acts, target, static_cast<int>(k), static_cast<int>(k),
                                            m->ws);
    if (grad != nullptr)
      SI_CUDA(cudaMemcpyAsync(grad, m->m.grad.get(), sizeof(float) * m->m.grad.size(), cudaMemcpyDeviceToHost,
                              ex.stream));
    SI_CUDA(cudaStreamSynchronize(ex.stream));
    if (loss) *loss = l;
  });
}

si_status si_model_predict(si_ctx* ctx, si_model* model, const si_operator* op, const double* sqrt_deg,
                           const float* features, uint64_t seed, float* out) {
  return guarded(ctx, [&] {
    si_model* m = checked_model(ctx, model);
    const si::Exec ex = ctx->ex();
    si::OpDev o = op_of(op);
    SI_REQUIRE(o.n > 0 && o.v32 != nullptr && out != nullptr, SI_INVALID_ARGUMENT,
               "predict: needs a non-empty operator with f32 values and an output");
    si::mpnn_features(ex, o, sqrt_deg, seed, features, m->acts);
    si::mpnn_forward(ex, m->m, o, m->acts, m->ws);
    SI_CUDA(cudaMemcpyAsync(out, m->acts.y.get(), sizeof(float) * o.n * si::kMpnnOut, cudaMemcpyDeviceToDevice,
                            ex.stream));
    si::gemm_check(ex, m->ws);
  });
}

si_status si_ctx_set_model(si_ctx* ctx, si_model* model) {
  return guarded(ctx, [&] {
    if (model != nullptr) checked_model(ctx, model);
    ctx->model = model;
  });
}

si_status si_gemm_bf16_nt(si_ctx* ctx, uint64_t m, uint32_t n, uint64_t k, const void* a, uint64_t lda,
                          const void* b, uint64_t ldb, float* c, uint64_t ldc, uint32_t k_splits) {
  return guarded(ctx, [&] {
    const si::Exec ex = ctx->ex();
    if (m == 0) return;
    if (a == nullptr || b == nullptr || c == nullptr)
      throw si::Error(SI_INVALID_ARGUMENT, "gemm_bf16_nt: null operand");
    si::GemmEpilogue ep;
    ep.mode = si::GEMM_STORE_F32;
    ep.out_f32 = c;
    ep.ldo = static_cast<int64_t>(ldc);
    si::GemmWorkspace ws;
    si::gemm_bf16_nt(ex, static_cast<int64_t>(m), static_cast<int>(n), static_cast<int64_t>(k),
                     static_cast<const __nv_bfloat16*>(a), static_cast<int64_t>(lda),
                     static_cast<const __nv_bfloat16*>(b), static_cast<int64_t>(ldb), ep,
                     static_cast<int>(k_splits), ws);
    si::gemm_check(ex, ws);
  });
}

si_status si_scale_and_add_noise(si_ctx* ctx, const double* coords, uint64_t n, uint32_t k, uint64_t seed,
                                 float* out) {
  return guarded(ctx, [&] {
    const si::Exec ex = ctx->ex();
    if (n == 0 || k == 0) throw si::Error(SI_INVALID_GRAPH, "invalid graph: scale_and_add_noise: input embedding is empty");
    si::GramWork gw;
    const double mx = si::max_abs_dev(ex, gw, coords, static_cast<int64_t>(n), static_cast<int>(k), static_cast<int>(k));
    if (!(mx > 0.0))
      throw si::Error(SI_INVALID_GRAPH, "invalid graph: scale_coords: embedding is all-zero; cannot scale to max=10");
    si::scale_noise_dev(ex, coords, static_cast<int64_t>(n), static_cast<int>(k), static_cast<int>(k), 10.0 / mx, seed,
                        out, true);
    SI_CUDA(cudaStreamSynchronize(ex.stream));
  });
}

}  // extern "C"
