/*
 * spectral_init_gpu.h -- C ABI of the B200 (sm_100a) spectral-initialisation
 * eigensolve path.
 *
 * Every entry point is `extern "C"`, takes plain pointers and sizes, never
 * throws or aborts across the boundary, and reports failures as an si_status
 * code plus a message readable through si_last_error().  Each declaration
 * names the function of the spectral-init crate (path:line inside that crate)
 * that it replaces.
 *
 * Memory conventions
 *   - "host" pointers are ordinary CPU memory (pageable or pinned);
 *   - "device" pointers are CUDA global memory on the context's device;
 *   - blocks of vectors are row-major [n x k] arrays of f64 (the crate's
 *     ndarray Array2<f64> layout);
 *   - graphs are CSR: indptr u64[n+1], indices u32[nnz] (sorted, unique per
 *     row), data f32[nnz] -- the crate's CsMatI<f32, u32, usize>.
 *
 * Threading: a context owns one CUDA stream and its workspace; use one
 * context per host thread.  Calls on different contexts may run
 * concurrently.
 */
#ifndef SPECTRAL_INIT_GPU_H
#define SPECTRAL_INIT_GPU_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define SI_ABI_VERSION 1

/* Status codes.  The first three mirror SpectralError (src/lib.rs:167-182). */
typedef enum si_status {
  SI_OK = 0,
  SI_CONVERGENCE_FAILURE = 1, /* SpectralError::ConvergenceFailure            */
  SI_INVALID_GRAPH = 2,       /* SpectralError::InvalidGraph(String)          */
  SI_TOO_FEW_NODES = 3,       /* SpectralError::TooFewNodes { n, dims }       */
  SI_CUDA_ERROR = 4,          /* a CUDA runtime call failed                   */
  SI_ITERATION_CAP = 5,       /* an iterative solve hit its iteration cap     */
  SI_INVALID_ARGUMENT = 6,    /* bad pointer / size / option                  */
  SI_OUT_OF_MEMORY = 7        /* device allocation failed                     */
} si_status;

/* ComputeMode (src/config.rs:5-14). */
typedef enum si_compute_mode {
  SI_COMPUTE_PYTHON_COMPAT = 0, /* f32 column-scatter degrees, bit-exact with scipy */
  SI_COMPUTE_RUST_NATIVE = 1    /* f64 row-sum degrees                               */
} si_compute_mode;

/* Arithmetic of the iterative eigensolve (new; the crate is f64 only). */
typedef enum si_precision {
  SI_PRECISION_FP64 = 0,  /* plain f64 throughout: the drop-in                     */
  SI_PRECISION_MIXED = 1  /* f32 SpMM/Chebyshev/LOBPCG bulk, f64 Gram/RR/refinement */
} si_precision;

/* Starting block of LOBPCG (new; the crate uses a seeded random block). */
typedef enum si_warm_start {
  SI_WARM_START_RANDOM = 0,
  SI_WARM_START_LEARNED = 1   /* message-passing network prediction (falls back to random) */
} si_warm_start;

/* SpectralInitConfig (src/config.rs:21-25) plus the B200 solver policy.
 * Always initialise with si_config_default(). */
typedef struct si_config {
  int32_t compute_mode;      /* si_compute_mode                                    */
  int32_t precision;         /* si_precision                                       */
  int32_t warm_start;        /* si_warm_start                                      */
  int32_t block_size;        /* LOBPCG block width; 0 = auto (guard vectors added) */
  int32_t dense_threshold;   /* Level-0 dense EVD for n < this; 0 = 2000           */
  int32_t force_level;       /* -1 = escalation chain; 0..5 = run only that level  */
  int32_t rsvd_oversampling; /* < 0 = crate formula (src/solvers/rsvd.rs:84-87)   */
  int32_t rsvd_nbiter;       /* <= 0 = 2 (src/solvers/rsvd.rs:123-126)           */
  int32_t max_iterations;    /* <= 0 = crate caps (300 first pass, 1000 restarts)  */
  int32_t learned_filter;    /* 1: also apply the Chebyshev start filter to a learned block */
  double tol;                /* LOBPCG convergence tolerance; <= 0 = 1e-5, the crate's
                                LOBPCG_ACCEPT_TOL (src/metrics.rs:40).  Smaller values
                                give more accurate pairs; the level-1/3 residual gate
                                stays 1e-5 (src/metrics.rs:30)                       */
  double mixed_switch_tol;   /* mixed mode: f32 phase stops at this residual; <=0 auto (1e-4, 1e-5 from a learned block) */
} si_config;

/* Per-call diagnostics. */
typedef struct si_report {
  int32_t level;             /* solver level reached (0..5), -1 if none            */
  int32_t iterations;        /* LOBPCG iterations over all passes                  */
  int32_t restarts;          /* warm restarts (src/solvers/lobpcg.rs:295-300)      */
  int32_t n_components_graph;/* connected components found                          */
  int32_t fp32_iterations;   /* iterations run in the f32 phase (mixed mode)       */
  int32_t spmm_calls;        /* operator applications                              */
  int32_t learned_start;     /* 1 when the accepted solve started from the learned block */
  int32_t reserved1;
  double max_residual;       /* level-gate residual (src/metrics.rs:73-92)         */
  double solve_ms;           /* device time of the eigensolve                      */
  double eigenvalues[16];    /* first min(k,16) eigenvalues of the accepted level  */
} si_report;

/* CSR graph (f32 weights) -- the crate's CsMatI<f32, u32, usize>. */
typedef struct si_csr_f32 {
  uint64_t n;                /* rows == cols */
  uint64_t nnz;
  const uint64_t* indptr;    /* [n+1] */
  const uint32_t* indices;   /* [nnz] sorted, unique within a row */
  const float* data;         /* [nnz] */
} si_csr_f32;

/* CSR f64 matrix with explicit diagonal -- the crate's CsMatI<f64, usize>
 * (the Laplacian handed to solve_eigenproblem). */
typedef struct si_csr_f64 {
  uint64_t n;
  uint64_t nnz;
  const uint64_t* indptr;
  const uint32_t* indices;
  const double* data;
} si_csr_f64;

/* Device operator: y = diag * x + sum_j values[ij] * x_j.  With diag == 1 and
 * values = -d_i^-1/2 w_ij d_j^-1/2 this is the normalised Laplacian with an
 * implicit unit diagonal (nnz entries instead of nnz + n). */
typedef struct si_operator {
  uint64_t n;
  uint64_t nnz;
  const uint64_t* indptr;    /* device [n+1] */
  const uint32_t* indices;   /* device [nnz] */
  const double* values;      /* device [nnz], f64                          */
  const float* values_f32;   /* device [nnz] or NULL (mixed-precision SpMM) */
  double diag;               /* coefficient of x_i                          */
} si_operator;

typedef struct si_ctx si_ctx;

/* ---- context -------------------------------------------------------------- */
void si_config_default(si_config* cfg);
int32_t si_abi_version(void);
/* Number of CUDA kernels this library has launched in this process
 * (diagnostics; no counterpart in the crate). */
uint64_t si_kernel_launches(void);
si_status si_ctx_create(int32_t device, si_ctx** out);
void si_ctx_destroy(si_ctx* ctx);
const char* si_last_error(const si_ctx* ctx);
/* Wait for all work queued on the context's stream. */
si_status si_ctx_synchronize(si_ctx* ctx);
/* Device-side stream of the context, as a cudaStream_t cast to void*. */
void* si_ctx_stream(si_ctx* ctx);

/* ---- full pipeline ---------------------------------------------------------- */
/* spectral_init (src/lib.rs:198-258).  graph: HOST CSR.  data: optional HOST
 * row-major f32 [n x n_features] (needed only when the graph has more than
 * 2*n_components connected components).  out: HOST f32 [n x n_components]. */
si_status si_spectral_init(si_ctx* ctx, const si_csr_f32* graph, uint32_t n_components,
                           uint64_t seed, const float* data, uint64_t n_features,
                           const si_config* cfg, float* out, si_report* report);

/* Same pipeline with every array already in DEVICE memory (graph arrays,
 * data and out are device pointers). */
si_status si_spectral_init_device(si_ctx* ctx, const si_csr_f32* graph, uint32_t n_components,
                                  uint64_t seed, const float* data, uint64_t n_features,
                                  const si_config* cfg, float* out, si_report* report);

/* ---- component calls (DEVICE pointers) ------------------------------------- */
/* compute_degrees (src/laplacian.rs:29-49): degrees and sqrt(degrees), f64 [n]. */
si_status si_compute_degrees(si_ctx* ctx, const si_csr_f32* graph, int32_t compute_mode,
                             double* degrees, double* sqrt_deg);

/* build_normalized_laplacian (src/laplacian.rs:60-88), implicit-diagonal form:
 * values[e] = -inv_sqrt_deg[i] * w_e * inv_sqrt_deg[j] for every stored entry
 * e = (i, j) of the graph (0 for self loops); the unit diagonal is implicit.
 * values_f32 may be NULL. */
si_status si_build_laplacian(si_ctx* ctx, const si_csr_f32* graph, const double* inv_sqrt_deg,
                             double* values, float* values_f32);

/* build_normalized_laplacian, explicit CSR exactly as the crate returns it:
 * sorted columns, unit diagonal inserted, self loops dropped.  Call first with
 * out_indices == NULL to get *out_nnz; then with arrays of that size. */
si_status si_build_laplacian_csr(si_ctx* ctx, const si_csr_f32* graph, const double* inv_sqrt_deg,
                                 uint64_t* out_indptr, uint32_t* out_indices, double* out_data,
                                 uint64_t* out_nnz);

/* The fuzzy-kNN graph the crate consumes, built from points the way its
 * fixture generator builds it (tests/generate_fixtures.py:70-182): exact
 * Euclidean kNN without the point itself (knn_indices i32 / knn_dists f32
 * [n x k]), umap-learn's smooth-kNN sigmas / rhos (f32 [n]), membership
 * strengths, the fuzzy union A + A^T - A.A^T and pruning below
 * max / n_epochs.  points: f64 [n x dims] row-major; the pruned graph goes to
 * indptr (u64 [n + 1]) / indices (u32) / data (f32) with room for `capacity`
 * entries (2 n k always suffices), its entry count to *nnz.  All device
 * pointers; k <= 32, dims <= 256; brute force (O(n^2 dims)). */
si_status si_fuzzy_graph(si_ctx* ctx, const double* points, uint64_t n, uint32_t dims, uint32_t k,
                         int32_t* knn_indices, float* knn_dists, float* sigmas, float* rhos, uint64_t* indptr,
                         uint32_t* indices, float* data, uint64_t capacity, uint64_t* nnz);

/* find_components (src/components.rs:7-44): labels numbered by the smallest
 * node of each component (BFS start order).  labels: device u32 [n]. */
si_status si_find_components(si_ctx* ctx, const si_csr_f32* graph, uint32_t* labels,
                             uint64_t* n_components);

/* LinearOperator::apply (src/operator.rs:7-12, :176-223): y = A x for row-major
 * blocks x, y [n x k] (device, f64). */
si_status si_spmm(si_ctx* ctx, const si_operator* op, const double* x, double* y, uint32_t k);

/* Same with f32 blocks and op->values_f32 (accumulation in f64). */
si_status si_spmm_f32(si_ctx* ctx, const si_operator* op, const float* x, float* y, uint32_t k);

/* A device operator prepared for repeated products (the crate's CsrOperator,
 * src/operator.rs:174-228, holds its matrix across LinearOperator::apply
 * calls): the row partitions of the tiled / gather / panel kernels are built
 * once; the sliced copy of the operator (the default kernel for operators the
 * autotuner times, about the size of the index and value arrays again) and the
 * panel kernel's x windows on first use, outside stream capture.  The
 * operator's arrays must stay allocated and unchanged while the plan lives,
 * and calls on one plan from several host threads must be serialised by the
 * caller (the first calls build that state). */
typedef struct si_operator_plan si_operator_plan;
si_status si_operator_plan_create(si_ctx* ctx, const si_operator* op, si_operator_plan** out);
void si_operator_plan_destroy(si_operator_plan* plan);
/* LinearOperator::apply on a prepared operator: y = A x, blocks [n x k]
 * (device, f64; the f32 form uses op->values_f32).  Asynchronous: queued on
 * the context's stream (si_ctx_synchronize waits). */
si_status si_spmm_planned(si_ctx* ctx, const si_operator_plan* plan, const double* x, double* y, uint32_t k);
si_status si_spmm_planned_f32(si_ctx* ctx, const si_operator_plan* plan, const float* x, float* y, uint32_t k);

/* solve_eigenproblem (src/solvers/mod.rs:70-224) on a device operator.
 * eigvals: HOST f64 [n_components+1]; eigvecs: DEVICE f64 [n x (n_components+1)];
 * sqrt_deg: DEVICE f64 [n] (trivial-vector hint).  *level receives 0..5. */
si_status si_solve_eigenproblem(si_ctx* ctx, const si_operator* op, uint32_t n_components,
                                uint64_t seed, const double* sqrt_deg, const si_config* cfg,
                                double* eigvals, double* eigvecs, int32_t* level,
                                si_report* report);

/* solve_eigenproblem_pub (src/lib.rs:67-75): HOST explicit f64 CSR Laplacian,
 * sqrt_deg = ones.  eigvals HOST [k], eigvecs HOST [n x k], k = n_components+1. */
si_status si_solve_eigenproblem_host(si_ctx* ctx, const si_csr_f64* laplacian, uint32_t n_components,
                                     uint64_t seed, const si_config* cfg, double* eigvals,
                                     double* eigvecs, int32_t* level, si_report* report);

/* lobpcg_solve (src/solvers/lobpcg.rs:227-465).  HOST explicit f64 CSR operator
 * and HOST sqrt_deg [n]; returns SI_CONVERGENCE_FAILURE where the crate
 * returns None.  eigvals HOST [k]; eigvecs HOST [n x k]; *restarts as the crate. */
si_status si_lobpcg_solve_host(si_ctx* ctx, const si_csr_f64* op, uint32_t n_components,
                               uint64_t seed, int32_t regularize, const double* sqrt_deg,
                               const si_config* cfg, double* eigvals, double* eigvecs,
                               int32_t* restarts, si_report* report);

/* rsvd_solve (src/solvers/rsvd.rs:135-213), HOST explicit f64 CSR Laplacian. */
si_status si_rsvd_solve_host(si_ctx* ctx, const si_csr_f64* laplacian, uint32_t n_components,
                             uint64_t seed, int32_t oversampling, int32_t nbiter,
                             double* eigvals, double* eigvecs);

/* dense_evd (src/solvers/dense.rs:9-46): k smallest eigenpairs of a HOST f64
 * CSR matrix, computed densely on the device. */
si_status si_dense_evd_host(si_ctx* ctx, const si_csr_f64* laplacian, uint32_t k,
                            double* eigvals, double* eigvecs);

/* normalize_signs (src/scaling.rs:62-74) on a DEVICE f64 block [n x k]. */
si_status si_normalize_signs(si_ctx* ctx, double* coords, uint64_t n, uint32_t k);

/* No counterpart in the reference.  The same sign normalisation as
 * si_normalize_signs on a DEVICE f64 block [n x k], for callers that cannot
 * let a library allocate device memory: a process whose HBM is already
 * reserved by another allocator (a serving engine or framework caching
 * allocator), or a latency-bound loop where an allocation or free on a shared
 * device may stall other streams.  It calls no cudaMalloc, cudaFree or pool
 * allocation: its temporaries live in one static device array of about
 * 513 KiB that every device loading the library holds until exit, which
 * limits k to 64 columns (larger k returns SI_INVALID_ARGUMENT); n is
 * unbounded.  The first call on a device looks up that array's device
 * address, so make it before any stream capture; the address is kept per CUDA
 * context, so after the device's context is re-created (cudaDeviceReset) the
 * next call looks it up again.  A column whose largest |x| (ranked as the
 * crate's f64::total_cmp ranks it, NaN highest) is a NaN keeps its signs, as
 * in the crate and in si_normalize_signs.  All calls on a device share
 * the array: calls that overlap on the GPU race and must be serialised by the
 * caller.  Returns after the stream has finished the work. */
si_status si_normalize_signs_noalloc(si_ctx* ctx, double* coords, uint64_t n, uint32_t k);

/* scale_and_add_noise (src/scaling.rs:78-89): DEVICE f64 [n x k] -> DEVICE f32
 * [n x k]: max-|.| scaled to 10, plus N(0, 1e-4) noise from `seed`. */
si_status si_scale_and_add_noise(si_ctx* ctx, const double* coords, uint64_t n, uint32_t k,
                                 uint64_t seed, float* out);

/* ---- learned warm start (no counterpart in the crate) ----------------------- */

/* The warm-start network: 3 message-passing layers (hidden width 64, bf16
 * weights, f32 accumulation) over the normalised adjacency, fed with the
 * square-root degree and 4 Chebyshev-filtered random probes per node, predicting
 * a 16-column block whose first k columns start LOBPCG.  Its parameters are a
 * flat f32 vector of si_model_param_count() values. */
typedef struct si_model si_model;
uint64_t si_model_param_count(void);
/* New model with He-initialised weights from `seed` on the context's device. */
si_status si_model_create(si_ctx* ctx, uint64_t seed, si_model** out);
void si_model_destroy(si_model* model);
si_status si_model_set_params(si_ctx* ctx, si_model* model, const float* params);  /* HOST [count] */
si_status si_model_get_params(si_ctx* ctx, si_model* model, float* params);        /* HOST [count] */
/* One Adam step (lr) of the subspace-projection loss on one graph.  op: DEVICE
 * Laplacian operator with f32 values; sqrt_deg: DEVICE [n]; target: DEVICE f64
 * [n x k] orthonormal eigenvectors (k <= 16); seed draws the random probes.
 * *loss (HOST) receives the loss before the step. */
si_status si_model_train_step(si_ctx* ctx, si_model* model, const si_operator* op, const double* sqrt_deg,
                              const double* target, uint32_t k, uint64_t seed, float lr, double* loss);
/* Loss and gradient (HOST [count]) without an update.  features: DEVICE f32
 * [n x 5] replacing the computed features, or NULL. */
si_status si_model_gradient(si_ctx* ctx, si_model* model, const si_operator* op, const double* sqrt_deg,
                            const float* features, const double* target, uint32_t k, uint64_t seed,
                            double* loss, float* grad);
/* Prediction Y: DEVICE f32 [n x 16].  features as for si_model_gradient. */
si_status si_model_predict(si_ctx* ctx, si_model* model, const si_operator* op, const double* sqrt_deg,
                           const float* features, uint64_t seed, float* out);
/* Model used by solves whose si_config.warm_start is SI_WARM_START_LEARNED
 * (NULL detaches).  The model must outlive its use by the context. */
si_status si_ctx_set_model(si_ctx* ctx, si_model* model);

/* Tensor-core building block of the warm-start network: C = A * B^T on the
 * DEVICE, A [m x k] and B [n x k] row-major bf16 (pitches lda, ldb in elements,
 * multiples of 8, 16-byte aligned), C [m x n] f32 with pitch ldc (multiple of 8;
 * == n when k_splits > 1).  n must be 16, 64 or 128.  k_splits > 1 splits the
 * k dimension across CTAs (for tall-skinny weight gradients). */
si_status si_gemm_bf16_nt(si_ctx* ctx, uint64_t m, uint32_t n, uint64_t k, const void* a, uint64_t lda,
                          const void* b, uint64_t ldb, float* c, uint64_t ldc, uint32_t k_splits);

#ifdef __cplusplus
}
#endif
#endif /* SPECTRAL_INIT_GPU_H */
