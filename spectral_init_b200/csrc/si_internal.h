// Internal declarations shared by the translation units of the library.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <memory>
#include <string>
#include <vector>

#include "si_common.cuh"
#include "spectral_init_gpu.h"

namespace si {

// Execution resources of a call: the context's stream and device facts.
struct Exec {
  cudaStream_t stream = nullptr;
  int sms = 148;
  int device = 0;
};

// CSR graph on the device (f32 weights).
struct GraphDev {
  int64_t n = 0, nnz = 0;
  const uint64_t* indptr = nullptr;
  const uint32_t* indices = nullptr;
  const float* data = nullptr;
};

struct RowBlocks;

// Sparse operator y = diag * x + sum_j v_ij x_j on the device.
struct OpDev {
  int64_t n = 0, nnz = 0;
  const uint64_t* indptr = nullptr;
  const uint32_t* indices = nullptr;
  const double* v64 = nullptr;
  const float* v32 = nullptr;
  double diag = 1.0;
  // optional row partition for the tiled SpMM: block b covers rows
  // [row_blocks[b], row_blocks[b+1]) (about kSpmmBlockNnz entries each)
  const int64_t* row_blocks = nullptr;
  const uint64_t* block_ptr = nullptr;  // indptr[row_blocks[b]]
  int64_t n_blocks = 0;
  // finer partition (about kGatherBlockNnz entries) for the TMA-gather SpMM
  const int64_t* gather_blocks = nullptr;
  const uint64_t* gather_ptr = nullptr;
  int64_t n_gather_blocks = 0;
  // panel partition (about kPanelBlockNnz entries a block) and its per-block
  // x windows, built on demand for each window size (null: not available)
  const RowBlocks* panels = nullptr;
};

constexpr int kSpmmBlockNnz = 1024;   // target entries per row block
constexpr int kSpmmBlockCap = 2048;   // entries a block may hold in shared memory
constexpr int kSpmmBlockRows = 1024;  // rows a block may hold in shared memory
constexpr int kGatherBlockNnz = 384;  // target entries per TMA-gather block
constexpr int kGatherCap = 512;       // entries a TMA-gather block may stage
constexpr int kPanelBlockNnz = 4096;  // target entries per panel block
constexpr int kPanelBytes = 200 * 1024;  // shared memory of the staged x window

// x window of the panel SpMM for one window size: block b gathers x rows
// [w0[b], w0[b] + W) from shared memory.
struct PanelWindows {
  int W = 0;
  DevBuf<int64_t> w0;
};

// Sliced-ELL copy of an operator for the sliced SpMM.  Rows of up to
// `long_min - 1` entries are sorted by length (longest first) inside windows
// of kSellSortRows consecutive rows and cut into slices of 32; slot (s, j, r),
// at slice_ptr[s] + 32 j + r, holds entry j of row perm[32 s + r]
// (plen[32 s + r] entries; slots past a row's length hold index 0 and value 0,
// lanes without a row have perm = 0xffffffff).  A slice is as wide as its
// longest row.  Rows of long_min or more entries are listed in long_rows
// (window order) and read from the CSR arrays by a whole warp each.
constexpr int kSellSortRows = 4096;
constexpr int kSellSortThreads = 1024;
constexpr int kSellMaxShort = 1024;  // long_min never exceeds this + 1
struct SellLayout {
  int64_t n_slices = 0, n_long = 0;
  uint64_t slots = 0;
  int long_min = 0;
  DevBuf<uint64_t> slice_ptr;  // n_slices + 1
  DevBuf<uint32_t> perm, plen, idx, long_rows;
  DevBuf<float> v32;
  DevBuf<double> v64;
};

// Row partition of an operator for the tiled SpMM (device array of
// n_blocks + 1 row starts, owned by the caller).
struct RowBlocks {
  DevBuf<int64_t> starts, gstarts, pstarts;
  DevBuf<uint64_t> ptrs, gptrs, pptrs;
  int64_t n_blocks = 0, n_gblocks = 0, n_pblocks = 0;
  // windows of the panel SpMM, one entry per window size used (built lazily
  // by the first SpMM that needs them outside stream capture)
  mutable std::vector<PanelWindows> windows;
  // sliced-ELL copy (built lazily outside stream capture, only when sell_ok:
  // owners that apply the operator many times with unchanged values)
  bool sell_ok = false;
  mutable std::unique_ptr<SellLayout> sell;
  mutable bool sell_failed = false;
  void attach(OpDev& op) const {
    op.row_blocks = starts.get();
    op.block_ptr = ptrs.get();
    op.n_blocks = n_blocks;
    op.gather_blocks = gstarts.get();
    op.gather_ptr = gptrs.get();
    op.n_gather_blocks = n_gblocks;
    op.panels = this;
  }
};
void make_row_blocks(const Exec& ex, const OpDev& op, RowBlocks& rb);

// Epilogue of an SpMM: out = alpha * (A x) + beta * z1 + gamma * z2 + delta * z3
// (z pointers share the layout of y; a null z contributes nothing).
template <class XT>
struct Epilogue {
  double alpha = 1.0, beta = 0.0, gamma = 0.0, delta = 0.0;
  const XT* z1 = nullptr;
  const XT* z2 = nullptr;
  const XT* z3 = nullptr;
};

// ---- laplacian.cu ---------------------------------------------------------
void validate_graph(const Exec& ex, const GraphDev& g);
bool graph_is_symmetric(const Exec& ex, const GraphDev& g);
void compute_degrees_dev(const Exec& ex, const GraphDev& g, int mode, double* deg, double* sqrt_deg);
void inv_sqrt_dev(const Exec& ex, const double* sqrt_deg, int64_t n, double* inv);
void laplacian_values_dev(const Exec& ex, const GraphDev& g, const double* inv_sqrt_deg, double* v64,
                          float* v32);
uint64_t laplacian_csr_nnz_dev(const Exec& ex, const GraphDev& g);
void laplacian_csr_dev(const Exec& ex, const GraphDev& g, const double* inv_sqrt_deg, uint64_t* out_indptr,
                       uint32_t* out_indices, double* out_data);
// Explicit f64 CSR (diagonal stored) -> operator with diag coefficient 0.
OpDev op_from_csr64(const uint64_t* indptr, const uint32_t* indices, const double* data, int64_t n, int64_t nnz);
// Exclusive scan of u64 counts (device), returns the total.
uint64_t exclusive_scan_u64(const Exec& ex, const uint64_t* in, uint64_t* out, int64_t n);

// ---- fuzzy.cu --------------------------------------------------------------------
// The fuzzy-kNN graph from f64 points [n x d] (exact kNN, smooth-kNN,
// memberships, fuzzy union, pruning); see si_fuzzy_graph.
void fuzzy_graph_dev(const Exec& ex, const double* x, int64_t n, int d, int k, int32_t* knn_idx, float* knn_dist,
                     float* sigma, float* rho, uint64_t* indptr, uint32_t* indices, float* data, uint64_t capacity,
                     uint64_t* nnz_out);

// ---- components.cu --------------------------------------------------------
int64_t find_components_dev(const Exec& ex, const GraphDev& g, uint32_t* labels);

// ---- spmm.cu ----------------------------------------------------------------
// y = epilogue(A x) for row-major blocks with row stride ld (ld in {4,8,16}
// uses the vectorised kernels; any other ld the generic one over k columns).
template <class XT>
void spmm_dev(const Exec& ex, const OpDev& op, const XT* x, XT* y, int ld, int k, const Epilogue<XT>& ep,
              const int* stop = nullptr, bool use_f32_values = false);
// Rows per group chosen for the operator's degree profile.
int spmm_group_lanes(const OpDev& op);

// ---- block_ops.cu -----------------------------------------------------------
constexpr int MAXM = 16;   // widest LOBPCG block
constexpr int SMAX = 64;   // widest small dense problem (rSVD subspace)

// Gram products over row-major blocks [n x ld] (first m columns used).
//  mode SYM2: S = blk[0..ns), AS = blk[ns..2ns); out = [S^T S ; S^T AS]
//             as two symmetric (ns*m)^2 matrices stacked (upper triangle
//             computed, mirrored).
//  mode FULL: out = S^T T with S = blk[0..ns), T = blk[ns..nblk), full.
enum GramMode { GRAM_SYM2 = 0, GRAM_FULL = 1 };
struct GramWork {
  DevBuf<double> partial;
  DevBuf<unsigned> counter;
  void ensure(size_t partial_count, cudaStream_t s);
};
template <class XT>
void gram_dev(const Exec& ex, GramWork& w, GramMode mode, const XT* const* blk, int ns, int nblk, int m,
              int ld, int64_t n, double* out, const int* stop = nullptr);

// out = sum_b in_b * C_b  (C_b: m_in x m_out, row stride cstride, device),
// blocks with row stride ld.  out must not alias an input.
template <class XT>
void combine_dev(const Exec& ex, const XT* const* in, const double* const* coef, int nin, XT* out, int m_in,
                 int m_out, int cstride, int ld, int64_t n);

// Column norms: out[c] = || a_c - lam_c b_c ||_2 (b may be null -> ||a_c||).
template <class XT>
void column_residual_norms_dev(const Exec& ex, GramWork& w, const XT* a, const XT* b, const double* lam_dev,
                               int m, int ld, int64_t n, double* out_dev);

// Fill [n x ld] with N(0,1) in the first m columns, zeros elsewhere.
template <class XT>
void fill_normal_dev(const Exec& ex, XT* x, int64_t n, int m, int ld, uint64_t seed, uint64_t stream);
// Column 0 <- v / ||v|| when ||v|| > 0 (v: f64 [n]).
template <class XT>
void set_column_normalized_dev(const Exec& ex, GramWork& w, XT* x, int ld, int64_t n, const double* v);
// Scale columns: x[:, c] *= s[c] (s device, length m).
template <class XT>
void scale_columns_dev(const Exec& ex, XT* x, int64_t n, int m, int ld, const double* s);
// Gather columns: out[i, j] = in[i, cols[j]] (cols host list, <= MAXM).
template <class XI, class XO>
void gather_columns_dev(const Exec& ex, const XI* in, int ld_in, XO* out, int ld_out, int64_t n,
                        const std::vector<int>& cols);
// Sign convention (first max-|.| element positive) on [n x k] f64, stride ld.
void normalize_signs_dev(const Exec& ex, GramWork& w, double* x, int64_t n, int k, int ld);
// Global max |x| of [n x k] f64.
double max_abs_dev(const Exec& ex, GramWork& w, const double* x, int64_t n, int k, int ld);
// out_f32 = (f32)(x * expansion) + 1e-4 * N(0,1) (f32), per element.
void scale_noise_dev(const Exec& ex, const double* x, int64_t n, int k, int ld, double expansion,
                     uint64_t seed, float* out, bool add_noise);
// x[:, :] += shift[c] per column (multi-component translate) ; generic axpy helpers.
void copy_strided_dev(const Exec& ex, const double* in, int ld_in, double* out, int ld_out, int64_t n, int k);

// ---- small_dense.cu -----------------------------------------------------------
enum SmallMode { SM_INIT = 0, SM_ITER = 1, SM_RR_PLAIN = 2, SM_CHOLQR = 3 };
enum LobpcgStatus { ST_RUNNING = 0, ST_CONVERGED = 1, ST_MAXITER = 2, ST_BREAKDOWN = 3 };

struct LobpcgCtrl {
  int m, k_wanted, maxiter, largest;
  double tol, chol_tol;
  int iter, done, status, has_p;
  int copy_best, mode, best_iter, n_active;
  int p_valid;  // P holds a search direction from a previous update
  int pad_;
  int active[MAXM];
  double lam[MAXM];
  double rnorm[MAXM];
  double best_sum;
  double best_lam[MAXM];
  double best_rnorm[MAXM];
  double Cx[MAXM * MAXM];
  double Cr[MAXM * MAXM];
  double Cp[MAXM * MAXM];
};

// One CTA: the small dense step of a LOBPCG iteration (or an init / plain
// Rayleigh-Ritz / CholQR step).  gram: output of gram_dev SYM2 with ns blocks.
void small_step_dev(const Exec& ex, LobpcgCtrl* ctrl, const double* gram, int ns, int mode, int m);
// Plain symmetric eigensolve / CholQR of an s x s matrix on the device (s <= SMAX):
//   SM_RR_PLAIN: a (s x s) -> evals[s] ascending, evecs (s x s, columns)
//   SM_CHOLQR:   a = B (s x s) -> evecs = L^-T (upper), evals[0] = 1 on success, 0 on failure
void small_dense_dev(const Exec& ex, const double* a, int s, int mode, double* evals, double* evecs);

// ---- lobpcg update (block_ops.cu) ----------------------------------------------
template <class XT>
struct LobpcgBlocks {
  XT* X;
  XT* R;
  XT* P;
  XT* AX;
  XT* AR;
  XT* AP;
  XT* Xbest;
};
template <class XT>
void lobpcg_update_dev(const Exec& ex, const LobpcgBlocks<XT>& b, const LobpcgCtrl* ctrl, int ld, int64_t n,
                       int init_mode);

// ---- cg.cu -----------------------------------------------------------------------
// Block CG on M Y = B (M symmetric positive definite, the operator with its
// diagonal coefficient), one CG per column; returns the iterations run.
struct CgWork {
  DevBuf<double> r, p, q, partial;
  DevBuf<unsigned> counter;
  DevBuf<unsigned char> scal;
};
// *converged (optional) tells whether every column reached rtol within maxit.
int cg_solve_block_dev(const Exec& ex, const OpDev& M, const double* b, double* y, int m, int ld, int64_t n,
                       double rtol, int maxit, CgWork& w, bool* converged = nullptr);

// ---- noalloc.cu -----------------------------------------------------------------
// Sign normalisation of a contiguous f64 block [n x k] with all temporaries in
// a static device array (no allocation); k <= kNoAllocMaxCols.
constexpr int kNoAllocMaxCols = 64;
void normalize_signs_noalloc_dev(const Exec& ex, double* x, int64_t n, int k);

// ---- dense_evd.cu ---------------------------------------------------------------
// k smallest eigenpairs of the dense symmetric matrix of an operator
// (explicit CSR or implicit-diagonal form).  evals host [k], evecs device
// [n x ld] (first k columns), ascending.
void dense_evd_dev(const Exec& ex, const OpDev& op, int k, double* evals_host, double* evecs, int ld);

}  // namespace si
