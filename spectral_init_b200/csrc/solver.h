// Eigensolver drivers (host C++ orchestrating the device kernels).
#pragma once

#include <functional>
#include <vector>

#include "si_internal.h"

namespace si {

struct SolverConfig {
  int block_size = 0;         // 0 = auto
  int dense_threshold = 2000; // Level 0 for n < this
  int force_level = -1;
  int rsvd_oversampling = -1;
  int rsvd_nbiter = 2;
  int max_iterations = 0;     // 0 = crate caps
  int precision = SI_PRECISION_FP64;
  double tol = 1e-5;
  double mixed_switch_tol = 0.0;
  // warm start: optional device block [n x ld_ws] (f64) replacing the random start
  const double* warm_start = nullptr;
  int warm_start_ld = 0;
  // learned warm start: writes a predicted block into columns [0, k) of the
  // device f64 block x [n x ld]; false falls back to the random start
  std::function<bool(const Exec& ex, const OpDev& op, const double* sqrt_deg, int k, uint64_t seed, double* x,
                     int ld)>
      learned_start;
  bool learned_chebyshev = false;  // also apply the Chebyshev start filter to the learned block
};

struct SolverStats {
  int learned_used = 0;  // the accepted solve started from the learned block
  int level = -1;
  int iterations = 0;
  int restarts = 0;
  int fp32_iterations = 0;
  int spmm_calls = 0;
  int sinv_cg_capped = 0;  // level-2 inner solves that stopped at their iteration cap
  double max_residual = 0.0;
};

// Eigenpairs on the device: vals host [k], vecs device [n x k] row-major.
struct EigenResult {
  std::vector<double> vals;
  DevBuf<double> vecs;
  int k = 0;
};

// lobpcg_solve (src/solvers/lobpcg.rs:227-465).  Returns false where the
// crate returns None.
bool lobpcg_solve_dev(const Exec& ex, const OpDev& op, int n_components, uint64_t seed, bool regularize,
                      const double* sqrt_deg, const SolverConfig& cfg, EigenResult& out, SolverStats& st);

// Subspace width K of rsvd_solve: n_components + 1 + oversampling, or the
// crate's default oversampling (src/solvers/rsvd.rs:84-87) when it is < 0.
int rsvd_width(int64_t n, int n_components, int oversampling);

// rsvd_solve (src/solvers/rsvd.rs:135-213).  K above the device small-problem
// limit (64) is an SI_INVALID_ARGUMENT error, not a silently narrower subspace.
void rsvd_solve_dev(const Exec& ex, const OpDev& op, int n_components, uint64_t seed, int oversampling, int nbiter,
                    EigenResult& out, SolverStats& st);

// dense_evd (src/solvers/dense.rs:9-46): k smallest pairs.
void dense_evd_result(const Exec& ex, const OpDev& op, int k, EigenResult& out);

// max_eigenpair_residual (src/metrics.rs:73-92) on the device.
double max_eigenpair_residual_dev(const Exec& ex, const OpDev& op, const EigenResult& r);
std::vector<double> eigenpair_residuals_dev(const Exec& ex, const OpDev& op, const double* vecs, int ld,
                                            const std::vector<double>& vals, int k, double floor);

// solve_eigenproblem (src/solvers/mod.rs:70-224).
void solve_eigenproblem_dev(const Exec& ex, const OpDev& op, int n_components, uint64_t seed, const double* sqrt_deg,
                            const SolverConfig& cfg, EigenResult& out, SolverStats& st);

}  // namespace si
