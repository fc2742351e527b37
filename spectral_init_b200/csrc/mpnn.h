// Learned warm start: the message-passing network's device state and passes.
#pragma once

#include "si_internal.h"
#include "umma_gemm.h"

namespace si {

constexpr int kMpnnFeatures = 5;   // sqrt-degree + 4 filtered probes
constexpr int kMpnnHidden = 64;
constexpr int kMpnnCat = 128;      // [H | Ahat H]
constexpr int kMpnnOut = 16;       // predicted columns (first k used)
constexpr int kMpnnLayers = 3;

int64_t mpnn_param_count();

// Parameters (f32 master copy, Adam moments) and the bf16 operands of the GEMMs.
struct MpnnModel {
  DevBuf<float> params, grad, m1, m2;
  DevBuf<__nv_bfloat16> wt;  // per layer [N x 128]  (forward B operand)
  DevBuf<__nv_bfloat16> w;   // per layer [128 x N]  (backward B operand)
  int64_t step = 0;
  void init(const Exec& ex, uint64_t seed);
  void sync_weights(const Exec& ex);
  void set(const Exec& ex, const float* host);
  void get(const Exec& ex, float* host) const;
};

// Activations of one graph: A_l = [H_l | Ahat H_l] (bf16 [n x 128]) and Y (f32 [n x 16]).
struct MpnnActs {
  int64_t n = 0, npad = 0;
  DevBuf<__nv_bfloat16> a[kMpnnLayers + 1];
  DevBuf<float> y;
  void ensure(const Exec& ex, int64_t n);
};

// H0 from the operator (Ahat = -offdiag of the Laplacian, f32 values) or from
// given device features [n x 5] (f32, already scaled).
void mpnn_features(const Exec& ex, const OpDev& op, const double* sqrt_deg, uint64_t seed, const float* given,
                   MpnnActs& acts);
void mpnn_forward(const Exec& ex, const MpnnModel& model, const OpDev& op, MpnnActs& acts, GemmWorkspace& ws);
// Subspace loss against target (device f64 [n x k], pitch vld); fills model.grad.
double mpnn_loss_backward(const Exec& ex, MpnnModel& model, const OpDev& op, MpnnActs& acts, const double* target,
                          int vld, int k, GemmWorkspace& ws);
void mpnn_adam(const Exec& ex, MpnnModel& model, float lr);

}  // namespace si
