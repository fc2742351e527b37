// tcgen05 BF16 GEMM (umma_gemm.cu): C = A * B^T, A [M x K] and B [N x K]
// row-major bf16 (pitches lda, ldb in elements, multiples of 8, 16-byte
// aligned), f32 accumulation; N in {16, 64, 128}.
#pragma once

#include <cuda_bf16.h>
#include <cudaTypedefs.h>

#include "si_internal.h"

namespace si {

enum GemmMode { GEMM_STORE_F32 = 0, GEMM_BIAS_F32 = 1, GEMM_BIAS_RELU_BF16 = 2 };

struct GemmEpilogue {
  int mode = GEMM_STORE_F32;
  float* out_f32 = nullptr;           // f32 modes: [M x ldo]
  __nv_bfloat16* out_bf16 = nullptr;  // GEMM_BIAS_RELU_BF16: [M x ldo]
  int64_t ldo = 0;
  const float* bias = nullptr;        // [N] or null
};

struct GemmWorkspace {
  DevBuf<float> partial;
  DevBuf<int> err;  // set by a kernel whose pipeline wait timed out
};

// k_splits > 1 splits K across CTAs (f32 modes, ldo == N) and adds the slabs in order.
void gemm_bf16_nt(const Exec& ex, int64_t M, int N, int64_t K, const __nv_bfloat16* A, int64_t lda,
                  const __nv_bfloat16* B, int64_t ldb, const GemmEpilogue& ep, int k_splits, GemmWorkspace& ws);
// The driver's cuTensorMapEncodeTiled (looked up once); throws if unavailable.
PFN_cuTensorMapEncodeTiled_v12000 tensor_map_encoder();

// Synchronises the stream and throws if a GEMM launched with ws reported a timeout.
void gemm_check(const Exec& ex, GemmWorkspace& ws);

}  // namespace si
