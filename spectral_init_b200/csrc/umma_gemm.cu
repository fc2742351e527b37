// BF16 tensor-core GEMM for the learned warm start: C = A * B^T with A [M x K]
// and B [N x K] both row-major bf16 (K contiguous), f32 accumulation in TMEM.
//
// One persistent CTA per SM, warp-specialised:
//   warp 0      TMA producer: 128 x 64 A tiles and N x 64 B tiles, 128-byte
//               swizzle, into a 4-stage shared-memory ring;
//   warp 1      allocates TMEM and issues tcgen05.mma (one thread), 4 MMAs of
//               K = 16 per stage, double-buffered accumulators (2 x N columns);
//   warps 2..5  epilogue: tcgen05.ld of the accumulator (warp w reads TMEM
//               lanes 32*(w%4) ..), fused bias / ReLU / bf16 conversion, store.
// Tiles are (128-row block, K split); with k_splits > 1 each split writes an
// f32 partial slab and a second kernel adds the slabs in split order.
// Ragged M and K edges read zeros (TMA out-of-bounds fill).
#include <cudaTypedefs.h>

#include <algorithm>
#include <mutex>

#include "umma.cuh"
#include "umma_gemm.h"

namespace si {

namespace {

constexpr int BM = 128;
constexpr int BK = 64;
constexpr int STAGES = 4;
constexpr int kGemmThreads = 192;

template <int BN>
struct GemmShape {
  static constexpr int a_bytes = BM * BK * 2;
  static constexpr int b_bytes = BN * BK * 2;
  static constexpr int tmem_cols = (2 * BN <= 32) ? 32 : (2 * BN <= 64) ? 64 : (2 * BN <= 128) ? 128 : 256;
  static constexpr int smem_bytes = 1024 + STAGES * (a_bytes + b_bytes) + 256;
};

__device__ __forceinline__ void store_chunk(const GemmEpilogue& ep, int64_t r, int c, int split, int64_t M,
                                            const float (&v)[16]) {
  if (ep.mode == GEMM_BIAS_RELU_BF16) {
    alignas(16) __nv_bfloat16 h[16];
#pragma unroll
    for (int i = 0; i < 16; ++i) {
      const float b = ep.bias != nullptr ? ep.bias[c + i] : 0.0f;
      h[i] = __float2bfloat16_rn(fmaxf(v[i] + b, 0.0f));
    }
    uint4* dst = reinterpret_cast<uint4*>(ep.out_bf16 + r * ep.ldo + c);
    dst[0] = reinterpret_cast<const uint4*>(h)[0];
    dst[1] = reinterpret_cast<const uint4*>(h)[1];
    return;
  }
  float* dst = ep.out_f32 + (static_cast<int64_t>(split) * M + r) * ep.ldo + c;
  const bool add_bias = ep.mode == GEMM_BIAS_F32 && ep.bias != nullptr;
  float w[16];
#pragma unroll
  for (int i = 0; i < 16; ++i) w[i] = v[i] + (add_bias ? ep.bias[c + i] : 0.0f);
#pragma unroll
  for (int i = 0; i < 4; ++i)
    reinterpret_cast<float4*>(dst)[i] = make_float4(w[4 * i], w[4 * i + 1], w[4 * i + 2], w[4 * i + 3]);
}

template <int BN>
__global__ void __launch_bounds__(kGemmThreads, 1)
    k_gemm_bf16(const __grid_constant__ CUtensorMap ta, const __grid_constant__ CUtensorMap tb, int64_t M,
                int64_t K, int m_tiles, int k_splits, int64_t k_per_split, GemmEpilogue ep, int* err) {
  using S = GemmShape<BN>;
  extern __shared__ uint8_t gemm_raw[];
  uint8_t* base = reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(gemm_raw) + 1023) & ~uintptr_t(1023));
  uint8_t* sA = base;
  uint8_t* sB = base + STAGES * S::a_bytes;
  uint64_t* full = reinterpret_cast<uint64_t*>(sB + STAGES * S::b_bytes);
  uint64_t* empty = full + STAGES;
  uint64_t* tfull = empty + STAGES;
  uint64_t* tempty = tfull + 2;
  uint64_t* drain = tempty + 2;
  uint32_t* tslot = reinterpret_cast<uint32_t*>(drain + 1);
  __shared__ volatile int s_abort;

  const int warp = threadIdx.x >> 5;
  const int lane = threadIdx.x & 31;
  if (threadIdx.x == 0) {
    for (int s = 0; s < STAGES; ++s) {
      umma::mbar_init(&full[s], 1);
      umma::mbar_init(&empty[s], 1);
    }
    for (int a = 0; a < 2; ++a) {
      umma::mbar_init(&tfull[a], 1);
      umma::mbar_init(&tempty[a], 128);
    }
    umma::mbar_init(drain, 1);
    umma::fence_mbar_init();
    s_abort = 0;
  }
  if (warp == 1) umma::tmem_alloc(tslot, S::tmem_cols);
  umma::fence_before_sync();
  __syncthreads();
  umma::fence_after_sync();
  const uint32_t tbase = *tslot;
  const int total = m_tiles * k_splits;

  if (warp == 0) {
    if (lane == 0) {
      umma::tma_prefetch_desc(&ta);
      umma::tma_prefetch_desc(&tb);
      uint32_t it = 0;
      bool ok = true;
      for (int tile = blockIdx.x; tile < total && ok; tile += gridDim.x) {
        const int mb = tile % m_tiles;
        const int split = tile / m_tiles;
        const int64_t k0 = split * k_per_split;
        const int64_t k1 = std::min<int64_t>(K, k0 + k_per_split);
        const int nch = static_cast<int>((k1 - k0 + BK - 1) / BK);
        for (int j = 0; j < nch; ++j, ++it) {
          const int s = it % STAGES;
          const uint32_t ph = (it / STAGES) & 1;
          if (!umma::mbar_wait(&empty[s], ph ^ 1)) {
            ok = false;
            break;
          }
          umma::mbar_arrive_expect_tx(&full[s], S::a_bytes + S::b_bytes);
          umma::tma_load_2d(sA + s * S::a_bytes, &ta, &full[s], static_cast<int32_t>(k0 + j * BK), mb * BM);
          umma::tma_load_2d(sB + s * S::b_bytes, &tb, &full[s], static_cast<int32_t>(k0 + j * BK), 0);
        }
        if (s_abort) ok = false;
      }
      if (!ok) s_abort = 1;
      // no copy may still be landing in shared memory when the CTA exits
      for (int s = 0; s < STAGES; ++s) {
        if (it <= static_cast<uint32_t>(s)) break;
        const uint32_t last = it - 1 - ((it - 1 - s) % STAGES);
        if (!umma::mbar_wait(&full[s], (last / STAGES) & 1)) s_abort = 1;
      }
    }
  } else if (warp == 1) {
    if (lane == 0) {
      const uint32_t idesc = umma::idesc_bf16_f32(BM, BN);
      uint32_t it = 0;
      int local = 0;
      bool ok = true;
      for (int tile = blockIdx.x; tile < total && ok; tile += gridDim.x, ++local) {
        const int split = tile / m_tiles;
        const int64_t k0 = split * k_per_split;
        const int64_t k1 = std::min<int64_t>(K, k0 + k_per_split);
        const int nch = static_cast<int>((k1 - k0 + BK - 1) / BK);
        const int acc = local & 1;
        if (!umma::mbar_wait(&tempty[acc], ((local >> 1) & 1) ^ 1)) {
          ok = false;
          break;
        }
        umma::fence_after_sync();
        const uint32_t d = tbase + acc * BN;
        for (int j = 0; j < nch; ++j, ++it) {
          const int s = it % STAGES;
          const uint32_t ph = (it / STAGES) & 1;
          if (!umma::mbar_wait(&full[s], ph)) {
            ok = false;
            break;
          }
          umma::fence_after_sync();
          const uint64_t ad = umma::smem_desc_k_sw128(sA + s * S::a_bytes);
          const uint64_t bd = umma::smem_desc_k_sw128(sB + s * S::b_bytes);
#pragma unroll
          for (int kk = 0; kk < BK / 16; ++kk)
            umma::mma_bf16(d, ad + 2 * kk, bd + 2 * kk, idesc, (j | kk) != 0 ? 1u : 0u);
          umma::mma_commit(&empty[s]);
        }
        if (!ok) break;
        umma::mma_commit(&tfull[acc]);
        if (s_abort) ok = false;
      }
      if (!ok) s_abort = 1;
      umma::mma_commit(drain);
      if (!umma::mbar_wait(drain, 0)) s_abort = 1;
    }
  } else {
    const int q = warp & 3;
    const int row = q * 32 + lane;
    int local = 0;
    bool ok = true;
    for (int tile = blockIdx.x; tile < total; tile += gridDim.x, ++local) {
      const int mb = tile % m_tiles;
      const int split = tile / m_tiles;
      const int acc = local & 1;
      bool got = umma::mbar_wait(&tfull[acc], (local >> 1) & 1);
      got = __all_sync(0xffffffffu, got);
      if (!got) {
        ok = false;
        break;
      }
      umma::fence_after_sync();
      const int64_t r = static_cast<int64_t>(mb) * BM + row;
      const uint32_t taddr = tbase + (static_cast<uint32_t>(q * 32) << 16) + acc * BN;
#pragma unroll 1
      for (int c = 0; c < BN; c += 16) {
        float v[16];
        umma::tmem_ld16(taddr + c, v);
        if (r < M) store_chunk(ep, r, c, split, M, v);
      }
      umma::fence_before_sync();
      umma::mbar_arrive(&tempty[acc]);
      if (__any_sync(0xffffffffu, s_abort != 0)) {
        ok = false;
        break;
      }
    }
    if (!ok) s_abort = 1;
  }
  __syncthreads();
  if (threadIdx.x == 0 && s_abort) atomicExch(err, 1);
  if (warp == 1) {
    umma::fence_after_sync();
    umma::tmem_dealloc(tbase, S::tmem_cols);
  }
}

__global__ void k_sum_splits(const float* __restrict__ part, int splits, int64_t count, float* __restrict__ out,
                             const float* __restrict__ bias, int n_cols) {
  const int64_t stride = static_cast<int64_t>(gridDim.x) * blockDim.x;
  for (int64_t e = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; e < count; e += stride) {
    float s = 0.0f;
    for (int k = 0; k < splits; ++k) s += part[static_cast<int64_t>(k) * count + e];
    if (bias != nullptr) s += bias[e % n_cols];
    out[e] = s;
  }
}

}  // namespace

PFN_cuTensorMapEncodeTiled_v12000 tensor_map_encoder() {
  static std::once_flag once;
  static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
  std::call_once(once, [] {
    cudaDriverEntryPointQueryResult q;
    void* p = nullptr;
    const cudaError_t rc = cudaGetDriverEntryPointByVersion("cuTensorMapEncodeTiled", &p, 12000, cudaEnableDefault, &q);
    if (rc == cudaSuccess && q == cudaDriverEntryPointSuccess)
      fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
  });
  SI_REQUIRE(fn != nullptr, SI_CUDA_ERROR, "cuTensorMapEncodeTiled is not available from the driver");
  return fn;
}

namespace {

// 2-D bf16 tensor map over rows x cols (row pitch ld elements), box 64 x box_rows.
CUtensorMap make_map(const __nv_bfloat16* ptr, int64_t rows, int64_t cols, int64_t ld, int box_rows) {
  SI_REQUIRE(reinterpret_cast<uintptr_t>(ptr) % 16 == 0, SI_INVALID_ARGUMENT, "gemm: operand not 16-byte aligned");
  SI_REQUIRE((ld * 2) % 16 == 0, SI_INVALID_ARGUMENT, "gemm: row pitch must be a multiple of 8 elements");
  SI_REQUIRE(ld >= cols, SI_INVALID_ARGUMENT, "gemm: row pitch smaller than the row");
  CUtensorMap map;
  const cuuint64_t dims[2] = {static_cast<cuuint64_t>(cols), static_cast<cuuint64_t>(rows)};
  const cuuint64_t strides[1] = {static_cast<cuuint64_t>(ld * 2)};
  const cuuint32_t box[2] = {static_cast<cuuint32_t>(BK), static_cast<cuuint32_t>(box_rows)};
  const cuuint32_t estr[2] = {1, 1};
  const CUresult r = tensor_map_encoder()(&map, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 2, const_cast<__nv_bfloat16*>(ptr), dims,
                                 strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B,
                                 CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  SI_REQUIRE(r == CUDA_SUCCESS, SI_CUDA_ERROR, "cuTensorMapEncodeTiled failed (" + std::to_string(int(r)) + ")");
  return map;
}

template <int BN>
void launch_gemm(const Exec& ex, int64_t M, int64_t K, const __nv_bfloat16* A, int64_t lda, const __nv_bfloat16* B,
                 int64_t ldb, const GemmEpilogue& ep, int k_splits, int64_t k_per_split, int* err) {
  using S = GemmShape<BN>;
  static std::once_flag attr_once[64];
  SI_REQUIRE(ex.device >= 0 && ex.device < 64, SI_INVALID_ARGUMENT, "gemm: device ordinal");
  cudaError_t attr_rc = cudaSuccess;
  std::call_once(attr_once[ex.device], [&] {
    attr_rc = cudaFuncSetAttribute(k_gemm_bf16<BN>, cudaFuncAttributeMaxDynamicSharedMemorySize, S::smem_bytes);
  });
  SI_CUDA(attr_rc);
  const CUtensorMap ta = make_map(A, M, K, lda, BM);
  const CUtensorMap tb = make_map(B, BN, K, ldb, BN);
  const int m_tiles = static_cast<int>((M + BM - 1) / BM);
  const int total = m_tiles * k_splits;
  const int grid = std::max(1, std::min(total, ex.sms));
  k_gemm_bf16<BN><<<grid, kGemmThreads, S::smem_bytes, ex.stream>>>(ta, tb, M, K, m_tiles, k_splits, k_per_split,
                                                                     ep, err);
  SI_LAUNCH_CHECK();
}

}  // namespace

void gemm_bf16_nt(const Exec& ex, int64_t M, int N, int64_t K, const __nv_bfloat16* A, int64_t lda,
                  const __nv_bfloat16* B, int64_t ldb, const GemmEpilogue& ep, int k_splits, GemmWorkspace& ws) {
  SI_REQUIRE(N == 16 || N == 64 || N == 128, SI_INVALID_ARGUMENT, "gemm: N must be 16, 64 or 128");
  SI_REQUIRE(M >= 0 && K >= 0, SI_INVALID_ARGUMENT, "gemm: negative size");
  if (M == 0) return;
  SI_REQUIRE(K > 0, SI_INVALID_ARGUMENT, "gemm: K must be positive");
  SI_REQUIRE(ep.ldo >= N && ep.ldo % 8 == 0, SI_INVALID_ARGUMENT,
             "gemm: output pitch must be >= N and a multiple of 8");
  k_splits = std::max(1, k_splits);
  const int64_t chunks = (K + BK - 1) / BK;
  const int64_t chunks_per_split = (chunks + k_splits - 1) / k_splits;
  k_splits = static_cast<int>((chunks + chunks_per_split - 1) / chunks_per_split);
  const int64_t k_per_split = chunks_per_split * BK;
  if (ws.err.size() < 1) {
    ws.err.alloc(1, ex.stream);
    ws.err.zero();
  }
  GemmEpilogue kep = ep;
  if (k_splits > 1) {
    SI_REQUIRE(ep.mode == GEMM_STORE_F32 || ep.mode == GEMM_BIAS_F32, SI_INVALID_ARGUMENT,
               "gemm: split-K needs an f32 output");
    SI_REQUIRE(ep.ldo == N, SI_INVALID_ARGUMENT, "gemm: split-K output must be dense (ldo == N)");
    const size_t need = static_cast<size_t>(k_splits) * M * N;
    if (ws.partial.size() < need) ws.partial.alloc(need, ex.stream);
    kep.mode = GEMM_STORE_F32;
    kep.out_f32 = ws.partial.get();
    kep.ldo = N;
  }
  switch (N) {
    case 16: launch_gemm<16>(ex, M, K, A, lda, B, ldb, kep, k_splits, k_per_split, ws.err.get()); break;
    case 64: launch_gemm<64>(ex, M, K, A, lda, B, ldb, kep, k_splits, k_per_split, ws.err.get()); break;
    default: launch_gemm<128>(ex, M, K, A, lda, B, ldb, kep, k_splits, k_per_split, ws.err.get()); break;
  }
  if (k_splits > 1) {
    const int64_t count = M * N;
    const int grid = static_cast<int>(std::max<int64_t>(1, std::min<int64_t>((count + 255) / 256, ex.sms * 4)));
    k_sum_splits<<<grid, 256, 0, ex.stream>>>(ws.partial.get(), k_splits, count, ep.out_f32,
                                              ep.mode == GEMM_BIAS_F32 ? ep.bias : nullptr, N);
    SI_LAUNCH_CHECK();
  }
}

void gemm_check(const Exec& ex, GemmWorkspace& ws) {
  if (ws.err.size() < 1) return;
  int h = 0;
  SI_CUDA(cudaMemcpyAsync(&h, ws.err.get(), sizeof(int), cudaMemcpyDeviceToHost, ex.stream));
  SI_CUDA(cudaStreamSynchronize(ex.stream));
  SI_REQUIRE(h == 0, SI_CUDA_ERROR, "tensor-core GEMM pipeline timed out (a wait exceeded its limit)");
}

}  // namespace si
