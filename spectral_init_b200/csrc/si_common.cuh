// Shared internals of the sm_100a spectral-init library: error handling,
// stream-ordered device buffers, the Philox4x32-10 counter RNG and warp /
// block reductions.
#pragma once

#include <cuda_runtime.h>

#include <atomic>
#include <cstdint>
#include <stdexcept>
#include <string>
#include <utility>

#include "spectral_init_gpu.h"

namespace si {

// ---------------------------------------------------------------------------
// Errors.  Internal C++ code throws si::Error; every extern "C" entry point
// catches it and turns it into an si_status plus a message.
// ---------------------------------------------------------------------------
struct Error : std::runtime_error {
  si_status code;
  Error(si_status c, const std::string& m) : std::runtime_error(m), code(c) {}
};

#define SI_CUDA(call)                                                                   \
  do {                                                                                  \
    cudaError_t e_ = (call);                                                            \
    if (e_ != cudaSuccess)                                                              \
      throw ::si::Error(e_ == cudaErrorMemoryAllocation ? SI_OUT_OF_MEMORY : SI_CUDA_ERROR, \
                        std::string(#call) + ": " + cudaGetErrorString(e_) + " (" +     \
                            __FILE__ + ":" + std::to_string(__LINE__) + ")");           \
  } while (0)

// Kernels launched by this library in this process (diagnostics export).
extern std::atomic<uint64_t> g_kernel_launches;
// launches made by the calling host thread (graph-capture accounting)
extern thread_local uint64_t tl_kernel_launches;

#define SI_LAUNCH_CHECK()                                            \
  do {                                                               \
    ::si::g_kernel_launches.fetch_add(1, std::memory_order_relaxed); \
    ++::si::tl_kernel_launches;                                      \
    SI_CUDA(cudaGetLastError());                                     \
  } while (0)

#define SI_REQUIRE(cond, code, msg)            \
  do {                                         \
    if (!(cond)) throw ::si::Error(code, msg); \
  } while (0)

// ---------------------------------------------------------------------------
// Stream-ordered device buffer (cudaMallocAsync pool allocations).
// ---------------------------------------------------------------------------
template <class T>
class DevBuf {
 public:
  DevBuf() = default;
  DevBuf(size_t count, cudaStream_t s) { alloc(count, s); }
  ~DevBuf() { release(); }
  DevBuf(const DevBuf&) = delete;
  DevBuf& operator=(const DevBuf&) = delete;
  DevBuf(DevBuf&& o) noexcept { swap(o); }
  DevBuf& operator=(DevBuf&& o) noexcept {
    if (this != &o) {
      release();
      swap(o);
    }
    return *this;
  }
  void alloc(size_t count, cudaStream_t s) {
    release();
    stream_ = s;
    count_ = count;
    if (count) SI_CUDA(cudaMallocAsync(reinterpret_cast<void**>(&ptr_), count * sizeof(T), s));
  }
  void zero() {
    if (count_) SI_CUDA(cudaMemsetAsync(ptr_, 0, count_ * sizeof(T), stream_));
  }
  void release() noexcept {
    if (ptr_) cudaFreeAsync(ptr_, stream_);
    ptr_ = nullptr;
    count_ = 0;
  }
  T* get() const { return ptr_; }
  size_t size() const { return count_; }

 private:
  void swap(DevBuf& o) {
    std::swap(ptr_, o.ptr_);
    std::swap(count_, o.count_);
    std::swap(stream_, o.stream_);
  }
  T* ptr_ = nullptr;
  size_t count_ = 0;
  cudaStream_t stream_ = nullptr;
};

// ---------------------------------------------------------------------------
// Philox4x32-10 (Salmon, Moraes, Dror, Shaw: "Parallel random numbers: as easy
// as 1, 2, 3", SC'11) and Box-Muller normals.
// ---------------------------------------------------------------------------
struct U4 {
  uint32_t x, y, z, w;
};

__host__ __device__ inline U4 philox4x32_10(U4 c, uint32_t k0, uint32_t k1) {
  const uint32_t M0 = 0xD2511F53u, M1 = 0xCD9E8D57u;
  const uint32_t W0 = 0x9E3779B9u, W1 = 0xBB67AE85u;
#pragma unroll
  for (int r = 0; r < 10; ++r) {
    const uint64_t p0 = static_cast<uint64_t>(M0) * c.x;
    const uint64_t p1 = static_cast<uint64_t>(M1) * c.z;
    const uint32_t hi0 = static_cast<uint32_t>(p0 >> 32), lo0 = static_cast<uint32_t>(p0);
    const uint32_t hi1 = static_cast<uint32_t>(p1 >> 32), lo1 = static_cast<uint32_t>(p1);
    c = U4{hi1 ^ c.y ^ k0, lo1, hi0 ^ c.w ^ k1, lo0};
    k0 += W0;
    k1 += W1;
  }
  return c;
}

// Two standard normals (f64) for counter `idx` of stream `stream` under `seed`.
// Uniforms use 53 random bits each and lie strictly inside (0, 1).
__device__ inline void philox_normal2(uint64_t seed, uint64_t stream, uint64_t idx, double& z0,
                                      double& z1) {
  U4 c{static_cast<uint32_t>(idx), static_cast<uint32_t>(idx >> 32), static_cast<uint32_t>(stream),
       static_cast<uint32_t>(stream >> 32)};
  U4 r = philox4x32_10(c, static_cast<uint32_t>(seed), static_cast<uint32_t>(seed >> 32));
  const uint64_t a = (static_cast<uint64_t>(r.x) << 21) ^ (r.y >> 11);
  const uint64_t b = (static_cast<uint64_t>(r.z) << 21) ^ (r.w >> 11);
  const double u1 = (static_cast<double>(a & ((1ull << 53) - 1)) + 0.5) * 0x1.0p-53;
  const double u2 = (static_cast<double>(b & ((1ull << 53) - 1)) + 0.5) * 0x1.0p-53;
  const double rad = sqrt(-2.0 * log(u1));
  double s, co;
  sincospi(2.0 * u2, &s, &co);
  z0 = rad * co;
  z1 = rad * s;
}

// ---------------------------------------------------------------------------
// Reductions.
// ---------------------------------------------------------------------------
__device__ inline double warp_sum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

__device__ inline double warp_max(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
  return v;
}

inline int ceil_div(int64_t a, int64_t b) { return static_cast<int>((a + b - 1) / b); }

template <class T>
struct VecTraits;
template <>
struct VecTraits<double> {
  static constexpr bool is_f32 = false;
};
template <>
struct VecTraits<float> {
  static constexpr bool is_f32 = true;
};

}  // namespace si
