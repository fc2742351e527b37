// Sign normalisation (src/scaling.rs:62-74) that allocates no device memory.
//
// Every other entry point of the library takes its temporary device buffers
// from the stream-ordered pool (cudaMallocAsync).  Some callers cannot let a
// library allocate: a process whose device memory is already reserved by
// another allocator (a serving engine or a framework caching allocator that
// has claimed nearly all of HBM, where a further allocation fails or
// fragments the reservation), or a latency-bound loop on a shared device
// where an allocation or a free may stall other streams.  For them the
// per-column argmax partials, the ticket counter and the sign vector live in
// one file-scope device array below, fixed in size and held by every device
// that loads the library until the process exits.
//
// The array is shared by every call on a device and keeps what the last call
// left in it; calls whose kernels overlap on the GPU (two threads, two
// contexts or two streams on the same device) race on it and must be
// serialised by the caller.  The first call on a device looks up the array's
// device address (cudaGetSymbolAddress with that device current, which may
// load the module there), so that call should come before any stream capture.
// The address is cached per CUDA context, not per device ordinal: if the
// device's primary context is destroyed and created again (cudaDeviceReset by
// the host program or another library), the module is loaded anew, the array
// moves, and the next call looks its address up again.
// Limit: k <= 64 columns; any n.
//
// Column maximum as the crate ranks it: |x| compared with f64::total_cmp, so
// a NaN (whose |.| has the sign bit clear) ranks above +inf, NaNs rank by
// payload, and ties keep the first row; a column whose maximum is a NaN is
// never flipped (signum(NaN) = NaN is not < 0).
#include <cuda.h>

#include <algorithm>
#include <mutex>

#include "si_internal.h"

namespace si {

namespace {

constexpr int kNaThreads = 256;
constexpr int kNaMaxCtas = 512;

// Layout of the scratch array.  Only `ticket` must be zero when the argmax
// kernel starts (it is cleared before every launch); the partials are written
// by every CTA before the last one reads them, and `sign` is written by that
// CTA before the apply kernel reads it.
struct SignScratch {
  long long val[kNaMaxCtas * kNoAllocMaxCols];
  long long idx[kNaMaxCtas * kNoAllocMaxCols];
  double sign[kNoAllocMaxCols];
  unsigned ticket;
};

static __device__ __align__(256) unsigned char g_sign_scratch[sizeof(SignScratch)];

constexpr int kMaxDevices = 64;
std::mutex g_addr_mu;
struct AddrEntry {
  unsigned long long ctx_id = 0;  // context the address belongs to (0: none yet)
  void* ptr = nullptr;
};
AddrEntry g_addr[kMaxDevices];

using CtxGetCurrentFn = CUresult (*)(CUcontext*);
using CtxGetIdFn = CUresult (*)(CUcontext, unsigned long long*);

// Identifier of the calling thread's current CUDA context (unique for the
// life of the process; a re-created primary context gets a new one).
unsigned long long current_context_id() {
  static std::once_flag once;
  static CtxGetCurrentFn get_current = nullptr;
  static CtxGetIdFn get_id = nullptr;
  std::call_once(once, [] {
    cudaDriverEntryPointQueryResult q;
    void* p = nullptr;
    if (cudaGetDriverEntryPointByVersion("cuCtxGetCurrent", &p, 12000, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      get_current = reinterpret_cast<CtxGetCurrentFn>(p);
    p = nullptr;
    if (cudaGetDriverEntryPointByVersion("cuCtxGetId", &p, 12000, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      get_id = reinterpret_cast<CtxGetIdFn>(p);
  });
  SI_REQUIRE(get_current != nullptr && get_id != nullptr, SI_CUDA_ERROR,
             "normalize_signs_noalloc: cuCtxGetCurrent / cuCtxGetId are not available from the driver");
  CUcontext c = nullptr;
  unsigned long long id = 0;
  SI_REQUIRE(get_current(&c) == CUDA_SUCCESS && c != nullptr, SI_CUDA_ERROR,
             "normalize_signs_noalloc: no current CUDA context");
  SI_REQUIRE(get_id(c, &id) == CUDA_SUCCESS && id != 0, SI_CUDA_ERROR,
             "normalize_signs_noalloc: cuCtxGetId failed");
  return id;
}

// Device address of the scratch array in the current context of `device`
// (the array's host-side name is not a device address).  Looked up once per
// context: the first call on a device, and again after that device's context
// was re-created.
SignScratch* scratch_address(int device) {
  SI_REQUIRE(device >= 0 && device < kMaxDevices, SI_INVALID_ARGUMENT,
             "normalize_signs_noalloc: device ordinal beyond the supported 64 devices");
  const unsigned long long ctx = current_context_id();
  std::lock_guard<std::mutex> lock(g_addr_mu);
  AddrEntry& e = g_addr[device];
  if (e.ptr == nullptr || e.ctx_id != ctx) {
    void* p = nullptr;
    SI_CUDA(cudaGetSymbolAddress(&p, g_sign_scratch));
    SI_REQUIRE(p != nullptr, SI_CUDA_ERROR, "normalize_signs_noalloc: scratch symbol has no device address");
    e.ptr = p;
    e.ctx_id = ctx;
  }
  return static_cast<SignScratch*>(e.ptr);
}

// Key of |x| whose unsigned order is f64::total_cmp on |x| (the sign bit of
// |x| is clear, so NaNs sort above +inf by payload); -1 marks "no row".
__device__ __forceinline__ long long abs_key(double v) {
  return __double_as_longlong(v) & 0x7fffffffffffffffLL;
}

__device__ __forceinline__ bool better(long long a2, long long i2, long long a1, long long i1) {
  return i2 >= 0 && (a2 > a1 || (a2 == a1 && (i1 < 0 || i2 < i1)));
}

// Per column c of a contiguous [n x k] block: the first row of largest |x|,
// then the sign of x there (Rust f64::signum: -1 for negatives and -0.0).
// Thread t of a CTA owns column t % k and rows t / k + R * (CTA + grid * j)
// with R = 256 / k rows per CTA, so a warp reads consecutive elements.
__global__ void __launch_bounds__(kNaThreads) k_argmax_abs_rows(const double* __restrict__ x, int64_t n, int k,
                                                                SignScratch* __restrict__ s) {
  __shared__ long long sv[kNaThreads];
  __shared__ long long sx[kNaThreads];
  __shared__ bool last;
  const int t = threadIdx.x;
  const int R = kNaThreads / k;
  const int c = t % k;
  const int r = t / k;
  long long best = -1;
  long long bi = -1;
  if (r < R) {
    const int64_t step = static_cast<int64_t>(gridDim.x) * R;
    int64_t i = static_cast<int64_t>(blockIdx.x) * R + r;
    for (; i + 3 * step < n; i += 4 * step) {
      long long a[4];
#pragma unroll
      for (int u = 0; u < 4; ++u) a[u] = abs_key(__ldg(x + (i + u * step) * k + c));
#pragma unroll
      for (int u = 0; u < 4; ++u)
        if (a[u] > best) {
          best = a[u];
          bi = i + u * step;
        }
    }
    for (; i < n; i += step) {
      const long long a = abs_key(__ldg(x + i * k + c));
      if (a > best) {
        best = a;
        bi = i;
      }
    }
  }
  sv[t] = best;
  sx[t] = bi;
  __syncthreads();
  // tree over the rows of each column: slot r combines with slot r + h
  for (int h = 1; h < R; h <<= 1) {
    if (r < R && (r % (2 * h)) == 0 && r + h < R) {
      const int o = t + h * k;
      if (better(sv[o], sx[o], sv[t], sx[t])) {
        sv[t] = sv[o];
        sx[t] = sx[o];
      }
    }
    __syncthreads();
  }
  if (t < k) {
    s->val[static_cast<int64_t>(blockIdx.x) * kNoAllocMaxCols + t] = sv[t];
    s->idx[static_cast<int64_t>(blockIdx.x) * kNoAllocMaxCols + t] = sx[t];
  }
  __threadfence();
  __syncthreads();
  if (t == 0) last = (atomicAdd(&s->ticket, 1u) == gridDim.x - 1);
  __syncthreads();
  if (!last) return;
  __threadfence();
  if (t < k) {
    long long b = -1;
    long long ib = -1;
    for (int blk = 0; blk < static_cast<int>(gridDim.x); ++blk) {
      const long long a = __ldcg(&s->val[static_cast<int64_t>(blk) * kNoAllocMaxCols + t]);
      const long long i = __ldcg(&s->idx[static_cast<int64_t>(blk) * kNoAllocMaxCols + t]);
      if (better(a, i, b, ib)) {
        b = a;
        ib = i;
      }
    }
    // Rust f64::signum: -1 for negatives and -0.0, NaN (never flipped) for NaN
    const double v = ib >= 0 ? x[ib * k + t] : 1.0;
    s->sign[t] = (!isnan(v) && signbit(v)) ? -1.0 : 1.0;
  }
  if (t == 0) s->ticket = 0u;
}

__global__ void __launch_bounds__(kNaThreads) k_apply_signs_rows(double* __restrict__ x, int64_t n, int k,
                                                                 const SignScratch* __restrict__ s) {
  __shared__ double sg[kNoAllocMaxCols];
  if (threadIdx.x < k) sg[threadIdx.x] = s->sign[threadIdx.x];
  __syncthreads();
  const int64_t total = n * k;
  const int64_t stride = static_cast<int64_t>(gridDim.x) * blockDim.x;
  for (int64_t e = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; e < total; e += stride)
    if (sg[e % k] < 0.0) x[e] = -x[e];
}

}  // namespace

void normalize_signs_noalloc_dev(const Exec& ex, double* x, int64_t n, int k) {
  SI_REQUIRE(k >= 0 && k <= kNoAllocMaxCols, SI_INVALID_ARGUMENT,
             "normalize_signs_noalloc: k = " + std::to_string(k) + " columns exceeds the maximum of " +
                 std::to_string(kNoAllocMaxCols) + " held by the static scratch");
  SI_REQUIRE(n >= 0 && (k == 0 || n <= (INT64_MAX / 2) / k), SI_INVALID_ARGUMENT,
             "normalize_signs_noalloc: n x k overflows a 64-bit element index");
  if (n == 0 || k == 0) return;
  SI_REQUIRE(x != nullptr, SI_INVALID_ARGUMENT, "normalize_signs_noalloc: coords is null");
  SignScratch* s = scratch_address(ex.device);
  const int rows_per_cta = kNaThreads / k;
  const int64_t need = (n + rows_per_cta - 1) / rows_per_cta;
  const int grid = static_cast<int>(std::max<int64_t>(
      1, std::min<int64_t>({need, static_cast<int64_t>(ex.sms) * 2, static_cast<int64_t>(kNaMaxCtas)})));
  SI_CUDA(cudaMemsetAsync(&s->ticket, 0, sizeof(unsigned), ex.stream));
  k_argmax_abs_rows<<<grid, kNaThreads, 0, ex.stream>>>(x, n, k, s);
  SI_LAUNCH_CHECK();
  const int64_t items = (n * k + kNaThreads - 1) / kNaThreads;
  const int agrid = static_cast<int>(std::max<int64_t>(1, std::min<int64_t>(items, int64_t(ex.sms) * 8)));
  k_apply_signs_rows<<<agrid, kNaThreads, 0, ex.stream>>>(x, n, k, s);
  SI_LAUNCH_CHECK();
}

}  // namespace si
