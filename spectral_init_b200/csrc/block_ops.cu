// Dense block kernels of the eigensolvers: tall-skinny Gram products,
// block combinations, the fused LOBPCG update, column norms, the seeded
// starting block, and the selection / sign / scaling steps of the pipeline
// (src/selection.rs:11-29, src/scaling.rs:9-89).
//
// All reductions are deterministic: every CTA writes its partial sums, and
// the last CTA to finish (atomic ticket) adds them in CTA order.
#include <algorithm>
#include <string>
#include <cstdlib>
#include <vector>

#include "si_internal.h"

namespace si {

void GramWork::ensure(size_t partial_count, cudaStream_t s) {
  if (partial.size() < partial_count) partial.alloc(partial_count, s);
  if (counter.size() < 1) {
    counter.alloc(1, s);
    counter.zero();
  }
}

namespace {

constexpr int GT = 256;         // threads per Gram CTA
constexpr int GTR = 32;         // rows per smem tile
constexpr int GEPT = 17;        // entries per thread (covers a 64 x 64 full product)
constexpr int GMAXE = GT * GEPT;
constexpr int GMAXW = 8 * MAXM; // widest tile row (8 blocks of 16)

template <class XT>
struct GramParams {
  const XT* blk[8];
  int nblk, ns, m, ld, mode, ne, P, Q;
  int64_t n;
  double* partial;
  double* out;
  unsigned* counter;
  const int* stop;
};

// entry e -> (tile column a, tile column b, out index, mirrored out index)
__device__ inline void gram_entry(int mode, int P, int Q, int e, int& a, int& b, int& o1, int& o2) {
  if (mode == GRAM_FULL) {
    a = e / Q;
    b = P + e % Q;
    o1 = e;
    o2 = -1;
    return;
  }
  const int half = P * (P + 1) / 2;
  const int which = e >= half ? 1 : 0;
  int r = which ? e - half : e;
  int i = 0;
  while (r >= P - i) {
    r -= P - i;
    ++i;
  }
  const int j = i + r;
  a = i;
  b = which ? P + j : j;
  o1 = which * P * P + i * P + j;
  o2 = which * P * P + j * P + i;
}

template <class XT>
__global__ void __launch_bounds__(GT) k_gram(GramParams<XT> p) {
  if (p.stop != nullptr && *p.stop != 0) return;
  __shared__ double tile[GTR][GMAXW + 1];
  __shared__ bool last;
  const int tid = threadIdx.x;
  int ea[GEPT], eb[GEPT];
  double acc[GEPT];
  int cnt = 0;
#pragma unroll
  for (int q = 0; q < GEPT; ++q) {
    const int e = tid + q * GT;
    acc[q] = 0.0;
    ea[q] = 0;
    eb[q] = 0;
    if (e < p.ne) {
      int o1, o2;
      gram_entry(p.mode, p.P, p.Q, e, ea[q], eb[q], o1, o2);
      cnt = q + 1;
    }
  }
  const int width = p.nblk * p.m;
  const int64_t ntiles = (p.n + GTR - 1) / GTR;
  for (int64_t t = blockIdx.x; t < ntiles; t += gridDim.x) {
    const int64_t row0 = t * GTR;
    for (int idx = tid; idx < GTR * width; idx += GT) {
      const int b = idx / (GTR * p.m);
      const int rem = idx % (GTR * p.m);
      const int r = rem / p.m;
      const int c = rem % p.m;
      const int64_t row = row0 + r;
      tile[r][b * p.m + c] = row < p.n ? static_cast<double>(p.blk[b][row * p.ld + c]) : 0.0;
    }
    __syncthreads();
#pragma unroll 4
    for (int r = 0; r < GTR; ++r) {
#pragma unroll
      for (int q = 0; q < GEPT; ++q)
        if (q < cnt) acc[q] = fma(tile[r][ea[q]], tile[r][eb[q]], acc[q]);
    }
    __syncthreads();
  }
  // partials entry-major: the finishing CTA reads each entry's partials coalesced
#pragma unroll
  for (int q = 0; q < GEPT; ++q)
    if (q < cnt) p.partial[static_cast<int64_t>(tid + q * GT) * gridDim.x + blockIdx.x] = acc[q];
  __threadfence();
  __syncthreads();
  if (tid == 0) last = (atomicAdd(p.counter, 1u) == gridDim.x - 1);
  __syncthreads();
  if (!last) return;
  __threadfence();
  const int warp = tid >> 5, lane = tid & 31;
  for (int e = warp; e < p.ne; e += GT / 32) {
    const double* pe = p.partial + static_cast<int64_t>(e) * gridDim.x;
    double s = 0.0;
    for (int c = lane; c < static_cast<int>(gridDim.x); c += 32) s += pe[c];
    s = warp_sum(s);
    if (lane == 0) {
      int a, b, o1, o2;
      gram_entry(p.mode, p.P, p.Q, e, a, b, o1, o2);
      p.out[o1] = s;
      if (o2 >= 0) p.out[o2] = s;
    }
  }
  if (tid == 0) *p.counter = 0u;
}

// ---------------------------------------------------------------------------
// Gram of one LOBPCG iteration for 4-column blocks:
//   G = S^T [S AS],  S = [X R P], AS = [AX AR AP]  (12 x 24).
// Rows stream through shared memory in 64-row tiles with cp.async double
// buffering; each lane owns a 3 x 3 register tile of G (lane = 8 * a + b:
// S columns 3a..3a+2 against T columns 3b..3b+2), so a warp covers all 288
// entries of a row with six shared loads per lane.  Accumulation is f64 (the
// product of two f32 values is exact in f64).
__device__ __forceinline__ void cp_async16(void* smem, const void* gmem, int src_bytes) {
  const unsigned s = static_cast<unsigned>(__cvta_generic_to_shared(smem));
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(s), "l"(gmem), "r"(src_bytes));
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::); }
template <int N>
__device__ __forceinline__ void cp_async_wait() {
  asm volatile("cp.async.wait_group %0;\n" ::"n"(N));
}

constexpr int G4_TR = 128;    // rows per pipeline stage
constexpr int G4_STAGES = 3;  // cp.async stages in flight
constexpr int G4_THREADS = 512;
constexpr int G4_WARPS = G4_THREADS / 32;

template <class XT>
constexpr size_t gram4_smem_bytes() {
  return static_cast<size_t>(G4_STAGES) * G4_TR * 24 * sizeof(XT);
}
static_assert(gram4_smem_bytes<float>() >= sizeof(double) * G4_WARPS * 288,
              "the stage memory must hold the per-warp reduction buffer");

template <class XT>
__global__ void __launch_bounds__(G4_THREADS) k_gram4(const XT* __restrict__ X, const XT* __restrict__ R,
                                               const XT* __restrict__ P, const XT* __restrict__ AX,
                                               const XT* __restrict__ AR, const XT* __restrict__ AP, int64_t n,
                                               double* __restrict__ partial, const int* __restrict__ stop) {
  if (stop != nullptr && *stop != 0) return;
  // stages of [G4_TR][24] rows; after the main loop the same memory holds the
  // per-warp reduction buffer red[G4_WARPS][288] (f64)
  extern __shared__ __align__(16) unsigned char gram4_raw[];
  XT (*tile)[G4_TR][24] = reinterpret_cast<XT (*)[G4_TR][24]>(gram4_raw);
  double (*red)[288] = reinterpret_cast<double (*)[288]>(gram4_raw);
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int ai = 3 * (lane >> 3);  // S column base
  const int bj = 3 * (lane & 7);   // T column base
  double acc[3][3];
#pragma unroll
  for (int p = 0; p < 3; ++p)
#pragma unroll
    for (int q = 0; q < 3; ++q) acc[p][q] = 0.0;
  const XT* src[6] = {X, R, P, AX, AR, AP};
  constexpr int EPC = 16 / sizeof(XT);          // elements per 16-byte chunk
  constexpr int CPB = 4 / EPC;                  // chunks per (row, block)
  constexpr int NCH = G4_TR * 6 * CPB;
  const int64_t ntiles = (n + G4_TR - 1) / G4_TR;
  auto load_tile = [&](int64_t t, int buf) {
    if (t < ntiles) {
      const int64_t row0 = t * G4_TR;
      for (int c = tid; c < NCH; c += G4_THREADS) {
        const int b = c / (G4_TR * CPB);
        const int rem = c % (G4_TR * CPB);
        const int r = rem / CPB, h = rem % CPB;
        const int64_t row = row0 + r;
        const bool ok = row < n;
        cp_async16(&tile[buf][r][b * 4 + h * EPC], src[b] + (ok ? row : 0) * 4 + h * EPC, ok ? 16 : 0);
      }
    }
    cp_async_commit();  // empty groups keep the group count uniform
  };
  const int64_t step = gridDim.x;
  int64_t t = blockIdx.x;
#pragma unroll
  for (int s0 = 0; s0 < G4_STAGES - 1; ++s0) load_tile(t + s0 * step, s0);
  int buf = 0;
  for (; t < ntiles; t += step) {
    load_tile(t + (G4_STAGES - 1) * step, (buf + G4_STAGES - 1) % G4_STAGES);
    cp_async_wait<G4_STAGES - 1>();
    __syncthreads();
#pragma unroll 4
    for (int r = warp; r < G4_TR; r += G4_WARPS) {
      const XT* row = tile[buf][r];
      const double s0 = static_cast<double>(row[ai]), s1 = static_cast<double>(row[ai + 1]),
                   s2 = static_cast<double>(row[ai + 2]);
      const double t0 = static_cast<double>(row[bj]), t1 = static_cast<double>(row[bj + 1]),
                   t2 = static_cast<double>(row[bj + 2]);
      acc[0][0] = fma(s0, t0, acc[0][0]);
      acc[0][1] = fma(s0, t1, acc[0][1]);
      acc[0][2] = fma(s0, t2, acc[0][2]);
      acc[1][0] = fma(s1, t0, acc[1][0]);
      acc[1][1] = fma(s1, t1, acc[1][1]);
      acc[1][2] = fma(s1, t2, acc[1][2]);
      acc[2][0] = fma(s2, t0, acc[2][0]);
      acc[2][1] = fma(s2, t1, acc[2][1]);
      acc[2][2] = fma(s2, t2, acc[2][2]);
    }
    __syncthreads();
    buf = (buf + 1) % G4_STAGES;
  }
  cp_async_wait<0>();
  __syncthreads();
#pragma unroll
  for (int p = 0; p < 3; ++p)
#pragma unroll
    for (int q = 0; q < 3; ++q) red[warp][(ai + p) * 24 + bj + q] = acc[p][q];
  __syncthreads();
  // one partial per entry and CTA (CTA-major); k_gram4_reduce adds them
  for (int e = tid; e < 288; e += G4_THREADS) {
    double sum = 0.0;
#pragma unroll
    for (int w = 0; w < G4_WARPS; ++w) sum += red[w][e];
    partial[static_cast<int64_t>(blockIdx.x) * 288 + e] = sum;
  }
}

// Task-split Gram of a 4-column LOBPCG iteration.  Only the upper triangles
// of S^T S and S^T AS are needed (156 of the 288 products a row of [S AS]
// offers), so each of the CTA's four warps owns one share and computes it for
// every row, one row per lane:
//   warp 0: X^T [X R P]      (i in X, j >= i)    42 products from 12 values
//   warp 1: [R P]^T [R P]    (i in R P, j >= i)  36 products from  8 values
//   warp 2: X^T [AX AR AP]   (i in X, j >= i)    42 products from 16 values
//   warp 3: [R P]^T [AR AP]  (i in R P, j >= i)  36 products from 16 values
// A tile of 128 rows of the six blocks is loaded with coalesced 16-byte loads
// (one warp reads 32 consecutive rows of one block), converted to f64 once
// and stored with a row stride of 25 doubles, so a warp's 32 rows of one
// column fall in distinct banks.  Accumulators stay in registers across all
// tiles of the CTA; at the end each warp sums its lanes and the CTA writes
// one 288-entry partial (the k_gram4 layout, unused entries zero) that
// k_gram4_reduce adds in CTA order.
constexpr int GT_TR = 128;
constexpr int GT_STRIDE = 25;
constexpr int GT_THREADS = 128;

template <int TASK>
struct GramTask;
template <>
struct GramTask<0> { static constexpr int I0 = 0, I1 = 4, TOFF = 0, N = 42; };
template <>
struct GramTask<1> { static constexpr int I0 = 4, I1 = 12, TOFF = 0, N = 36; };
template <>
struct GramTask<2> { static constexpr int I0 = 0, I1 = 4, TOFF = 12, N = 42; };
template <>
struct GramTask<3> { static constexpr int I0 = 4, I1 = 12, TOFF = 12, N = 36; };

template <int TASK>
__device__ __forceinline__ void gram_task_row(const double* __restrict__ row, double (&acc)[42]) {
  using T = GramTask<TASK>;
  double s[12], t[12];
#pragma unroll
  for (int i = T::I0; i < 12; ++i) s[i] = row[i];
  if constexpr (T::TOFF != 0) {
#pragma unroll
    for (int j = T::I0; j < 12; ++j) t[j] = row[T::TOFF + j];
  }
  int e = 0;
#pragma unroll
  for (int i = T::I0; i < T::I1; ++i) {
#pragma unroll
    for (int j = i; j < 12; ++j) {
      const double tj = (T::TOFF != 0) ? t[j] : s[j];
      acc[e] = fma(s[i], tj, acc[e]);
      ++e;
    }
  }
}

template <int TASK>
__device__ __forceinline__ void gram_task_store(const double (&acc)[42], double* red) {
  using T = GramTask<TASK>;
  int e = 0;
#pragma unroll
  for (int i = T::I0; i < T::I1; ++i) {
#pragma unroll
    for (int j = i; j < 12; ++j) {
      red[i * 24 + T::TOFF + j] = acc[e];
      ++e;
    }
  }
}

template <class XT>
__global__ void __launch_bounds__(GT_THREADS) k_gram4t(const XT* __restrict__ X, const XT* __restrict__ R,
                                                        const XT* __restrict__ P, const XT* __restrict__ AX,
                                                        const XT* __restrict__ AR, const XT* __restrict__ AP,
                                                        int64_t n, double* __restrict__ partial,
                                                        const int* __restrict__ stop) {
  if (stop != nullptr && *stop != 0) return;
  __shared__ double tile[GT_TR * GT_STRIDE];
  __shared__ double red[288];
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const XT* src[6] = {X, R, P, AX, AR, AP};
  double acc[42];
#pragma unroll
  for (int e = 0; e < 42; ++e) acc[e] = 0.0;
  for (int e = tid; e < 288; e += GT_THREADS) red[e] = 0.0;
  constexpr int EPC = 16 / sizeof(XT);  // elements per 16-byte load
  constexpr int CPR = 4 / EPC;          // loads per (row, block)
  const int64_t ntiles = (n + GT_TR - 1) / GT_TR;
  for (int64_t tl = blockIdx.x; tl < ntiles; tl += gridDim.x) {
    const int64_t row0 = tl * GT_TR;
    // load: chunk c = (block b, half h, row r), rows fastest so a warp reads
    // 32 consecutive rows of one block
#pragma unroll 4
    for (int c = tid; c < 6 * CPR * GT_TR; c += GT_THREADS) {
      const int r = c % GT_TR;
      const int bh = c / GT_TR;
      const int b = bh / CPR, h = bh % CPR;
      const int64_t row = row0 + r;
      double v[EPC];
      if (row < n) {
        if constexpr (sizeof(XT) == 4) {
          const float4 q = __ldcs(reinterpret_cast<const float4*>(src[b] + row * 4));
          v[0] = q.x;
          v[1] = q.y;
          v[2] = q.z;
          v[3] = q.w;
        } else {
          const double2 q = __ldcs(reinterpret_cast<const double2*>(src[b] + row * 4 + h * 2));
          v[0] = q.x;
          v[1] = q.y;
        }
      } else {
#pragma unroll
        for (int u = 0; u < EPC; ++u) v[u] = 0.0;
      }
#pragma unroll
      for (int u = 0; u < EPC; ++u) tile[r * GT_STRIDE + b * 4 + h * EPC + u] = v[u];
    }
    __syncthreads();
#pragma unroll 1
    for (int r = lane; r < GT_TR; r += 32) {
      const double* row = tile + r * GT_STRIDE;
      switch (warp) {
        case 0: gram_task_row<0>(row, acc); break;
        case 1: gram_task_row<1>(row, acc); break;
        case 2: gram_task_row<2>(row, acc); break;
        default: gram_task_row<3>(row, acc); break;
      }
    }
    __syncthreads();
  }
  // sum each accumulator over the warp's lanes (fixed butterfly order)
#pragma unroll
  for (int e = 0; e < 42; ++e) {
    double v = acc[e];
#pragma unroll
    for (int o = 16; o >= 1; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    acc[e] = v;
  }
  if (lane == 0) {
    switch (warp) {
      case 0: gram_task_store<0>(acc, red); break;
      case 1: gram_task_store<1>(acc, red); break;
      case 2: gram_task_store<2>(acc, red); break;
      default: gram_task_store<3>(acc, red); break;
    }
  }
  __syncthreads();
  for (int e = tid; e < 288; e += GT_THREADS) partial[static_cast<int64_t>(blockIdx.x) * 288 + e] = red[e];
}

bool gram4_old_forced() {
  const char* e = std::getenv("SPECTRAL_INIT_GRAM");
  return e != nullptr && std::string(e) == "tile";
}

// Adds the per-CTA partials of k_gram4 in CTA order (warp w takes CTAs w,
// w + 8, ..., then the warp sums in warp order) and writes both
// (4 ns_out) x (4 ns_out) matrices (upper triangles mirrored); ns_out = 1
// keeps only the first block of S and of AS (the Gram of X and AX alone).
__global__ void __launch_bounds__(256) k_gram4_reduce(const double* __restrict__ partial, int nparts, int ns_out,
                                                      double* __restrict__ out, const int* __restrict__ stop) {
  if (stop != nullptr && *stop != 0) return;
  __shared__ double red[8][32];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int e = blockIdx.x * 32 + lane;
  double sum = 0.0;
  if (e < 288)
    for (int c = warp; c < nparts; c += 8) sum += partial[static_cast<int64_t>(c) * 288 + e];
  red[warp][lane] = sum;
  __syncthreads();
  if (warp != 0 || e >= 288) return;
  double v = 0.0;
#pragma unroll
  for (int w = 0; w < 8; ++w) v += red[w][lane];
  const int i = e / 24, j = e % 24;
  const int h = j / 12, jj = j % 12;  // h = 0: S^T S, h = 1: S^T AS
  const int P = 4 * ns_out;
  if (i > jj || i >= P || jj >= P) return;
  out[h * P * P + i * P + jj] = v;
  out[h * P * P + jj * P + i] = v;
}

// ---------------------------------------------------------------------------
// Gram of one LOBPCG iteration for 8- and 16-column blocks (row width LD,
// any m <= LD wanted columns):
//   G1 = S^T S,  G2 = S^T AS  (upper triangles, mirrored),  S = [X R P].
// Each 3LD x 3LD product is cut into 8 x 8 tiles of TS x TS entries
// (TS = 3LD / 8); the 36 upper tiles of the two products are 72 register
// tiles, one per thread of a row group.  A CTA has 7 row groups (504
// threads: 16 warps, so 128 registers a thread fit each SM sub-partition's
// register file); group g takes rows g, g + 7, ... of each staged 63-row
// tile (cp.async, three stages).  The groups are added pairwise in a fixed
// order, each CTA writes one partial per entry, and a second kernel adds the
// CTAs' partials in CTA order (a wide reduction instead of one finishing
// CTA).
template <int LD>
struct GramLd {
  static constexpr int TS = 3 * LD / 8;
  static constexpr int W = 6 * LD;  // staged row: X R P AX AR AP
  static constexpr int TILES = 72;
  static constexpr int GROUPS = 7;
  static constexpr int THREADS = TILES * GROUPS;  // 504
  static constexpr int TR = 63;                   // rows per stage (9 per group)
  static constexpr int STAGES = 3;
  static constexpr int ENTRIES = TILES * TS * TS;  // partials per CTA
};
template <class XT, int LD>
__host__ __device__ constexpr int gram_ld_stride() {
  return GramLd<LD>::W + static_cast<int>(16 / sizeof(XT));  // padded row, 16-byte multiple
}
template <class XT, int LD>
constexpr size_t gram_ld_smem() {
  using C = GramLd<LD>;
  const size_t stages = static_cast<size_t>(C::STAGES) * C::TR * gram_ld_stride<XT, LD>() * sizeof(XT);
  const size_t red = static_cast<size_t>(C::GROUPS - C::GROUPS / 2) * C::ENTRIES * sizeof(double);
  return stages > red ? stages : red;
}

// upper tile u in [0, 36) of an 8 x 8 tile grid -> (ti, tj), ti <= tj
__device__ __forceinline__ void upper_tile(int u, int& ti, int& tj) {
  ti = 0;
  while (u >= 8 - ti) {
    u -= 8 - ti;
    ++ti;
  }
  tj = ti + u;
}

template <class XT, int LD>
__global__ void __maxnreg__(128)
    k_gram_ld(const XT* __restrict__ X, const XT* __restrict__ R, const XT* __restrict__ P,
              const XT* __restrict__ AX, const XT* __restrict__ AR, const XT* __restrict__ AP, int64_t n,
              double* __restrict__ partial, const int* __restrict__ stop) {
  using C = GramLd<LD>;
  constexpr int TS = C::TS, SW = gram_ld_stride<XT, LD>();
  if (stop != nullptr && *stop != 0) return;
  extern __shared__ __align__(16) unsigned char gram_ld_raw[];
  XT* tile = reinterpret_cast<XT*>(gram_ld_raw);
  double* red = reinterpret_cast<double*>(gram_ld_raw);
  const int tid = threadIdx.x;
  const int g = tid / C::TILES, tau = tid % C::TILES;
  const int h = tau / 36;
  int ti, tj;
  upper_tile(tau % 36, ti, tj);
  const int sb = ti * TS;                  // S columns sb .. sb + TS - 1
  const int tb = h * 3 * LD + tj * TS;     // T = [S AS] columns
  double acc[TS][TS];
#pragma unroll
  for (int p = 0; p < TS; ++p)
#pragma unroll
    for (int q = 0; q < TS; ++q) acc[p][q] = 0.0;
  constexpr int EPC = 16 / sizeof(XT);       // elements per 16-byte chunk
  constexpr int CPB = LD / EPC;              // chunks per (row, block)
  constexpr int NCH = C::TR * 6 * CPB;
  const int64_t ntiles = (n + C::TR - 1) / C::TR;
  auto load_tile = [&](int64_t t, int buf) {
    if (t < ntiles) {
      const int64_t row0 = t * C::TR;
      for (int c = tid; c < NCH; c += C::THREADS) {
        const int b = c / (C::TR * CPB);
        const int rem = c % (C::TR * CPB);
        const int r = rem / CPB, hh = rem % CPB;
        const int64_t row = row0 + r;
        const bool ok = row < n;
        const XT* base = b < 3 ? (b == 0 ? X : (b == 1 ? R : P)) : (b == 3 ? AX : (b == 4 ? AR : AP));
        cp_async16(tile + (static_cast<size_t>(buf) * C::TR + r) * SW + b * LD + hh * EPC,
                   base + (ok ? row : 0) * LD + hh * EPC, ok ? 16 : 0);
      }
    }
    cp_async_commit();  // empty groups keep the group count uniform
  };
  const int64_t step = gridDim.x;
  int64_t t = blockIdx.x;
#pragma unroll
  for (int s0 = 0; s0 < C::STAGES - 1; ++s0) load_tile(t + s0 * step, s0);
  int buf = 0;
  for (; t < ntiles; t += step) {
    load_tile(t + (C::STAGES - 1) * step, (buf + C::STAGES - 1) % C::STAGES);
    cp_async_wait<C::STAGES - 1>();
    __syncthreads();
#pragma unroll 2
    for (int r = g; r < C::TR; r += C::GROUPS) {
      const XT* row = tile + (static_cast<size_t>(buf) * C::TR + r) * SW;
      double s[TS];
#pragma unroll
      for (int p = 0; p < TS; ++p) s[p] = static_cast<double>(row[sb + p]);
#pragma unroll
      for (int q = 0; q < TS; ++q) {
        const double tv = static_cast<double>(row[tb + q]);
#pragma unroll
        for (int p = 0; p < TS; ++p) acc[p][q] = fma(s[p], tv, acc[p][q]);
      }
    }
    __syncthreads();
    buf = (buf + 1) % C::STAGES;
  }
  cp_async_wait<0>();
  __syncthreads();
  // row groups added pairwise: g += g + 4, then g + 2, then g + 1
  const int e0 = tau * TS * TS;
#pragma unroll
  for (int half = 4; half >= 1; half >>= 1) {
    if (g >= half && g < 2 * half) {
#pragma unroll
      for (int p = 0; p < TS; ++p)
#pragma unroll
        for (int q = 0; q < TS; ++q) red[(g - half) * C::ENTRIES + e0 + p * TS + q] = acc[p][q];
    }
    __syncthreads();
    if (g < half && g + half < C::GROUPS) {
#pragma unroll
      for (int p = 0; p < TS; ++p)
#pragma unroll
        for (int q = 0; q < TS; ++q) acc[p][q] += red[g * C::ENTRIES + e0 + p * TS + q];
    }
    __syncthreads();
  }
  if (g == 0) {
    double* dst = partial + static_cast<int64_t>(blockIdx.x) * C::ENTRIES + e0;
#pragma unroll
    for (int p = 0; p < TS; ++p)
#pragma unroll
      for (int q = 0; q < TS; ++q) dst[p * TS + q] = acc[p][q];
  }
}

// Adds the per-CTA partials of k_gram_ld in CTA order and writes both
// (3m) x (3m) matrices.  A CTA takes 32 entries: warp w adds CTAs w, w + 8,
// ..., then the eight warp sums are added in warp order.
template <int LD>
__global__ void __launch_bounds__(256) k_gram_ld_reduce(const double* __restrict__ partial, int nparts, int m,
                                                        int ns_out, double* __restrict__ out,
                                                        const int* __restrict__ stop) {
  using C = GramLd<LD>;
  constexpr int TS = C::TS;
  if (stop != nullptr && *stop != 0) return;
  __shared__ double red[8][32];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int e = blockIdx.x * 32 + lane;
  double s = 0.0;
  if (e < C::ENTRIES)
    for (int c = warp; c < nparts; c += 8) s += partial[static_cast<int64_t>(c) * C::ENTRIES + e];
  red[warp][lane] = s;
  __syncthreads();
  if (warp != 0 || e >= C::ENTRIES) return;
  double v = 0.0;
#pragma unroll
  for (int w = 0; w < 8; ++w) v += red[w][lane];
  const int tau = e / (TS * TS), pq = e % (TS * TS), p = pq / TS, q = pq % TS;
  const int h = tau / 36;
  int ti, tj;
  upper_tile(tau % 36, ti, tj);
  if (ti == tj && p > q) return;  // lower half of a diagonal tile
  const int i = ti * TS + p, j = tj * TS + q;  // entry (i, j) of the 3LD x 3LD product, i <= j
  const int ci = i % LD, cj = j % LD;
  if (ci >= m || cj >= m || i / LD >= ns_out || j / LD >= ns_out) return;
  const int P = ns_out * m;
  const int I = (i / LD) * m + ci, J = (j / LD) * m + cj;
  double* o = out + h * P * P;
  o[I * P + J] = v;
  o[J * P + I] = v;
}

// LOBPCG update with 4-column blocks: four threads per row, thread j produces
// output column j (inputs are read as 4-vectors; the four threads of a row
// share the same sectors).
template <class XT>
__global__ void __launch_bounds__(256) k_lobpcg_update4(LobpcgBlocks<XT> b, const LobpcgCtrl* __restrict__ ctrl,
                                                        int64_t n, int init_mode) {
  __shared__ double sC[3][4][4];
  __shared__ double sLam[4];
  __shared__ int sF[4];
  if (threadIdx.x == 0) {
    sF[0] = ctrl->done;
    sF[1] = ctrl->copy_best;
    sF[2] = ctrl->has_p;
    sF[3] = ctrl->m;
  }
  if (threadIdx.x < 48) {
    const int w = threadIdx.x / 16, r = (threadIdx.x / 4) % 4, c = threadIdx.x % 4;
    const double* src = w == 0 ? ctrl->Cx : (w == 1 ? ctrl->Cr : ctrl->Cp);
    sC[w][r][c] = src[r * MAXM + c];
  }
  if (threadIdx.x < 4) sLam[threadIdx.x] = ctrl->lam[threadIdx.x];
  __syncthreads();
  const int done = sF[0], copy_best = sF[1], use_p = sF[2], m = sF[3];
  if (done && !copy_best) return;
  const int64_t total = n * 4;
  const int64_t stride = static_cast<int64_t>(gridDim.x) * blockDim.x;  // multiple of 32
  // the loop condition uses the warp's base index, so all lanes of a warp run
  // the same trip count and reach the __syncwarp below together
  for (int64_t t = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; (t & ~int64_t(31)) < total;
       t += stride) {
    const bool valid = t < total;  // rows are 4-aligned: a row's lanes agree
    const int64_t i = valid ? (t >> 2) : 0;
    const int j = static_cast<int>(t & 3);
    const int64_t o = i * 4;
    if (valid && copy_best) b.Xbest[o + j] = b.X[o + j];
    if (done) continue;  // uniform
    // lanes past the end compute on row 0 (always readable) and store nothing
    double x[4], ax[4];
#pragma unroll
    for (int c = 0; c < 4; ++c) {
      x[c] = static_cast<double>(b.X[o + c]);
      ax[c] = static_cast<double>(b.AX[o + c]);
    }
    double pn = 0.0, apn = 0.0;
    if (!init_mode) {
#pragma unroll
      for (int c = 0; c < 4; ++c) {
        pn = fma(static_cast<double>(b.R[o + c]), sC[1][c][j], pn);
        apn = fma(static_cast<double>(b.AR[o + c]), sC[1][c][j], apn);
      }
      if (use_p) {
#pragma unroll
        for (int c = 0; c < 4; ++c) {
          pn = fma(static_cast<double>(b.P[o + c]), sC[2][c][j], pn);
          apn = fma(static_cast<double>(b.AP[o + c]), sC[2][c][j], apn);
        }
      }
    }
    double xn = pn, axn = apn;
#pragma unroll
    for (int c = 0; c < 4; ++c) {
      xn = fma(x[c], sC[0][c][j], xn);
      axn = fma(ax[c], sC[0][c][j], axn);
    }
    // every thread of the row has read its inputs before any column is overwritten
    __syncwarp();
    if (!valid) continue;
    const bool active = j < m;
    const XT xs = static_cast<XT>(active ? xn : 0.0);
    const XT axs = static_cast<XT>(active ? axn : 0.0);
    b.X[o + j] = xs;
    b.AX[o + j] = axs;
    b.R[o + j] = static_cast<XT>(active ? static_cast<double>(axs) - sLam[j] * static_cast<double>(xs) : 0.0);
    if (!init_mode) {
      b.P[o + j] = static_cast<XT>(active ? pn : 0.0);
      b.AP[o + j] = static_cast<XT>(active ? apn : 0.0);
    }
  }
}

template <class XT>
__global__ void k_combine(const XT* in0, const XT* in1, const XT* in2, const double* c0, const double* c1,
                          const double* c2, int nin, XT* out, int m_in, int m_out, int cstride, int ld,
                          int64_t n) {
  extern __shared__ double sc_dyn[];
  const int tot = m_in * m_out;
  double* sc[3] = {sc_dyn, sc_dyn + tot, sc_dyn + 2 * tot};
  for (int i = threadIdx.x; i < tot; i += blockDim.x) {
    const int src = (i / m_out) * cstride + i % m_out;
    sc[0][i] = c0[src];
    if (nin > 1) sc[1][i] = c1[src];
    if (nin > 2) sc[2][i] = c2[src];
  }
  __syncthreads();
  const XT* ins[3] = {in0, in1, in2};
  const int64_t stride = static_cast<int64_t>(gridDim.x) * blockDim.x;
  for (int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; i < n; i += stride) {
    for (int j0 = 0; j0 < m_out; j0 += 4) {
      double acc[4] = {0.0, 0.0, 0.0, 0.0};
      for (int b = 0; b < nin; ++b) {
        const XT* row = ins[b] + i * ld;
        for (int c = 0; c < m_in; ++c) {
          const double v = static_cast<double>(row[c]);
#pragma unroll
          for (int t = 0; t < 4; ++t)
            if (j0 + t < m_out) acc[t] = fma(v, sc[b][c * m_out + j0 + t], acc[t]);
        }
      }
#pragma unroll
      for (int t = 0; t < 4; ++t)
        if (j0 + t < m_out) out[i * ld + j0 + t] = static_cast<XT>(acc[t]);
    }
  }
}

// ---------------------------------------------------------------------------
// Column residual norms with deterministic reduction.
template <class XT>
__global__ void k_colnorms(const XT* a, const XT* b, const double* lam, int m, int ld, int64_t n, double* partial,
                           unsigned* counter, double* out) {
  __shared__ double red[8][MAXM];
  __shared__ bool last;
  double acc[MAXM];
  double l[MAXM];
#pragma unroll
  for (int c = 0; c < MAXM; ++c) {
    acc[c] = 0.0;
    l[c] = (b != nullptr && c < m) ? lam[c] : 0.0;
  }
  const int64_t stride = static_cast<int64_t>(gridDim.x) * blockDim.x;
  for (int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; i < n; i += stride) {
#pragma unroll
    for (int c = 0; c < MAXM; ++c) {
      if (c < m) {
        double d = static_cast<double>(a[i * ld + c]);
        if (b != nullptr) d -= l[c] * static_cast<double>(b[i * ld + c]);
        acc[c] = fma(d, d, acc[c]);
      }
    }
  }
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
#pragma unroll
  for (int c = 0; c < MAXM; ++c) {
    const double s = warp_sum(acc[c]);
    if (lane == 0) red[warp][c] = s;
  }
  __syncthreads();
  if (threadIdx.x < m) {
    double s = 0.0;
    for (int w = 0; w < static_cast<int>(blockDim.x >> 5); ++w) s += red[w][threadIdx.x];
    partial[static_cast<int64_t>(threadIdx.x) * gridDim.x + blockIdx.x] = s;
  }
  __threadfence();
  __syncthreads();
  if (threadIdx.x == 0) last = (atomicAdd(counter, 1u) == gridDim.x - 1);
  __syncthreads();
  if (!last) return;
  __threadfence();
  for (int c = warp; c < m; c += blockDim.x >> 5) {
    double s = 0.0;
    for (int b = lane; b < static_cast<int>(gridDim.x); b += 32) s += partial[static_cast<int64_t>(c) * gridDim.x + b];
    s = warp_sum(s);
    if (lane == 0) out[c] = sqrt(s);
  }
  if (threadIdx.x == 0) *counter = 0u;
}

template <class XT>
__global__ void k_fill_normal(XT* x, int64_t n, int m, int ld, uint64_t seed, uint64_t stream) {
  const int64_t total = n * m;
  const int64_t pairs = (total + 1) / 2;
  const int64_t stride = static_cast<int64_t>(gridDim.x) * blockDim.x;
  for (int64_t q = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; q < pairs; q += stride) {
    double z0, z1;
    philox_normal2(seed, stream, static_cast<uint64_t>(q), z0, z1);
    const int64_t e0 = 2 * q, e1 = 2 * q + 1;
    x[(e0 / m) * ld + e0 % m] = static_cast<XT>(z0);
    if (e1 < total) x[(e1 / m) * ld + e1 % m] = static_cast<XT>(z1);
  }
}

__global__ void k_sumsq(const double* v, int64_t n, double* partial, unsigned* counter, double* out) {
  __shared__ double red[32];
  __shared__ bool last;
  double acc = 0.0;
  const int64_t stride = static_cast<int64_t>(gridDim.x) * blockDim.x;
  for (int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; i < n; i += stride)
    acc = fma(v[i], v[i], acc);
  acc = warp_sum(acc);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = acc;
  __syncthreads();
  if (threadIdx.x == 0) {
    double s = 0.0;
    for (int w = 0; w < static_cast<int>(blockDim.x >> 5); ++w) s += red[w];
    partial[blockIdx.x] = s;
  }
  __threadfence();
  __syncthreads();
  if (threadIdx.x == 0) last = (atomicAdd(counter, 1u) == gridDim.x - 1);
  __syncthreads();
  if (!last) return;
  __threadfence();
  if (threadIdx.x < 32) {
    double s = 0.0;
    for (int c = threadIdx.x; c < static_cast<int>(gridDim.x); c += 32) s += partial[c];
    s = warp_sum(s);
    if (threadIdx.x == 0) {
      *out = s;
      *counter = 0u;
    }
  }
}

template <class XT>
__global__ void k_set_col0(XT* x, int ld, int64_t n, const double* v, const double* sumsq) {
  const double s = *sumsq;
  if (!(s > 0.0)) return;
  const double nrm = sqrt(s);
  const int64_t stride = static_cast<int64_t>(gridDim.x) * blockDim.x;
  for (int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; i < n; i += stride)
    x[i * ld] = static_cast<XT>(v[i] / nrm);
}

template <class XT>
__global__ void k_scale_cols(XT* x, int64_t n, int m, int ld, const double* s) {
  const int64_t total = n * m;
  const int64_t stride = static_cast<int64_t>(gridDim.x) * blockDim.x;
  for (int64_t e = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; e < total; e += stride) {
    const int64_t i = e / m;
    const int c = static_cast<int>(e % m);
    x[i * ld + c] = static_cast<XT>(static_cast<double>(x[i * ld + c]) * s[c]);
  }
}

struct ColList {
  int c[SMAX];
  int k;
};

template <class XI, class XO>
__global__ void k_gather_cols(const XI* in, int ld_in, XO* out, int ld_out, int64_t n, ColList cols) {
  const int64_t total = n * cols.k;
  const int64_t stride = static_cast<int64_t>(gridDim.x) * blockDim.x;
  for (int64_t e = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; e < total; e += stride) {
    const int64_t i = e / cols.k;
    const int j = static_cast<int>(e % cols.k);
    out[i * ld_out + j] = static_cast<XO>(in[i * ld_in + cols.c[j]]);
  }
}

// per column: (max |x|, first index) ; deterministic
__global__ void k_argmax_abs(const double* x, int64_t n, int k, int ld, double* pval, long long* pidx,
                             unsigned* counter, double* sign_out) {
  // |x| is ranked by f64::total_cmp, as the crate's reduce does: the bit
  // pattern of |x| (sign bit clear) compared as an integer, so a NaN ranks
  // above +inf.  The partial keys travel through the f64 partial buffer
  // bit for bit.
  __shared__ long long sv[256];
  __shared__ long long si_[256];
  __shared__ bool last;
  for (int c = 0; c < k; ++c) {
    long long best = -1;
    long long bi = -1;
    const int64_t stride = static_cast<int64_t>(gridDim.x) * blockDim.x;
    for (int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; i < n; i += stride) {
      const long long a = __double_as_longlong(x[i * ld + c]) & 0x7fffffffffffffffLL;
      if (a > best) {
        best = a;
        bi = i;
      }
    }
    sv[threadIdx.x] = best;
    si_[threadIdx.x] = bi;
    __syncthreads();
    for (int o = blockDim.x / 2; o > 0; o >>= 1) {
      if (threadIdx.x < o) {
        const long long a2 = sv[threadIdx.x + o];
        const long long i2 = si_[threadIdx.x + o];
        const long long a1 = sv[threadIdx.x];
        const long long i1 = si_[threadIdx.x];
        if (i2 >= 0 && (a2 > a1 || (a2 == a1 && (i1 < 0 || i2 < i1)))) {
          sv[threadIdx.x] = a2;
          si_[threadIdx.x] = i2;
        }
      }
      __syncthreads();
    }
    if (threadIdx.x == 0) {
      pval[static_cast<int64_t>(blockIdx.x) * SMAX + c] = __longlong_as_double(sv[0]);
      pidx[static_cast<int64_t>(blockIdx.x) * SMAX + c] = si_[0];
    }
    __syncthreads();
  }
  __threadfence();
  __syncthreads();
  if (threadIdx.x == 0) last = (atomicAdd(counter, 1u) == gridDim.x - 1);
  __syncthreads();
  if (!last) return;
  __threadfence();
  if (threadIdx.x < k) {
    const int c = threadIdx.x;
    long long best = -1;
    long long bi = -1;
    for (int b = 0; b < static_cast<int>(gridDim.x); ++b) {
      const long long a = __double_as_longlong(pval[static_cast<int64_t>(b) * SMAX + c]);
      const long long i = pidx[static_cast<int64_t>(b) * SMAX + c];
      if (i >= 0 && (a > best || (a == best && (bi < 0 || i < bi)))) {
        best = a;
        bi = i;
      }
    }
    // Rust f64::signum: -1 for negative values and -0.0; NaN (never flipped) for NaN
    const double v = bi >= 0 ? x[bi * ld + c] : 1.0;
    sign_out[c] = (!isnan(v) && signbit(v)) ? -1.0 : 1.0;
  }
  if (threadIdx.x == 0) *counter = 0u;
}

__global__ void k_apply_signs(double* x, int64_t n, int k, int ld, const double* sign) {
  const int64_t total = n * k;
  const int64_t stride = static_cast<int64_t>(gridDim.x) * blockDim.x;
  for (int64_t e = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; e < total; e += stride) {
    const int64_t i = e / k;
    const int c = static_cast<int>(e % k);
    if (sign[c] < 0.0) x[i * ld + c] = -x[i * ld + c];
  }
}

__global__ void k_maxabs(const double* x, int64_t n, int k, int ld, double* partial, unsigned* counter,
                         double* out) {
  __shared__ double red[32];
  __shared__ bool last;
  double m = 0.0;
  const int64_t total = n * k;
  const int64_t stride = static_cast<int64_t>(gridDim.x) * blockDim.x;
  for (int64_t e = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; e < total; e += stride) {
    const double a = fabs(x[(e / k) * ld + e % k]);
    m = a > m ? a : m;  // NaN is ignored like f64::max
  }
  m = warp_max(m);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = m;
  __syncthreads();
  if (threadIdx.x == 0) {
    double s = 0.0;
    for (int w = 0; w < static_cast<int>(blockDim.x >> 5); ++w) s = fmax(s, red[w]);
    partial[blockIdx.x] = s;
  }
  __threadfence();
  __syncthreads();
  if (threadIdx.x == 0) last = (atomicAdd(counter, 1u) == gridDim.x - 1);
  __syncthreads();
  if (!last) return;
  __threadfence();
  if (threadIdx.x < 32) {
    double s = 0.0;
    for (int c = threadIdx.x; c < static_cast<int>(gridDim.x); c += 32) s = fmax(s, partial[c]);
    s = warp_max(s);
    if (threadIdx.x == 0) {
      *out = s;
      *counter = 0u;
    }
  }
}

__global__ void k_scale_noise(const double* x, int64_t n, int k, int ld, double expansion, uint64_t seed,
                              float* out, int add_noise) {
  const int64_t total = n * k;
  const int64_t pairs = (total + 1) / 2;
  const int64_t stride = static_cast<int64_t>(gridDim.x) * blockDim.x;
  for (int64_t q = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; q < pairs; q += stride) {
    double z[2] = {0.0, 0.0};
    if (add_noise) philox_normal2(seed, 0x5ca1eull, static_cast<uint64_t>(q), z[0], z[1]);
#pragma unroll
    for (int t = 0; t < 2; ++t) {
      const int64_t e = 2 * q + t;
      if (e >= total) break;
      const float s = static_cast<float>(x[(e / k) * ld + e % k] * expansion);
      out[e] = add_noise ? __fadd_rn(s, __fmul_rn(static_cast<float>(z[t]), 1.0e-4f)) : s;
    }
  }
}

__global__ void k_copy_strided(const double* in, int ld_in, double* out, int ld_out, int64_t n, int k) {
  const int64_t total = n * k;
  const int64_t stride = static_cast<int64_t>(gridDim.x) * blockDim.x;
  for (int64_t e = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; e < total; e += stride)
    out[(e / k) * ld_out + e % k] = in[(e / k) * ld_in + e % k];
}

// ---------------------------------------------------------------------------
// LOBPCG update (one thread per row):
//   P' = R Cr + P Cp,  AP' = AR Cr + AP Cp,  X' = X Cx + P',  AX' = AX Cx + AP',
//   R' = AX' - X' diag(lam').  init mode: X' = X Cx, AX' = AX Cx, R' as above.
// When the small step flagged the current X as the best iterate, the row of X
// is first copied to Xbest.  Rows are updated in place.
template <class XT, int LD>
__global__ void __launch_bounds__(256) k_lobpcg_update(LobpcgBlocks<XT> b, const LobpcgCtrl* __restrict__ ctrl,
                                                       int64_t n, int init_mode) {
  __shared__ double sCx[MAXM * MAXM], sCr[MAXM * MAXM], sCp[MAXM * MAXM], sLam[MAXM];
  __shared__ int sF[4];
  if (threadIdx.x == 0) {
    sF[0] = ctrl->done;
    sF[1] = ctrl->copy_best;
    sF[2] = ctrl->has_p;
    sF[3] = ctrl->m;
  }
  __syncthreads();
  const int done = sF[0], copy_best = sF[1], use_p = sF[2], m = sF[3];
  if (done && !copy_best) return;
  for (int i = threadIdx.x; i < m * m; i += blockDim.x) {
    const int r = i / m, c = i % m;
    sCx[r * MAXM + c] = ctrl->Cx[r * MAXM + c];
    sCr[r * MAXM + c] = ctrl->Cr[r * MAXM + c];
    sCp[r * MAXM + c] = ctrl->Cp[r * MAXM + c];
  }
  if (threadIdx.x < MAXM) sLam[threadIdx.x] = threadIdx.x < m ? ctrl->lam[threadIdx.x] : 0.0;
  __syncthreads();
  const int64_t stride = static_cast<int64_t>(gridDim.x) * blockDim.x;
  for (int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; i < n; i += stride) {
    const int64_t o = i * LD;
    double x[LD];
#pragma unroll
    for (int c = 0; c < LD; ++c) x[c] = static_cast<double>(b.X[o + c]);
    if (copy_best) {
#pragma unroll
      for (int c = 0; c < LD; ++c) b.Xbest[o + c] = static_cast<XT>(x[c]);
    }
    if (done) continue;
    double ax[LD];
#pragma unroll
    for (int c = 0; c < LD; ++c) ax[c] = static_cast<double>(b.AX[o + c]);
    double xn[LD], axn[LD], pn[LD], apn[LD];
#pragma unroll
    for (int c = 0; c < LD; ++c) {
      xn[c] = 0.0;
      axn[c] = 0.0;
      pn[c] = 0.0;
      apn[c] = 0.0;
    }
    if (!init_mode) {
      double r[LD], ar[LD];
#pragma unroll
      for (int c = 0; c < LD; ++c) {
        r[c] = static_cast<double>(b.R[o + c]);
        ar[c] = static_cast<double>(b.AR[o + c]);
      }
#pragma unroll
      for (int c = 0; c < LD; ++c) {
        if (c < m) {
#pragma unroll
          for (int j = 0; j < LD; ++j) {
            if (j < m) {
              pn[j] = fma(r[c], sCr[c * MAXM + j], pn[j]);
              apn[j] = fma(ar[c], sCr[c * MAXM + j], apn[j]);
            }
          }
        }
      }
      if (use_p) {
        double p[LD], ap[LD];
#pragma unroll
        for (int c = 0; c < LD; ++c) {
          p[c] = static_cast<double>(b.P[o + c]);
          ap[c] = static_cast<double>(b.AP[o + c]);
        }
#pragma unroll
        for (int c = 0; c < LD; ++c) {
          if (c < m) {
#pragma unroll
            for (int j = 0; j < LD; ++j) {
              if (j < m) {
                pn[j] = fma(p[c], sCp[c * MAXM + j], pn[j]);
                apn[j] = fma(ap[c], sCp[c * MAXM + j], apn[j]);
              }
            }
          }
        }
      }
    }
#pragma unroll
    for (int c = 0; c < LD; ++c) {
      if (c < m) {
#pragma unroll
        for (int j = 0; j < LD; ++j) {
          if (j < m) {
            xn[j] = fma(x[c], sCx[c * MAXM + j], xn[j]);
            axn[j] = fma(ax[c], sCx[c * MAXM + j], axn[j]);
          }
        }
      }
    }
#pragma unroll
    for (int j = 0; j < LD; ++j) {
      xn[j] += pn[j];
      axn[j] += apn[j];
      b.X[o + j] = static_cast<XT>(xn[j]);
      b.AX[o + j] = static_cast<XT>(axn[j]);
      // residual from the stored (rounded) values so R matches AX - X lam of the block
      const double xr = static_cast<double>(static_cast<XT>(xn[j]));
      const double axr = static_cast<double>(static_cast<XT>(axn[j]));
      b.R[o + j] = static_cast<XT>(j < m ? axr - sLam[j] * xr : 0.0);
      if (!init_mode) {
        b.P[o + j] = static_cast<XT>(pn[j]);
        b.AP[o + j] = static_cast<XT>(apn[j]);
      }
    }
  }
}

// 16-byte vector of XT
template <class XT>
struct Vec16;
template <>
struct Vec16<double> {
  using type = double2;
};
template <>
struct Vec16<float> {
  using type = float4;
};

// LOBPCG update for 8- and 16-column blocks: LD / 4 threads per row, each
// producing four output columns.  A thread loads only its own four input
// columns of each block (so a warp's loads are contiguous) and takes the
// row's other columns from the row's lanes by warp shuffles; coefficients come
// from shared memory (zero outside the m x m block).  Same formulas as
// k_lobpcg_update.
template <class XT, int LD>
__global__ void __launch_bounds__(256) k_lobpcg_update_q(LobpcgBlocks<XT> b, const LobpcgCtrl* __restrict__ ctrl,
                                                         int64_t n, int init_mode) {
  constexpr int TPR = LD / 4;
  constexpr int EPV = 16 / sizeof(XT);  // elements per 16-byte load
  using V = typename Vec16<XT>::type;
  __shared__ __align__(16) double sC[3][LD][LD];
  __shared__ double sLam[LD];
  const int done = ctrl->done, copy_best = ctrl->copy_best, use_p = ctrl->has_p, m = ctrl->m;
  if (done && !copy_best) return;
  for (int i = threadIdx.x; i < 3 * LD * LD; i += blockDim.x) {
    const int w = i / (LD * LD), r = (i / LD) % LD, c = i % LD;
    const double* src = w == 0 ? ctrl->Cx : (w == 1 ? ctrl->Cr : ctrl->Cp);
    sC[w][r][c] = (r < m && c < m) ? src[r * MAXM + c] : 0.0;
  }
  if (threadIdx.x < LD) sLam[threadIdx.x] = static_cast<int>(threadIdx.x) < m ? ctrl->lam[threadIdx.x] : 0.0;
  __syncthreads();
  const int64_t total = n * TPR;
  const int64_t stride = static_cast<int64_t>(gridDim.x) * blockDim.x;  // multiple of 32
  // the loop condition uses the warp's base index, so all lanes of a warp run
  // the same trip count and reach the __syncwarp below together
  for (int64_t t = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; (t & ~int64_t(31)) < total;
       t += stride) {
    const bool valid = t < total;  // a row's TPR lanes agree
    const int64_t i = valid ? t / TPR : 0;
    const int j0 = static_cast<int>(t % TPR) * 4;
    const int64_t o = i * LD;
    if (valid && copy_best) {
#pragma unroll
      for (int jj = 0; jj < 4; ++jj) b.Xbest[o + j0 + jj] = b.X[o + j0 + jj];
    }
    if (done) continue;  // uniform
    double xn[4] = {0.0, 0.0, 0.0, 0.0}, axn[4] = {0.0, 0.0, 0.0, 0.0};
    double pn[4] = {0.0, 0.0, 0.0, 0.0}, apn[4] = {0.0, 0.0, 0.0, 0.0};
    // out[jj] += sum_c in_a[c] C[c][j0 + jj], out2[jj] += sum_c in_b[c] C[c][j0 + jj];
    // column c of the row is held by lane (first lane of the row) + c / 4
    const int lane = static_cast<int>(threadIdx.x & 31);
    const int row_lane0 = lane & ~(TPR - 1);
    auto accumulate = [&](const XT* ina, const XT* inb, int w, double* outa, double* outb) {
      XT va[4], vb[4];
#pragma unroll
      for (int h = 0; h < 4; h += EPV) {
        *reinterpret_cast<V*>(va + h) = *reinterpret_cast<const V*>(ina + o + j0 + h);
        *reinterpret_cast<V*>(vb + h) = *reinterpret_cast<const V*>(inb + o + j0 + h);
      }
      double da[4], db[4];
#pragma unroll
      for (int h = 0; h < 4; ++h) {
        da[h] = static_cast<double>(va[h]);
        db[h] = static_cast<double>(vb[h]);
      }
#pragma unroll
      for (int c = 0; c < LD; ++c) {
        const double a = __shfl_sync(0xffffffffu, da[c % 4], row_lane0 + c / 4);
        const double bb = __shfl_sync(0xffffffffu, db[c % 4], row_lane0 + c / 4);
#pragma unroll
        for (int jj = 0; jj < 4; ++jj) {
          const double cf = sC[w][c][j0 + jj];
          outa[jj] = fma(a, cf, outa[jj]);
          outb[jj] = fma(bb, cf, outb[jj]);
        }
      }
    };
    if (!init_mode) {
      accumulate(b.R, b.AR, 1, pn, apn);
      if (use_p) accumulate(b.P, b.AP, 2, pn, apn);
    }
    accumulate(b.X, b.AX, 0, xn, axn);
    // every thread of the row has read its inputs before any column is overwritten
    __syncwarp();
    if (!valid) continue;
    XT xs[4], axs[4], rs[4], ps[4], aps[4];
#pragma unroll
    for (int jj = 0; jj < 4; ++jj) {
      const int j = j0 + jj;
      const bool active = j < m;
      xs[jj] = static_cast<XT>(active ? xn[jj] + pn[jj] : 0.0);
      axs[jj] = static_cast<XT>(active ? axn[jj] + apn[jj] : 0.0);
      rs[jj] = static_cast<XT>(active ? static_cast<double>(axs[jj]) - sLam[j] * static_cast<double>(xs[jj]) : 0.0);
      ps[jj] = static_cast<XT>(active ? pn[jj] : 0.0);
      aps[jj] = static_cast<XT>(active ? apn[jj] : 0.0);
    }
#pragma unroll
    for (int jj = 0; jj < 4; ++jj) {
      b.X[o + j0 + jj] = xs[jj];
      b.AX[o + j0 + jj] = axs[jj];
      b.R[o + j0 + jj] = rs[jj];
      if (!init_mode) {
        b.P[o + j0 + jj] = ps[jj];
        b.AP[o + j0 + jj] = aps[jj];
      }
    }
  }
}

// Generic update for any ld (column loop, reads straight from global).
template <class XT>
__global__ void __launch_bounds__(256) k_lobpcg_update_generic(LobpcgBlocks<XT> b, const LobpcgCtrl* __restrict__ ctrl,
                                                               int64_t n, int ld, int init_mode) {
  __shared__ double sCx[MAXM * MAXM], sCr[MAXM * MAXM], sCp[MAXM * MAXM], sLam[MAXM];
  __shared__ int sF[4];
  if (threadIdx.x == 0) {
    sF[0] = ctrl->done;
    sF[1] = ctrl->copy_best;
    sF[2] = ctrl->has_p;
    sF[3] = ctrl->m;
  }
  __syncthreads();
  const int done = sF[0], copy_best = sF[1], use_p = sF[2], m = sF[3];
  if (done && !copy_best) return;
  for (int i = threadIdx.x; i < MAXM * MAXM; i += blockDim.x) {
    sCx[i] = ctrl->Cx[i];
    sCr[i] = ctrl->Cr[i];
    sCp[i] = ctrl->Cp[i];
  }
  if (threadIdx.x < MAXM) sLam[threadIdx.x] = threadIdx.x < m ? ctrl->lam[threadIdx.x] : 0.0;
  __syncthreads();
  const int64_t stride = static_cast<int64_t>(gridDim.x) * blockDim.x;
  for (int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; i < n; i += stride) {
    const int64_t o = i * ld;
    if (copy_best)
      for (int c = 0; c < ld; ++c) b.Xbest[o + c] = b.X[o + c];
    if (done) continue;
    double xn[MAXM], axn[MAXM], pn[MAXM], apn[MAXM];
#pragma unroll
    for (int j = 0; j < MAXM; ++j) {
      xn[j] = 0.0;
      axn[j] = 0.0;
      pn[j] = 0.0;
      apn[j] = 0.0;
    }
    for (int c = 0; c < m; ++c) {
      const double xv = static_cast<double>(b.X[o + c]);
      const double axv = static_cast<double>(b.AX[o + c]);
      double rv = 0.0, arv = 0.0, pv = 0.0, apv = 0.0;
      if (!init_mode) {
        rv = static_cast<double>(b.R[o + c]);
        arv = static_cast<double>(b.AR[o + c]);
        if (use_p) {
          pv = static_cast<double>(b.P[o + c]);
          apv = static_cast<double>(b.AP[o + c]);
        }
      }
#pragma unroll
      for (int j = 0; j < MAXM; ++j) {
        if (j < m) {
          xn[j] = fma(xv, sCx[c * MAXM + j], xn[j]);
          axn[j] = fma(axv, sCx[c * MAXM + j], axn[j]);
          if (!init_mode) {
            pn[j] = fma(rv, sCr[c * MAXM + j], pn[j]);
            apn[j] = fma(arv, sCr[c * MAXM + j], apn[j]);
            if (use_p) {
              pn[j] = fma(pv, sCp[c * MAXM + j], pn[j]);
              apn[j] = fma(apv, sCp[c * MAXM + j], apn[j]);
            }
          }
        }
      }
    }
#pragma unroll
    for (int j = 0; j < MAXM; ++j) {
      if (j < m) {
        xn[j] += pn[j];
        axn[j] += apn[j];
        const XT xs = static_cast<XT>(xn[j]);
        const XT axs = static_cast<XT>(axn[j]);
        b.X[o + j] = xs;
        b.AX[o + j] = axs;
        b.R[o + j] = static_cast<XT>(static_cast<double>(axs) - sLam[j] * static_cast<double>(xs));
        if (!init_mode) {
          b.P[o + j] = static_cast<XT>(pn[j]);
          b.AP[o + j] = static_cast<XT>(apn[j]);
        }
      }
    }
  }
}

int grid_rows(const Exec& ex, int64_t items, int threads = 256, int per_sm = 8) {
  const int64_t need = (items + threads - 1) / threads;
  return static_cast<int>(std::max<int64_t>(1, std::min<int64_t>(need, int64_t(ex.sms) * per_sm)));
}

template <class XT, int LD>
void gram_ld_launch(const Exec& ex, GramWork& w, const XT* const* blk, int m, int ns_out, int64_t n, double* out,
                    const int* stop) {
  using C = GramLd<LD>;
  constexpr size_t smem = gram_ld_smem<XT, LD>();
  // resident CTAs per SM (set once per device)
  static std::atomic<int> resident[64];
  SI_REQUIRE(ex.device >= 0 && ex.device < 64, SI_INVALID_ARGUMENT, "gram: device ordinal");
  if (resident[ex.device] == 0) {
    SI_CUDA(cudaFuncSetAttribute(k_gram_ld<XT, LD>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 static_cast<int>(smem)));
    int r = 0;
    SI_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&r, k_gram_ld<XT, LD>, C::THREADS, smem));
    resident[ex.device] = std::max(1, r);
  }
  const int64_t ntiles = (n + C::TR - 1) / C::TR;
  const int grid = static_cast<int>(
      std::max<int64_t>(1, std::min<int64_t>(ntiles, int64_t(ex.sms) * resident[ex.device].load())));
  w.ensure(static_cast<size_t>(grid) * C::ENTRIES, ex.stream);
  k_gram_ld<XT, LD><<<grid, C::THREADS, smem, ex.stream>>>(blk[0], blk[1], blk[2], blk[3], blk[4], blk[5], n,
                                                           w.partial.get(), stop);
  SI_LAUNCH_CHECK();
  k_gram_ld_reduce<LD><<<(C::ENTRIES + 31) / 32, 256, 0, ex.stream>>>(w.partial.get(), grid, m, ns_out, out, stop);
  SI_LAUNCH_CHECK();
}

}  // namespace

template <class XT>
void gram_dev(const Exec& ex, GramWork& w, GramMode mode, const XT* const* blk, int ns, int nblk, int m, int ld,
              int64_t n, double* out, const int* stop) {
  SI_REQUIRE(nblk >= 1 && nblk <= 8 && m >= 1 && nblk * m <= GMAXW, SI_INVALID_ARGUMENT, "gram: too many columns");
  // The per-iteration LOBPCG Gram ([X R P], [AX AR AP]) and the Gram of X and
  // AX alone (start and final Rayleigh-Ritz) run on the register-tiled
  // kernels; the latter passes X and AX three times and keeps the first block.
  const bool iter = mode == GRAM_SYM2 && ns == 3 && nblk == 6;
  const bool xonly = mode == GRAM_SYM2 && ns == 1 && nblk == 2;
  const XT* const six[6] = {blk[0], xonly ? blk[0] : blk[1], xonly ? blk[0] : blk[2],
                            xonly ? blk[1] : blk[3], xonly ? blk[1] : blk[4], xonly ? blk[1] : blk[5]};
  const int ns_out = xonly ? 1 : 3;
  if ((iter || xonly) && m <= ld && (ld == 8 || ld == 16)) {
    if (ld == 8)
      gram_ld_launch<XT, 8>(ex, w, six, m, ns_out, n, out, stop);
    else
      gram_ld_launch<XT, 16>(ex, w, six, m, ns_out, n, out, stop);
    return;
  }
  if ((iter || xonly) && m == 4 && ld == 4 && !gram4_old_forced()) {
    // 4-column blocks: the task-split kernel
    static std::atomic<int> resident_t[2][64];
    const int ti = sizeof(XT) == 8 ? 1 : 0;
    SI_REQUIRE(ex.device >= 0 && ex.device < 64, SI_INVALID_ARGUMENT, "gram: device ordinal");
    if (resident_t[ti][ex.device] == 0) {
      int r = 0;
      SI_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&r, k_gram4t<XT>, GT_THREADS, 0));
      resident_t[ti][ex.device] = std::max(1, r);
    }
    const int64_t ntiles = (n + GT_TR - 1) / GT_TR;
    const int grid = static_cast<int>(
        std::max<int64_t>(1, std::min<int64_t>(ntiles, int64_t(ex.sms) * resident_t[ti][ex.device].load())));
    w.ensure(static_cast<size_t>(grid) * 288, ex.stream);
    k_gram4t<XT><<<grid, GT_THREADS, 0, ex.stream>>>(six[0], six[1], six[2], six[3], six[4], six[5], n,
                                                     w.partial.get(), stop);
    SI_LAUNCH_CHECK();
    k_gram4_reduce<<<9, 256, 0, ex.stream>>>(w.partial.get(), grid, ns_out, out, stop);
    SI_LAUNCH_CHECK();
    return;
  }
  if ((iter || xonly) && m == 4 && ld == 4) {
    // 4-column blocks (SPECTRAL_INIT_GRAM=tile: the register-tiled kernel)
    // resident CTAs per SM from the stage memory (set once per device)
    static std::atomic<int> resident[2][64];
    const int ti = sizeof(XT) == 8 ? 1 : 0;
    SI_REQUIRE(ex.device >= 0 && ex.device < 64, SI_INVALID_ARGUMENT, "gram: device ordinal");
    if (resident[ti][ex.device] == 0) {
      SI_CUDA(cudaFuncSetAttribute(k_gram4<XT>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                   static_cast<int>(gram4_smem_bytes<XT>())));
      int r = 0;
      SI_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&r, k_gram4<XT>, G4_THREADS, gram4_smem_bytes<XT>()));
      resident[ti][ex.device] = std::max(1, r);
    }
    const int64_t ntiles = (n + G4_TR - 1) / G4_TR;
    const int grid = static_cast<int>(
        std::max<int64_t>(1, std::min<int64_t>(ntiles, int64_t(ex.sms) * resident[ti][ex.device].load())));
    w.ensure(static_cast<size_t>(grid) * 288, ex.stream);
    k_gram4<XT><<<grid, G4_THREADS, gram4_smem_bytes<XT>(), ex.stream>>>(six[0], six[1], six[2], six[3], six[4],
                                                                        six[5], n, w.partial.get(), stop);
    SI_LAUNCH_CHECK();
    k_gram4_reduce<<<9, 256, 0, ex.stream>>>(w.partial.get(), grid, ns_out, out, stop);
    SI_LAUNCH_CHECK();
    return;
  }
  GramParams<XT> p{};
  for (int b = 0; b < nblk; ++b) p.blk[b] = blk[b];
  p.nblk = nblk;
  p.ns = ns;
  p.m = m;
  p.ld = ld;
  p.n = n;
  p.mode = mode;
  p.P = ns * m;
  if (mode == GRAM_SYM2) {
    SI_REQUIRE(nblk == 2 * ns, SI_INVALID_ARGUMENT, "gram SYM2 needs 2*ns blocks");
    p.Q = p.P;
    p.ne = p.P * (p.P + 1);
  } else {
    p.Q = (nblk - ns) * m;
    p.ne = p.P * p.Q;
  }
  SI_REQUIRE(p.ne <= GMAXE, SI_INVALID_ARGUMENT, "gram: too many entries");
  const int64_t ntiles = (n + GTR - 1) / GTR;
  const int grid = static_cast<int>(std::max<int64_t>(1, std::min<int64_t>(ntiles, int64_t(ex.sms) * 2)));
  w.ensure(static_cast<size_t>(grid) * GMAXE, ex.stream);
  p.partial = w.partial.get();
  p.counter = w.counter.get();
  p.out = out;
  p.stop = stop;
  k_gram<XT><<<grid, GT, 0, ex.stream>>>(p);
  SI_LAUNCH_CHECK();
}

template <class XT>
void combine_dev(const Exec& ex, const XT* const* in, const double* const* coef, int nin, XT* out, int m_in,
                 int m_out, int cstride, int ld, int64_t n) {
  SI_REQUIRE(nin >= 1 && nin <= 3 && m_in <= SMAX && m_out <= SMAX, SI_INVALID_ARGUMENT, "combine: bad sizes");
  if (n == 0) return;
  const size_t smem = sizeof(double) * nin * m_in * m_out;
  SI_REQUIRE(smem <= 160 * 1024, SI_INVALID_ARGUMENT, "combine: coefficients too large");
  if (smem > 48 * 1024)
    SI_CUDA(cudaFuncSetAttribute(k_combine<XT>, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem)));
  k_combine<XT><<<grid_rows(ex, n), 256, smem, ex.stream>>>(in[0], nin > 1 ? in[1] : nullptr,
                                                          nin > 2 ? in[2] : nullptr, coef[0],
                                                          nin > 1 ? coef[1] : nullptr, nin > 2 ? coef[2] : nullptr,
                                                          nin, out, m_in, m_out, cstride, ld, n);
  SI_LAUNCH_CHECK();
}

template <class XT>
void column_residual_norms_dev(const Exec& ex, GramWork& w, const XT* a, const XT* b, const double* lam_dev, int m,
                               int ld, int64_t n, double* out_dev) {
  SI_REQUIRE(m <= MAXM, SI_INVALID_ARGUMENT, "colnorms: m too large");
  const int grid = grid_rows(ex, std::max<int64_t>(n, 1), 256, 2);
  w.ensure(static_cast<size_t>(grid) * MAXM, ex.stream);
  k_colnorms<XT><<<grid, 256, 0, ex.stream>>>(a, b, lam_dev, m, ld, n, w.partial.get(), w.counter.get(), out_dev);
  SI_LAUNCH_CHECK();
}

template <class XT>
void fill_normal_dev(const Exec& ex, XT* x, int64_t n, int m, int ld, uint64_t seed, uint64_t stream) {
  SI_CUDA(cudaMemsetAsync(x, 0, sizeof(XT) * n * ld, ex.stream));
  if (n * m == 0) return;
  k_fill_normal<XT><<<grid_rows(ex, (n * m + 1) / 2), 256, 0, ex.stream>>>(x, n, m, ld, seed, stream);
  SI_LAUNCH_CHECK();
}

template <class XT>
void set_column_normalized_dev(const Exec& ex, GramWork& w, XT* x, int ld, int64_t n, const double* v) {
  if (n == 0) return;
  const int grid = grid_rows(ex, n, 256, 2);
  w.ensure(static_cast<size_t>(grid) + 1, ex.stream);
  DevBuf<double> s(1, ex.stream);
  k_sumsq<<<grid, 256, 0, ex.stream>>>(v, n, w.partial.get(), w.counter.get(), s.get());
  SI_LAUNCH_CHECK();
  k_set_col0<XT><<<grid_rows(ex, n), 256, 0, ex.stream>>>(x, ld, n, v, s.get());
  SI_LAUNCH_CHECK();
}

template <class XT>
void scale_columns_dev(const Exec& ex, XT* x, int64_t n, int m, int ld, const double* s) {
  if (n * m == 0) return;
  k_scale_cols<XT><<<grid_rows(ex, n * m), 256, 0, ex.stream>>>(x, n, m, ld, s);
  SI_LAUNCH_CHECK();
}

template <class XI, class XO>
void gather_columns_dev(const Exec& ex, const XI* in, int ld_in, XO* out, int ld_out, int64_t n,
                        const std::vector<int>& cols) {
  SI_REQUIRE(cols.size() <= static_cast<size_t>(SMAX), SI_INVALID_ARGUMENT, "gather: too many columns");
  ColList cl{};
  cl.k = static_cast<int>(cols.size());
  for (size_t j = 0; j < cols.size(); ++j) cl.c[j] = cols[j];
  if (n * cl.k == 0) return;
  k_gather_cols<XI, XO><<<grid_rows(ex, n * cl.k), 256, 0, ex.stream>>>(in, ld_in, out, ld_out, n, cl);
  SI_LAUNCH_CHECK();
}

void normalize_signs_dev(const Exec& ex, GramWork& w, double* x, int64_t n, int k, int ld) {
  SI_REQUIRE(k <= SMAX, SI_INVALID_ARGUMENT, "normalize_signs: too many columns");
  if (n == 0 || k == 0) return;
  const int grid = grid_rows(ex, n, 256, 2);
  DevBuf<double> pval(static_cast<size_t>(grid) * SMAX, ex.stream), sign(SMAX, ex.stream);
  DevBuf<long long> pidx(static_cast<size_t>(grid) * SMAX, ex.stream);
  w.ensure(1, ex.stream);
  k_argmax_abs<<<grid, 256, 0, ex.stream>>>(x, n, k, ld, pval.get(), pidx.get(), w.counter.get(), sign.get());
  SI_LAUNCH_CHECK();
  k_apply_signs<<<grid_rows(ex, n * k), 256, 0, ex.stream>>>(x, n, k, ld, sign.get());
  SI_LAUNCH_CHECK();
}

double max_abs_dev(const Exec& ex, GramWork& w, const double* x, int64_t n, int k, int ld) {
  if (n * k == 0) return 0.0;
  const int grid = grid_rows(ex, n * k, 256, 2);
  w.ensure(static_cast<size_t>(grid), ex.stream);
  DevBuf<double> out(1, ex.stream);
  k_maxabs<<<grid, 256, 0, ex.stream>>>(x, n, k, ld, w.partial.get(), w.counter.get(), out.get());
  SI_LAUNCH_CHECK();
  double h = 0.0;
  SI_CUDA(cudaMemcpyAsync(&h, out.get(), sizeof(double), cudaMemcpyDeviceToHost, ex.stream));
  SI_CUDA(cudaStreamSynchronize(ex.stream));
  return h;
}

void scale_noise_dev(const Exec& ex, const double* x, int64_t n, int k, int ld, double expansion, uint64_t seed,
                     float* out, bool add_noise) {
  if (n * k == 0) return;
  k_scale_noise<<<grid_rows(ex, (n * k + 1) / 2), 256, 0, ex.stream>>>(x, n, k, ld, expansion, seed, out,
                                                                        add_noise ? 1 : 0);
  SI_LAUNCH_CHECK();
}

void copy_strided_dev(const Exec& ex, const double* in, int ld_in, double* out, int ld_out, int64_t n, int k) {
  if (n * k == 0) return;
  k_copy_strided<<<grid_rows(ex, n * k), 256, 0, ex.stream>>>(in, ld_in, out, ld_out, n, k);
  SI_LAUNCH_CHECK();
}

template <class XT>
void lobpcg_update_dev(const Exec& ex, const LobpcgBlocks<XT>& b, const LobpcgCtrl* ctrl, int ld, int64_t n,
                       int init_mode) {
  if (n == 0) return;
  const int grid = grid_rows(ex, n);
  if (ld == 4)
    k_lobpcg_update4<XT><<<grid_rows(ex, n * 4), 256, 0, ex.stream>>>(b, ctrl, n, init_mode);
  else if (ld == 8)
    k_lobpcg_update_q<XT, 8><<<grid_rows(ex, n * 2), 256, 0, ex.stream>>>(b, ctrl, n, init_mode);
  else if (ld == 16)
    k_lobpcg_update_q<XT, 16><<<grid_rows(ex, n * 4), 256, 0, ex.stream>>>(b, ctrl, n, init_mode);
  else
    k_lobpcg_update_generic<XT><<<grid, 256, 0, ex.stream>>>(b, ctrl, n, ld, init_mode);
  SI_LAUNCH_CHECK();
}

// explicit instantiations
template void gram_dev<double>(const Exec&, GramWork&, GramMode, const double* const*, int, int, int, int, int64_t,
                               double*, const int*);
template void gram_dev<float>(const Exec&, GramWork&, GramMode, const float* const*, int, int, int, int, int64_t,
                              double*, const int*);
template void combine_dev<double>(const Exec&, const double* const*, const double* const*, int, double*, int, int,
                                  int, int, int64_t);
template void combine_dev<float>(const Exec&, const float* const*, const double* const*, int, float*, int, int,
                                 int, int, int64_t);
template void column_residual_norms_dev<double>(const Exec&, GramWork&, const double*, const double*,
                                                const double*, int, int, int64_t, double*);
template void column_residual_norms_dev<float>(const Exec&, GramWork&, const float*, const float*, const double*,
                                               int, int, int64_t, double*);
template void fill_normal_dev<double>(const Exec&, double*, int64_t, int, int, uint64_t, uint64_t);
template void fill_normal_dev<float>(const Exec&, float*, int64_t, int, int, uint64_t, uint64_t);
template void set_column_normalized_dev<double>(const Exec&, GramWork&, double*, int, int64_t, const double*);
template void set_column_normalized_dev<float>(const Exec&, GramWork&, float*, int, int64_t, const double*);
template void scale_columns_dev<double>(const Exec&, double*, int64_t, int, int, const double*);
template void scale_columns_dev<float>(const Exec&, float*, int64_t, int, int, const double*);
template void gather_columns_dev<double, double>(const Exec&, const double*, int, double*, int, int64_t,
                                                 const std::vector<int>&);
template void gather_columns_dev<float, double>(const Exec&, const float*, int, double*, int, int64_t,
                                                const std::vector<int>&);
template void gather_columns_dev<double, float>(const Exec&, const double*, int, float*, int, int64_t,
                                                const std::vector<int>&);
template void lobpcg_update_dev<double>(const Exec&, const LobpcgBlocks<double>&, const LobpcgCtrl*, int, int64_t,
                                        int);
template void lobpcg_update_dev<float>(const Exec&, const LobpcgBlocks<float>&, const LobpcgCtrl*, int, int64_t,
                                       int);

}  // namespace si
