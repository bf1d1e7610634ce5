// Allocation-free variant of the f64 diagnostics reduction.
//
// Some callers cannot allocate device memory while they run: a host
// application that owns every device byte through its own arena, a process
// under a hard device-memory quota, or a time-stepping loop that must not
// call cudaMalloc/cudaFree (those calls can synchronize the device and stall
// the loop). lbmb_reduce_populations_noalloc serves them: it reduces
// populations the caller already holds in device memory and keeps its block
// partials in a fixed file-scope device array instead of allocating.
//
// The array holds NOALLOC_MAX_BLOCKS x 5 partial sums plus the final sums
// (about 640 KiB) on every device that loads this library, until the
// process exits. It is shared by every call: each call overwrites exactly
// the partials it later reads, so nothing must be cleared between calls,
// but calls whose kernels overlap on the GPU (different streams, or
// different host threads on the same device) race on it and must be
// serialized by the caller.
#include <cstdint>
#include <string>

#include "../../include/lbmb.h"
#include "common.cuh"
#include "lattice.cuh"

namespace lbmb {
extern thread_local std::string g_last_error;
}

namespace {

constexpr int NOALLOC_THREADS = 256;
constexpr int NOALLOC_CELLS_PER_THREAD = 8;
constexpr int64_t NOALLOC_CELLS_PER_BLOCK = int64_t(NOALLOC_THREADS) * NOALLOC_CELLS_PER_THREAD;
constexpr int64_t NOALLOC_MAX_BLOCKS = 16384;
constexpr int64_t NOALLOC_MAX_CELLS = NOALLOC_MAX_BLOCKS * NOALLOC_CELLS_PER_BLOCK;  // 2^25
constexpr int64_t NOALLOC_RESULT = NOALLOC_MAX_BLOCKS * 5;                       // result offset
constexpr int64_t NOALLOC_DOUBLES = NOALLOC_RESULT + 8;
constexpr int NOALLOC_FINISH_THREADS = 256;

__device__ __align__(256) double g_noalloc_scratch[NOALLOC_DOUBLES];

struct NoAllocError {
  int code;
  std::string msg;
};

// Device address of the scratch array in the current device's context. In
// host code g_noalloc_scratch only names a host-side shadow, so the address
// is looked up with the device current. The lookup runs on every call (it
// allocates nothing): a cached address would go stale when the context is
// torn down and rebuilt (cudaDeviceReset) and the module loaded again.
double* scratch_on_current_device() {
  void* p = nullptr;
  const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
  if (e != cudaSuccess || !p)
    throw NoAllocError{LBMB_ERR_CUDA, std::string("cudaGetSymbolAddress: ") + cudaGetErrorString(e)};
  return static_cast<double*>(p);
}

// Block b reduces cells [b * 2048, (b + 1) * 2048) in a fixed order and
// writes {fluid cells, sum f, momentum x, y, z (+ F/2)} to part[5 b ...].
template <int Q, class S>
__global__ void __launch_bounds__(NOALLOC_THREADS)
    reduce_linear_kernel(const S* f, int64_t plane, const uint8_t* solid, int64_t n, double gx, double gy,
                         double gz, double* part) {
  using L = lbmb::Lat<Q>;
  __shared__ double sh[5][NOALLOC_THREADS / 32];
  double v[5] = {0.0, 0.0, 0.0, 0.0, 0.0};
  const int64_t base = int64_t(blockIdx.x) * NOALLOC_CELLS_PER_BLOCK;
#pragma unroll 1
  for (int k = 0; k < NOALLOC_CELLS_PER_THREAD; ++k) {
    const int64_t cell = base + int64_t(k) * NOALLOC_THREADS + threadIdx.x;
    if (cell >= n) break;
    if (solid && solid[cell]) continue;
    double s = 0.0, m0 = 0.0, m1 = 0.0, m2 = 0.0;
#pragma unroll
    for (int q = 0; q < Q; ++q) {
      const double fq = double(lbmb::Codec<S>::ld(f + q * plane + cell));
      s += fq;
      m0 += double(L::cx(q)) * fq;
      m1 += double(L::cy(q)) * fq;
      m2 += double(L::cz(q)) * fq;
    }
    v[0] += 1.0;
    v[1] += s;
    v[2] += m0 + 0.5 * gx;
    v[3] += m1 + 0.5 * gy;
    v[4] += m2 + 0.5 * gz;
  }
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
#pragma unroll
  for (int k = 0; k < 5; ++k)
    for (int o = 16; o > 0; o >>= 1) v[k] += __shfl_down_sync(0xffffffffu, v[k], o);
  if (lane == 0)
    for (int k = 0; k < 5; ++k) sh[k][wid] = v[k];
  __syncthreads();
  if (threadIdx.x == 0)
    for (int k = 0; k < 5; ++k) {
      double t = 0.0;
      for (int w = 0; w < NOALLOC_THREADS / 32; ++w) t += sh[k][w];
      part[5 * blockIdx.x + k] = t;
    }
}

// One block: thread t sums the partials of blocks t, t + 256, t + 512, ...
// in that order, then a fixed shared-memory tree folds the 256 sums; the
// result does not depend on timing.
__global__ void __launch_bounds__(NOALLOC_FINISH_THREADS)
    reduce_linear_finish_kernel(const double* part, int64_t nblk, double* out) {
  __shared__ double sh[5][NOALLOC_FINISH_THREADS];
  const int t = threadIdx.x;
  double v[5] = {0.0, 0.0, 0.0, 0.0, 0.0};
  for (int64_t b = t; b < nblk; b += NOALLOC_FINISH_THREADS)
#pragma unroll
    for (int k = 0; k < 5; ++k) v[k] += part[5 * b + k];
#pragma unroll
  for (int k = 0; k < 5; ++k) sh[k][t] = v[k];
  __syncthreads();
  for (int w = NOALLOC_FINISH_THREADS / 2; w > 0; w >>= 1) {
    if (t < w)
#pragma unroll
      for (int k = 0; k < 5; ++k) sh[k][t] += sh[k][t + w];
    __syncthreads();
  }
  if (t < 5) out[t] = sh[t][0];
}

template <int Q, class S>
void launch(const void* f, int64_t plane, const uint8_t* solid, int64_t n, const double* g, double* scratch,
            int64_t nblk, cudaStream_t st) {
  reduce_linear_kernel<Q, S><<<unsigned(nblk), NOALLOC_THREADS, 0, st>>>(static_cast<const S*>(f), plane, solid, n,
                                                                          g[0], g[1], g[2], scratch);
}

}  // namespace

extern "C" int lbmb_reduce_populations_noalloc(const void* f, int32_t storage, int32_t q, int64_t ncells,
                                               int64_t plane, const uint8_t* solid, const double force[3],
                                               double out[5], void* stream) {
  try {
    if (!f || !out) throw NoAllocError{LBMB_ERR_INVALID, "null populations or output"};
    if (q != 19 && q != 27) throw NoAllocError{LBMB_ERR_INVALID, "lattice must be 19 or 27"};
    if (ncells <= 0) throw NoAllocError{LBMB_ERR_INVALID, "ncells must be positive"};
    if (ncells > NOALLOC_MAX_CELLS)
      throw NoAllocError{LBMB_ERR_INVALID, "ncells " + std::to_string(ncells) + " exceeds the no-alloc maximum of " +
                                               std::to_string(NOALLOC_MAX_CELLS) + " cells"};
    if (plane < ncells) throw NoAllocError{LBMB_ERR_INVALID, "plane stride must be >= ncells"};
    const double zero[3] = {0.0, 0.0, 0.0};
    const double* g = force ? force : zero;
    double* scratch = scratch_on_current_device();
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    const int64_t nblk = (ncells + NOALLOC_CELLS_PER_BLOCK - 1) / NOALLOC_CELLS_PER_BLOCK;
    switch (storage) {
      case LBMB_STORE_F32:
        q == 19 ? launch<19, float>(f, plane, solid, ncells, g, scratch, nblk, st)
                : launch<27, float>(f, plane, solid, ncells, g, scratch, nblk, st);
        break;
      case LBMB_STORE_F64:
        q == 19 ? launch<19, double>(f, plane, solid, ncells, g, scratch, nblk, st)
                : launch<27, double>(f, plane, solid, ncells, g, scratch, nblk, st);
        break;
      case LBMB_STORE_F16:
        q == 19 ? launch<19, __half>(f, plane, solid, ncells, g, scratch, nblk, st)
                : launch<27, __half>(f, plane, solid, ncells, g, scratch, nblk, st);
        break;
      case LBMB_STORE_BF16:
        q == 19 ? launch<19, __nv_bfloat16>(f, plane, solid, ncells, g, scratch, nblk, st)
                : launch<27, __nv_bfloat16>(f, plane, solid, ncells, g, scratch, nblk, st);
        break;
      default:
        throw NoAllocError{LBMB_ERR_INVALID, "unknown storage precision"};
    }
    reduce_linear_finish_kernel<<<1, NOALLOC_FINISH_THREADS, 0, st>>>(scratch, nblk, scratch + NOALLOC_RESULT);
    cudaError_t e = cudaGetLastError();
    if (e == cudaSuccess)
      e = cudaMemcpyAsync(out, scratch + NOALLOC_RESULT, 5 * sizeof(double), cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) throw NoAllocError{LBMB_ERR_CUDA, std::string("no-alloc reduction: ") + cudaGetErrorString(e)};
    lbmb::g_last_error.clear();
    return LBMB_OK;
  } catch (const NoAllocError& e) {
    lbmb::g_last_error = e.msg;
    return e.code;
  }
}
