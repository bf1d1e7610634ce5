// TMA-staged AA collide-stream: persistent blocks stream 128-cell tiles of
// all Q population planes into shared memory with bulk asynchronous copies
// (cp.async.bulk + mbarrier, two stages), so the next tile is in flight
// while the current one is collided. Memory latency is then hidden by the
// copy engine instead of by per-thread registers, which the central-moment
// collision needs for itself.
//
// Even step: window q = plane q, cells [c0, c0 + 128) (16-byte aligned).
// Odd step:  window q = plane opp(q), cells [c0 - d_q, c0 - d_q + 128) with
//            d_q = cx + cy nx + cz nx ny; the start is rounded down to a
//            128-byte line and the window is widened by one line (PAD
//            elements); thread j reads element j + r_q (r_q = (-d_q) mod PAD,
//            the same for every tile).
// Windows never leave the allocation: the population buffer carries a guard
// margin on both sides. Only the elements of the tile's own cells are used,
// and by the AA ownership rule (each location is read and written by one
// cell's thread per step) a prefetched window is never stale.
//
// Cells with a solid neighbour read the directions coming off a wall from
// their own slot (global load) and everything else from shared memory;
// cells on a periodic face take the generic direct-load path. Every wait on
// an mbarrier is bounded (about a second); a timeout sets a device error
// flag, waits (bounded) for the copies still in flight and leaves.
#pragma once
#include "hydro.cuh"

namespace lbmb {

constexpr int TMA_TILE = 128;

// Odd-step windows start on a 128-byte line (PAD elements of slack) so the
// bulk copies move whole cache lines; even-step windows are the tile itself.
template <class S>
struct TmaWin {
  static constexpr int PAD = 128 / int(sizeof(S));
  static constexpr int WIN = TMA_TILE + PAD;
  static constexpr int BYTES = WIN * int(sizeof(S));
  static constexpr int EVEN_BYTES = TMA_TILE * int(sizeof(S));
};

template <int Q, class S>
constexpr size_t tma_smem_bytes() {
  return size_t(2) * Q * TmaWin<S>::BYTES + 3 * sizeof(uint64_t);
}

// Default bound on one mbarrier wait of the bulk-copy sweeps, in SM clock
// cycles (about a second at 1.9 GHz).
constexpr long long WAIT_LIMIT_DEFAULT = 1LL << 31;

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}

__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
               : "memory");
}

__device__ __forceinline__ void bulk_g2s(void* dst, const void* src, uint32_t bytes, uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
          smem_u32(dst)),
      "l"(src), "r"(bytes), "r"(smem_u32(bar))
      : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
      : "=r"(ok)
      : "r"(smem_u32(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}

// Wait for phase `parity` of an mbarrier for at most `limit` clock cycles.
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t* bar, uint32_t parity,
                                                  long long limit = WAIT_LIMIT_DEFAULT) {
  if (mbar_try_wait(bar, parity)) return true;
  const long long t0 = clock64();
  while (!mbar_try_wait(bar, parity))
    if (clock64() - t0 > limit) return false;
  return true;
}

// Self-test of the timeout path (wait_limit < 0): thread 0 waits up to
// -wait_limit cycles on an mbarrier that nothing arrives at, then reports
// the timeout through the device error flag. Nothing is copied or written.
__device__ __forceinline__ void wait_selftest(uint64_t* bar, long long wait_limit, int* err) {
  if (!mbar_wait_bounded(bar, 0u, -wait_limit)) atomicOr(err, 1);
}

template <int Q, class S, int COLL, bool ODD, bool ROWS_ALIGNED>
__global__ void __launch_bounds__(TMA_TILE, HydroOccupancy<typename Codec<S>::A>::MIN_BLOCKS)
    hydro_tma_kernel(HydroParams<typename Codec<S>::A> p, int64_t ncells, int ntiles, int* err,
                     const typename Codec<S>::A* omega, long long wait_limit) {
  using A = typename Codec<S>::A;
  using L = Lat<Q>;
  using CD = Codec<S>;
  using W = TmaWin<S>;
  extern __shared__ __align__(128) unsigned char smem_raw[];
  S* sm = reinterpret_cast<S*>(smem_raw);
  uint64_t* bar = reinterpret_cast<uint64_t*>(smem_raw + size_t(2) * Q * W::BYTES);
  __shared__ int timed_out;
  const int j = threadIdx.x;
  S* fb = static_cast<S*>(p.f);
  const int64_t pl = p.plane;
  const int nx = p.nx, nxy = p.nxy;
  auto dq = [&](int q) -> int64_t {
    return int64_t(L::cx(q)) + int64_t(L::cy(q)) * nx + int64_t(L::cz(q)) * nxy;
  };
  auto rq = [&](int q) -> int {
    if (!ODD) return 0;
    if (ROWS_ALIGNED) return (-L::cx(q)) & (W::PAD - 1);
    return int(((-dq(q)) % W::PAD + W::PAD) % W::PAD);
  };
  if (j == 0) {
    timed_out = 0;
    mbar_init(&bar[0], 1);
    mbar_init(&bar[1], 1);
    mbar_init(&bar[2], 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  __syncthreads();
  if (wait_limit < 0) {
    if (j == 0) wait_selftest(&bar[2], wait_limit, err);
    return;
  }
  auto issue = [&](int t, int s) {
    const int64_t c0 = int64_t(t) * TMA_TILE;
    const uint32_t bytes = ODD ? uint32_t(W::BYTES) : uint32_t(W::EVEN_BYTES);
    mbar_expect_tx(&bar[s], uint32_t(Q) * bytes);
#pragma unroll 1
    for (int q = 0; q < Q; ++q) {
      const int64_t e = ODD ? (int64_t(opp(q)) * pl + c0 - dq(q) - rq(q)) : (int64_t(q) * pl + c0);
      bulk_g2s(sm + (s * Q + q) * W::WIN, fb + e, bytes, &bar[s]);
    }
  };
  int it = 0;
  int t = blockIdx.x;
  if (j == 0 && t < ntiles) issue(t, 0);
  for (; t < ntiles; t += gridDim.x, ++it) {
    const int s = it & 1;
    const int tn = t + int(gridDim.x);
    if (j == 0 && tn < ntiles) {
      asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
      issue(tn, s ^ 1);
    }
    if (!mbar_wait_bounded(&bar[s], uint32_t((it >> 1) & 1), wait_limit)) atomicOr(&timed_out, 1);
    __syncthreads();
    if (timed_out) {
      if (j == 0) {
        atomicOr(err, 1);
        if (tn < ntiles) mbar_wait_bounded(&bar[s ^ 1], uint32_t(((it + 1) >> 1) & 1), wait_limit);
      }
      return;
    }
    const int64_t cell = int64_t(t) * TMA_TILE + j;
    if (cell < ncells) {
      const uint8_t fl = p.flags[cell];
      if (!(fl & (F_SOLID | F_FORCED))) {
        if (fl & (F_WRAP | F_SLIP)) {
          const int z = int(cell / nxy);
          const int64_t r = cell - int64_t(z) * nxy;
          const int y = int(r / nx);
          const int x = int(r - int64_t(y) * nx);
          hydro_cell_generic_field<Q, S, COLL, ODD, false>(p, x, y, z, uint32_t(cell), fl, omega);
        } else {
          const S* w = sm + s * Q * W::WIN;
          const uint32_t mask = (fl & F_BOUNDARY) ? p.nbr[cell] : 0u;
          A f[Q];
#pragma unroll
          for (int q = 0; q < Q; ++q) {
            // generic-pointer select: own slot in global memory for a
            // direction coming off a wall, the staged window otherwise
            const S* src = (ODD && ((mask >> opp(q)) & 1u)) ? (fb + int64_t(q) * pl + cell)
                                                           : (w + q * W::WIN + j + rq(q));
            f[q] = CD::ld(src);
          }
          A dr = A(0), m0 = A(0), m1 = A(0), m2 = A(0);
#pragma unroll
          for (int q = 0; q < Q; ++q) {
            dr = dr + f[q];
            if (L::cx(q) == 1) m0 = m0 + f[q];
            if (L::cx(q) == -1) m0 = m0 - f[q];
            if (L::cy(q) == 1) m1 = m1 + f[q];
            if (L::cy(q) == -1) m1 = m1 - f[q];
            if (L::cz(q) == 1) m2 = m2 + f[q];
            if (L::cz(q) == -1) m2 = m2 - f[q];
          }
          const A rho = A(1) + dr;
          const A inv = A(1) / rho;
          const A ux = m0 * inv, uy = m1 * inv, uz = m2 * inv;
          const A z0 = A(0);
          A op, om, cp, cm, os;
          cell_rates<Q, A>(p, f, rho, ux, uy, uz, op, om, cp, cm, os, int64_t(cell), omega);
          if constexpr (COLL == COLL_CM)
            collide_cm<Q, false, A>(f, rho, ux, uy, uz, z0, z0, z0, os);
          else
            collide_trt<Q, false, A>(f, rho, ux, uy, uz, z0, z0, z0, op, om, cp, cm);
#pragma unroll
          for (int q = 0; q < Q; ++q) {
            A v = f[q];
            const int o = opp(q);
            const bool wall = (mask >> q) & 1u;
            if (wall && (fl & F_MOVING)) {
              const Vec4<A> wu = p.wall_u[cell + dq(q)];
              const A cu = (A(L::cx(o)) * wu.x + A(L::cy(o)) * wu.y) + A(L::cz(o)) * wu.z;
              v = v + ((A(6) * A(L::w(o))) * rho) * cu;
            }
            const int64_t off = (!ODD || wall) ? int64_t(o) * pl : int64_t(q) * pl + dq(q);
            CD::st(fb + cell + off, v);
          }
        }
      }
    }
    __syncthreads();
  }
}

}  // namespace lbmb
