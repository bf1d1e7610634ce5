// Software-pipelined AA collide-stream with per-thread asynchronous copies.
//
// Persistent blocks of 128 threads walk the grid in 128-cell tiles. Each
// thread keeps a ring of STAGES x Q population slots in shared memory (its
// own column: [stage][q][thread]) and, while colliding the cell of tile i,
// already has the populations of its cells in tiles i+1 .. i+STAGES-1 in
// flight (cp.async, 4/8-byte copies). A thread only ever reads back what it
// copied itself, so cp.async.wait_group is the only synchronisation: there
// are no block barriers and no spin loops. The copy addresses follow the AA
// rule of hydro.cuh (odd step: slot opp(q) of x - c_q, own slot q when that
// neighbour is solid) as branchless selects; cells on a periodic face use
// the out-of-line generic path, which keeps the unrolled body small enough
// for the instruction cache. Requires 4- or 8-byte population storage.
#pragma once
#include "hydro.cuh"

namespace lbmb {

constexpr int ASYNC_TILE = 128;

// Shared memory per block: the population ring [stage][q][thread], then per
// stage and thread the solid-neighbour mask (u32) and the flags (u8) the
// copies were issued with.
template <int Q, class S, int STAGES>
constexpr size_t async_smem_bytes() {
  return size_t(STAGES) * ASYNC_TILE * (Q * sizeof(S) + sizeof(uint32_t) + sizeof(uint8_t));
}

template <class S>
__device__ __forceinline__ void cp_async_elem(S* dst_smem, const S* src) {
  static_assert(sizeof(S) == 4 || sizeof(S) == 8, "cp.async needs 4- or 8-byte elements");
  const uint32_t d = static_cast<uint32_t>(__cvta_generic_to_shared(dst_smem));
  if constexpr (sizeof(S) == 4)
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4;" ::"r"(d), "l"(src) : "memory");
  else
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" ::"r"(d), "l"(src) : "memory");
}

__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }

template <int N>
__device__ __forceinline__ void cp_async_wait() {
  asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory");
}

// MINB: resident blocks per SM the register allocation is sized for (fp32:
// 4 = 128 registers, 5 = 96 (102), 6 = 80 (85); the ring of STAGES x Q x 128
// elements per block must fit MINB times in shared memory).
template <int Q, class S, int COLL, bool ODD, int STAGES, int MINB = HydroOccupancy<typename Codec<S>::A>::MIN_BLOCKS>
__global__ void __launch_bounds__(ASYNC_TILE, MINB)
    hydro_async_kernel(HydroParams<typename Codec<S>::A> p, int64_t ncells, int ntiles) {
  using A = typename Codec<S>::A;
  using L = Lat<Q>;
  using CD = Codec<S>;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  S* sm = reinterpret_cast<S*>(smem_raw);
  uint32_t* smk = reinterpret_cast<uint32_t*>(smem_raw + size_t(STAGES) * Q * ASYNC_TILE * sizeof(S));
  uint8_t* sfl = reinterpret_cast<uint8_t*>(smk + STAGES * ASYNC_TILE);
  const int j = threadIdx.x;
  S* fb = static_cast<S*>(p.f);
  // 32-bit element offsets relative to the cell (the engine keeps Q x plane
  // below 2^31). P(k): slot k of the cell; T(k): slot k of the neighbour
  // x + c_k (the odd step reads T(opp q) and writes T(q)); both depend on
  // launch parameters only.
  const int32_t pl = int32_t(p.plane);
  const int nx = p.nx, nxy = p.nxy;
  auto dq = [&](int q) -> int32_t { return L::cx(q) + L::cy(q) * nx + L::cz(q) * nxy; };
  auto P = [&](int k) -> int32_t { return k * pl; };
  auto T = [&](int k) -> int32_t { return k * pl + dq(k); };
  // Cells on a periodic face take the out-of-line generic path; all other
  // active cells go through the pipeline.
  auto piped = [&](uint8_t fl) { return !(fl & (F_SOLID | F_FORCED | F_WRAP | F_SLIP)); };
  // Flags of this thread's cell in tile t (solid past the grid). They are
  // loaded one tile ahead of the copies that need them, so their latency
  // hides behind a collision.
  auto flags_of = [&](int t) -> uint8_t {
    const int64_t cell = int64_t(t) * ASYNC_TILE + j;
    return (t < ntiles && cell < ncells) ? p.flags[cell] : uint8_t(F_SOLID);
  };
  // Issue the copies of this thread's cell in tile t (flags fl) into ring
  // stage s; the flags and mask go to the stage's metadata for the collision.
  auto issue = [&](int t, int s, uint8_t fl) {
    const int64_t cell = int64_t(t) * ASYNC_TILE + j;
    uint32_t mk = 0u;
    if (piped(fl)) {
      if (fl & F_BOUNDARY) mk = p.nbr[cell];
      S* dst = sm + size_t(s) * Q * ASYNC_TILE + j;
      const S* src0 = fb + cell;
      if (!ODD) {
#pragma unroll
        for (int q = 0; q < Q; ++q) cp_async_elem(dst + q * ASYNC_TILE, src0 + P(q));
      } else {
        const uint32_t mask = mk;
        // a warp whose cells have no solid neighbour copies straight from
        // the neighbours (warp-uniform vote); the others select per link
        if (__all_sync(__activemask(), mask == 0u)) {
#pragma unroll
          for (int q = 0; q < Q; ++q) cp_async_elem(dst + q * ASYNC_TILE, src0 + T(opp(q)));
        } else {
#pragma unroll
          for (int q = 0; q < Q; ++q) {
            const int o = opp(q);
            cp_async_elem(dst + q * ASYNC_TILE, src0 + (((mask >> o) & 1u) ? P(q) : T(o)));
          }
        }
      }
    }
    smk[s * ASYNC_TILE + j] = mk;
    sfl[s * ASYNC_TILE + j] = fl;
    cp_async_commit();
  };
  const int G = int(gridDim.x);
  uint8_t fl_next = flags_of(int(blockIdx.x));
#pragma unroll
  for (int s = 0; s < STAGES - 1; ++s) {
    const int t = int(blockIdx.x) + s * G;
    const uint8_t fl = fl_next;
    fl_next = flags_of(t + G);
    issue(t, s, fl);
  }
  int it = 0;
  for (int t = blockIdx.x; t < ntiles; t += G, ++it) {
    {
      const int tn = t + (STAGES - 1) * G;
      const uint8_t fl = fl_next;
      fl_next = flags_of(tn + G);
      issue(tn, (it + STAGES - 1) % STAGES, fl);
    }
    cp_async_wait<STAGES - 1>();
    const int64_t cell = int64_t(t) * ASYNC_TILE + j;
    const int stage = it % STAGES;
    const uint8_t fl = sfl[stage * ASYNC_TILE + j];
    if (fl & (F_SOLID | F_FORCED)) continue;
    if (fl & (F_WRAP | F_SLIP)) {
      const int z = int(cell / nxy);
      const int64_t r = cell - int64_t(z) * nxy;
      const int y = int(r / nx);
      hydro_cell_generic<Q, S, COLL, ODD, false>(p, int(r - int64_t(y) * nx), y, z, uint32_t(cell), fl);
      continue;
    }
    const S* src = sm + size_t(stage) * Q * ASYNC_TILE + j;
    A f[Q];
#pragma unroll
    for (int q = 0; q < Q; ++q) f[q] = CD::ld(src + q * ASYNC_TILE);
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
    const A inv = fast_rcp(rho);
    const A ux = m0 * inv, uy = m1 * inv, uz = m2 * inv;
    const A z0 = A(0);
    if constexpr (COLL == COLL_CM) {
      // subgrid rate from the transformed moments (fp32), else les_tau
      constexpr bool LK = std::is_same<A, float>::value;
      A os = p.omega_shear;
      if constexpr (!LK) {
        A op, om, cp, cm;
        cell_rates<Q, A>(p, f, rho, ux, uy, uz, op, om, cp, cm, os);
      }
      collide_cm<Q, false, A, LK>(f, rho, ux, uy, uz, z0, z0, z0, os, p.les_c, p.tau0);
    } else {
      A op, om, cp, cm, os;
      cell_rates<Q, A, true>(p, f, rho, ux, uy, uz, op, om, cp, cm, os);
      collide_trt<Q, false, A>(f, rho, ux, uy, uz, z0, z0, z0, op, om, cp, cm);
    }
    const uint32_t mask = smk[stage * ASYNC_TILE + j];
    S* dst0 = fb + cell;
    if (fl & F_MOVING) {
#pragma unroll
      for (int q = 0; q < Q; ++q)
        if ((mask >> q) & 1u) {
          const int o = opp(q);
          const Vec4<A> wu = p.wall_u[cell + dq(q)];
          const A cu = (A(L::cx(o)) * wu.x + A(L::cy(o)) * wu.y) + A(L::cz(o)) * wu.z;
          f[q] = f[q] + ((A(6) * A(L::w(o))) * rho) * cu;
        }
    }
    if (!ODD) {
#pragma unroll
      for (int q = 0; q < Q; ++q) CD::st(dst0 + P(opp(q)), f[q]);
    } else if (__all_sync(__activemask(), mask == 0u)) {
#pragma unroll
      for (int q = 0; q < Q; ++q) CD::st(dst0 + T(q), f[q]);
    } else {
#pragma unroll
      for (int q = 0; q < Q; ++q) CD::st(dst0 + (((mask >> q) & 1u) ? P(opp(q)) : T(q)), f[q]);
    }
  }
  cp_async_wait<0>();
}

}  // namespace lbmb
