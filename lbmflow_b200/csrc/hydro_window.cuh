// Window-staged AA collide-stream: one cell per thread, populations staged
// in shared memory by the tile kernel's 16-byte cp.async windows (TRT / BGK
// or D3Q27 central moment, no uniform body force, fp32 | fp16 | bf16
// storage, any nx).
//
// A block of TILE_CELLS threads walks the compacted tile list of
// hydro_tile.cuh with a ring of STAGES window sets; thread j updates cell
// c0 + j of the tile. The windows move the populations in 16-byte chunks
// whatever the storage width, so 2-byte storage needs no per-element copy
// (cp.async has no 2-byte form) and 8 cells travel per copy instruction.
// Reads that bounce off a solid neighbour (odd step) come from the cell's
// own slot in global memory; cells on a periodic face or under the
// free-slip top take the generic path; IBM-forced cells are left to
// hydro_cells_kernel. Stores go straight to global memory through 32-bit
// offsets that depend only on launch parameters (the engine keeps Q x plane
// below 2^31). The central-moment collision takes its subgrid rate from the
// transformed order-2 moments; TRT uses the lean kernel's folded algebra.
#pragma once
#include "hydro_lean.cuh"
#include "hydro_tile.cuh"

namespace lbmb {

template <int Q, class S, int STAGES>
constexpr size_t window_smem_bytes() {
  return size_t(STAGES) * Q * TileWin<S>::LEN * sizeof(S);
}

// Ring depth for MINB resident blocks: 3 window sets where MINB x 3 fit in
// about 200 KB of shared memory per SM, else 2; 2 at 4 blocks per SM (on
// B200, deeper rings at 4 blocks ran slower).
template <int Q, class S, int MINB>
constexpr int window_stages() {
  const size_t per = window_smem_bytes<Q, S, 1>();
  const size_t fit = size_t(200 * 1024) / (size_t(MINB) * per);
  return (MINB < 4 && fit >= 3) ? 3 : 2;
}

// MINB: resident blocks of TILE_CELLS threads per SM the register
// allocation is sized for (2 = 128 registers, 3 = 85 -> 80, 4 = 64).
template <int Q, class S, bool ODD, int STAGES, int COLL, int MINB>
__global__ void __launch_bounds__(TILE_CELLS, MINB)
    hydro_window_kernel(HydroParams<float> p, const int32_t* tiles, int ntiles, TileDirs dirs, const float* omega) {
  using L = Lat<Q>;
  using W = TileWin<S>;
  using CD = Codec<S>;
  constexpr int CH = ODD ? W::CH_ODD : W::CH_EVEN;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  S* sm = reinterpret_cast<S*>(smem_raw);
  const int j = threadIdx.x;
  S* fb = static_cast<S*>(p.f);
  const int32_t pl = int32_t(p.plane);
  const int nx = p.nx, nxy = p.nxy;
  const uint32_t n = uint32_t(nxy) * uint32_t(p.nz);
  auto dq = [&](int q) -> int32_t { return L::cx(q) + L::cy(q) * nx + L::cz(q) * nxy; };
  auto P = [&](int k) -> int32_t { return k * pl; };
  auto T = [&](int k) -> int32_t { return k * pl + dq(k); };

  auto issue = [&](int i, int s) {
    if (i < ntiles) {
      const int32_t c0 = tiles[i] * TILE_CELLS;
      S* buf = sm + size_t(s) * Q * W::LEN;
      for (int k = j; k < Q * CH; k += TILE_CELLS) {
        const int q = k / CH, ch = k - q * CH;
        cp_async16(buf + q * W::LEN + ch * W::E, fb + (c0 + dirs.ws[q] + ch * W::E));
      }
    }
    cp_async_commit();
  };

  const int G = gridDim.x;
#pragma unroll
  for (int s = 0; s < STAGES - 1; ++s) issue(int(blockIdx.x) + s * G, s);
  int it = 0;
  for (int i = blockIdx.x; i < ntiles; i += G, ++it) {
    cp_async_wait<STAGES - 2>();
    __syncthreads();
    issue(i + (STAGES - 1) * G, (it + STAGES - 1) % STAGES);
    const S* w = sm + size_t(it % STAGES) * Q * W::LEN + j;
    const uint32_t c = uint32_t(tiles[i]) * TILE_CELLS + uint32_t(j);
    if (c >= n) continue;
    const uint32_t fl = p.flags[c];
    if (fl & (F_SOLID | F_FORCED)) continue;
    if (fl & (F_WRAP | F_SLIP)) {
      const int z = int(c / uint32_t(nxy));
      const int r = int(c - uint32_t(z) * uint32_t(nxy));
      const int y = r / nx;
      hydro_cell_generic_field<Q, S, COLL, ODD, false>(p, r - y * nx, y, z, c, uint8_t(fl), omega);
      continue;
    }
    const uint32_t mk = (fl & F_BOUNDARY) ? p.nbr[c] : 0u;
    S* cb = fb + c;
    float f[Q];
#pragma unroll
    for (int q = 0; q < Q; ++q) f[q] = CD::ld(w + q * W::LEN + (ODD ? dirs.r[q] : 0));
    if (ODD && mk) {
#pragma unroll
      for (int q = 0; q < Q; ++q)
        if ((mk >> opp(q)) & 1u) f[q] = CD::ld(cb + P(q));  // neighbour solid: own slot
    }
    float rho;
    if constexpr (COLL == COLL_CM) {
      float dr = 0.f, m0 = 0.f, m1 = 0.f, m2 = 0.f;
#pragma unroll
      for (int q = 0; q < Q; ++q) {
        dr += f[q];
        if (L::cx(q) == 1) m0 += f[q];
        if (L::cx(q) == -1) m0 -= f[q];
        if (L::cy(q) == 1) m1 += f[q];
        if (L::cy(q) == -1) m1 -= f[q];
        if (L::cz(q) == 1) m2 += f[q];
        if (L::cz(q) == -1) m2 -= f[q];
      }
      rho = 1.f + dr;
      const float inv = fast_rcp(rho);
      collide_cm<Q, false, float, true>(f, rho, m0 * inv, m1 * inv, m2 * inv, 0.f, 0.f, 0.f,
                                        omega ? omega[c] : p.omega_shear, p.les_c,
                                        p.tau0);
    } else {
      rho = trt_lean_collide<Q, true>(f, p, int64_t(c), omega);
    }
    if (fl & F_MOVING) {
#pragma unroll
      for (int q = 0; q < Q; ++q)
        if ((mk >> q) & 1u) {
          const int o = opp(q);
          const Vec4<float> wu = p.wall_u[int32_t(c) + dq(q)];
          f[q] += ((6.f * float(L::w(o))) * rho) * ((float(L::cx(o)) * wu.x + float(L::cy(o)) * wu.y) +
                                                    float(L::cz(o)) * wu.z);
        }
    }
    if (!ODD) {
#pragma unroll
      for (int q = 0; q < Q; ++q) CD::st(cb + P(opp(q)), f[q]);
    } else if (__all_sync(__activemask(), mk == 0u)) {
#pragma unroll
      for (int q = 0; q < Q; ++q) CD::st(cb + T(q), f[q]);
    } else {
#pragma unroll
      for (int q = 0; q < Q; ++q) CD::st(cb + (((mk >> q) & 1u) ? P(opp(q)) : T(q)), f[q]);
    }
  }
  cp_async_wait<0>();
}

}  // namespace lbmb
