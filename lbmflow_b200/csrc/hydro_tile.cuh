// Tile-pipelined AA collide-stream: two cells per thread, populations
// staged in shared memory by 16-byte cp.async copies several tiles ahead
// (TRT / BGK, no uniform body force, fp32 | fp16 | bf16 storage, even nx).
//
// A tile is TILE_CELLS consecutive cells (linear index, rows may wrap inside
// a tile). For every direction q a block copies one window of the plane it
// reads into shared memory:
//   even step: plane q,      cells [c0, c0 + TILE_CELLS)             (aligned)
//   odd step:  plane opp(q), cells [c0 - d_q, c0 - d_q + TILE_CELLS)  rounded
//              down to a 16-byte boundary (r_q elements of slack in front,
//              window TILE_CELLS + E elements, E = 16 / sizeof(S))
// with d_q = cx + cy nx + cz nx ny. r_q is the same for every tile (tile
// starts and plane sizes are multiples of E), and its parity equals the
// parity of c_x, so which directions need two element reads from shared
// memory is known at compile time. Windows stay inside the population
// allocation (guard margin on both sides of the planes).
//
// Persistent blocks walk a compacted list of tiles that hold at least one
// cell to update (solid-only tiles are never read) with a ring of STAGES
// buffers: while tile i is collided, tiles i+1 .. i+STAGES-1 are in flight,
// so the bytes in flight per SM are bounded by shared memory rather than by
// registers. By the AA ownership rule a window element that a cell uses is
// written in this step by that cell only, so prefetched windows are never
// stale; elements of the slack belong to other cells and are ignored.
//
// Reads that bounce off a solid neighbour (odd step) come from the cell's
// own slot in global memory; cells on a periodic face take the generic
// path; IBM-forced cells are left to hydro_cells_kernel. Stores go straight
// to global memory (2-element stores where the destination pair is aligned).
#pragma once
#include "hydro_async.cuh"
#include "hydro_pair.cuh"

namespace lbmb {

constexpr int TILE_CELLS = 256;
constexpr int TILE_THREADS = TILE_CELLS / 2;

template <class S>
struct TileWin {
  static constexpr int E = 16 / int(sizeof(S));      // elements per 16-byte chunk
  static constexpr int LEN = TILE_CELLS + E;          // window elements (odd step)
  static constexpr int CH_EVEN = TILE_CELLS / E;      // chunks per window
  static constexpr int CH_ODD = TILE_CELLS / E + 1;
};

template <int Q, class S, int STAGES>
constexpr size_t tile_smem_bytes() {
  return size_t(STAGES) * Q * TileWin<S>::LEN * sizeof(S);
}

// Per-direction window start (elements, relative to the tile's first cell)
// and read offset inside the window, for one parity.
struct TileDirs {
  int32_t ws[27];
  int32_t r[27];
};

__device__ __forceinline__ void cp_async16(void* dst_smem, const void* src) {
  const uint32_t d = static_cast<uint32_t>(__cvta_generic_to_shared(dst_smem));
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(d), "l"(src) : "memory");
}

template <int Q, class S, bool ODD, int STAGES, int COLL = COLL_TRT>
__global__ void __launch_bounds__(TILE_THREADS, COLL == COLL_CM ? 2 : 3)
    hydro_tile_kernel(HydroParams<float> p, const int32_t* tiles, int ntiles, TileDirs dirs) {
  using L = Lat<Q>;
  using W = TileWin<S>;
  using IO = PairIO<S>;
  constexpr int CH = ODD ? W::CH_ODD : W::CH_EVEN;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  S* sm = reinterpret_cast<S*>(smem_raw);
  const int j = threadIdx.x;
  S* fb = static_cast<S*>(p.f);
  const uint32_t pl = p.plane;
  const int nx = p.nx, nxy = p.nxy;
  auto dq = [&](int q) { return L::cx(q) + L::cy(q) * nx + L::cz(q) * nxy; };

  auto issue = [&](int i, int s) {
    if (i < ntiles) {
      const int32_t c0 = tiles[i] * TILE_CELLS;
      S* buf = sm + size_t(s) * Q * W::LEN;
      for (int k = j; k < Q * CH; k += TILE_THREADS) {
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
    const S* w = sm + size_t(it % STAGES) * Q * W::LEN;
    const uint32_t c = uint32_t(tiles[i]) * TILE_CELLS + 2 * j;
    if (c >= uint32_t(p.nx) * uint32_t(p.ny) * uint32_t(p.nz)) continue;
    const uint32_t fl2 = reinterpret_cast<const uint16_t*>(p.flags)[c >> 1];
    const uint32_t fl0 = fl2 & 0xffu, fl1 = fl2 >> 8;
    const bool act0 = !(fl0 & (F_SOLID | F_FORCED)), act1 = !(fl1 & (F_SOLID | F_FORCED));
    if (!(act0 || act1)) continue;
    if ((fl0 | fl1) & (F_WRAP | F_SLIP)) {
      const int z = int(c / uint32_t(nxy));
      const int r = int(c - uint32_t(z) * uint32_t(nxy));
      const int y = r / nx, x = r - y * nx;
      if (act0) hydro_cell_generic<Q, S, COLL, ODD, false>(p, x, y, z, c, uint8_t(fl0));
      if (act1) hydro_cell_generic<Q, S, COLL, ODD, false>(p, x + 1, y, z, c + 1, uint8_t(fl1));
      continue;
    }
    const uint32_t mk0 = (fl0 & F_BOUNDARY) ? p.nbr[c] : 0u;
    const uint32_t mk1 = (fl1 & F_BOUNDARY) ? p.nbr[c + 1] : 0u;
    const uint32_t mk = mk0 | mk1;
    float2 f[Q];
#pragma unroll
    for (int q = 0; q < Q; ++q) {
      const S* src = w + q * W::LEN + 2 * j + (ODD ? dirs.r[q] : 0);
      if (ODD && (L::cx(q) & 1)) f[q] = make_float2(IO::ld1(src), IO::ld1(src + 1));
      else f[q] = IO::ld2(src);
      if (ODD) {
        const int o = opp(q);
        if ((mk >> o) & 1u) {
          const S* own = fb + (uint32_t(q) * pl + c);
          if ((mk0 >> o) & 1u) f[q].x = IO::ld1(own);
          if ((mk1 >> o) & 1u) f[q].y = IO::ld1(own + 1);
        }
      }
    }
    const float2 rho = pair_collide<Q, COLL>(f, p);
    const bool both = act0 && act1;
    const bool moving = (fl0 | fl1) & F_MOVING;
#pragma unroll
    for (int q = 0; q < Q; ++q) {
      const int o = opp(q);
      float2 v = f[q];
      const bool w0 = (mk0 >> q) & 1u, w1 = (mk1 >> q) & 1u;
      if (moving && (w0 || w1)) {
        const float k6 = 6.f * float(L::w(o));
        if (w0 && (fl0 & F_MOVING)) {
          const Vec4<float> wu = p.wall_u[int32_t(c) + dq(q)];
          v.x += (k6 * rho.x) * ((float(L::cx(o)) * wu.x + float(L::cy(o)) * wu.y) + float(L::cz(o)) * wu.z);
        }
        if (w1 && (fl1 & F_MOVING)) {
          const Vec4<float> wu = p.wall_u[int32_t(c) + 1 + dq(q)];
          v.y += (k6 * rho.y) * ((float(L::cx(o)) * wu.x + float(L::cy(o)) * wu.y) + float(L::cz(o)) * wu.z);
        }
      }
      S* own = fb + (uint32_t(o) * pl + c);
      if (!ODD) {
        if (both) {
          IO::st2(own, v);
        } else {
          if (act0) IO::st1(own, v.x);
          if (act1) IO::st1(own + 1, v.y);
        }
      } else {
        S* dst = fb + int32_t(uint32_t(q) * pl + c + uint32_t(dq(q)));
        if (both && !((mk >> q) & 1u)) {
          if (L::cx(q) & 1) {
            IO::st1(dst, v.x);
            IO::st1(dst + 1, v.y);
          } else {
            IO::st2(dst, v);
          }
        } else {
          if (act0) IO::st1(w0 ? own : dst, v.x);
          if (act1) IO::st1(w1 ? own + 1 : dst + 1, v.y);
        }
      }
    }
  }
  cp_async_wait<0>();
}

}  // namespace lbmb
