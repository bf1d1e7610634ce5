// Shared device definitions: cell flags, storage codecs, small helpers.
#pragma once
#include <cuda_bf16.h>
#include <cuda_fp16.h>
#include <cuda_runtime.h>

#include <cstdint>

namespace lbmb {

// Per-cell flag byte (one byte per cell, the only per-cell array every
// cell reads besides its populations).
enum : uint8_t {
  F_SOLID = 1,     // half-way bounce-back obstacle / wall rim
  F_BOUNDARY = 2,  // fluid cell with >= 1 solid neighbour: read nbr mask
  F_MOVING = 4,    // ... and >= 1 of them has a nonzero wall velocity
  F_FORCED = 8,    // fluid cell inside an IBM stencil: read force slots
  F_WRAP = 16,     // fluid cell on a periodic face: neighbours wrap around
  F_SLIP = 32,     // fluid cell under a free-slip (specular) top wall
};

// Bit of the per-cell solid-neighbour mask (bits 0..Q-1 are directions)
// marking a cell under a free-slip top wall: a link with c_z = +1 into the
// wall reflects specularly, to direction (cx, cy, -1) of the cell
// x + (cx, cy, 0) when that cell is fluid, and bounces back otherwise.
constexpr uint32_t NBR_SLIP = 1u << 31;

// Storage codecs: populations are stored as S and computed in A. st() is
// the store of a fused step; stage() converts a value staged from the host.
template <class S>
struct Codec;

template <>
struct Codec<float> {
  using A = float;
  __device__ __forceinline__ static float ld(const float* p) { return *p; }
  __device__ __forceinline__ static void st(float* p, float v) { *p = v; }
  __device__ __forceinline__ static void stage(float* p, float v) { *p = v; }
};

template <>
struct Codec<double> {
  using A = double;
  __device__ __forceinline__ static double ld(const double* p) { return *p; }
  __device__ __forceinline__ static void st(double* p, double v) { *p = v; }
  __device__ __forceinline__ static void stage(double* p, double v) { *p = v; }
};

// The reference's host binary16 encoder (crates/lbm-core/src/gpu/
// backend.rs:160-186), used where populations are staged from the host:
// nearest with ties away from zero (the first dropped mantissa bit decides),
// magnitudes below 2^-25 flush to a signed zero, exponents >= 31 (NaN
// included) saturate to infinity. The fused steps store with the device's
// nearest-even conversion.
__device__ __forceinline__ uint16_t f16_bits_ref(float v) {
  const uint32_t x = __float_as_uint(v);
  const uint16_t sign = uint16_t((x >> 16) & 0x8000u);
  const int32_t e = int32_t((x >> 23) & 0xffu) - 127 + 15;
  const uint32_t mant = x & 0x7fffffu;
  if (e <= 0) {
    if (e < -10) return sign;
    const uint32_t m = mant | 0x800000u;
    const uint32_t shift = uint32_t(14 - e);
    uint16_t h = uint16_t(m >> shift);
    if ((m >> (shift - 1)) & 1u) h = uint16_t(h + 1);
    return uint16_t(sign | h);
  }
  if (e >= 31) return uint16_t(sign | 0x7c00u);
  uint16_t h = uint16_t(sign | (uint16_t(e) << 10) | uint16_t(mant >> 13));
  if (mant & 0x1000u) h = uint16_t(h + 1);
  return h;
}

template <>
struct Codec<__half> {
  using A = float;
  __device__ __forceinline__ static float ld(const __half* p) { return __half2float(*p); }
  __device__ __forceinline__ static void st(__half* p, float v) { *p = __float2half_rn(v); }
  __device__ __forceinline__ static void stage(__half* p, float v) { *p = __ushort_as_half(f16_bits_ref(v)); }
};

template <>
struct Codec<__nv_bfloat16> {
  using A = float;
  __device__ __forceinline__ static float ld(const __nv_bfloat16* p) { return __bfloat162float(*p); }
  __device__ __forceinline__ static void st(__nv_bfloat16* p, float v) { *p = __float2bfloat16_rn(v); }
  __device__ __forceinline__ static void stage(__nv_bfloat16* p, float v) { *p = __float2bfloat16_rn(v); }
};

// Force slot / wall velocity records (x, y, z, pad) in the arithmetic type.
template <class A>
struct Vec4 {
  A x, y, z, w;
};

// Periodic-wrap neighbour addressing for a cell at (x, y, z). Non-periodic
// faces are full solid rims (validated on the host), so the wrap is only
// ever taken by periodic axes; it never leaves the grid either way.
struct Nbr {
  int64_t zr[3];  // z rows (z-1, z, z+1) * ny
  int ys[3];
  int xs[3];
  int nx;
  __device__ __forceinline__ Nbr(int x, int y, int z, int nx_, int ny, int nz) : nx(nx_) {
    xs[0] = x == 0 ? nx_ - 1 : x - 1;
    xs[1] = x;
    xs[2] = x == nx_ - 1 ? 0 : x + 1;
    ys[0] = y == 0 ? ny - 1 : y - 1;
    ys[1] = y;
    ys[2] = y == ny - 1 ? 0 : y + 1;
    const int z0 = z == 0 ? nz - 1 : z - 1;
    const int z2 = z == nz - 1 ? 0 : z + 1;
    zr[0] = int64_t(z0) * ny;
    zr[1] = int64_t(z) * ny;
    zr[2] = int64_t(z2) * ny;
  }
  __device__ __forceinline__ int64_t at(int dx, int dy, int dz) const {
    return (zr[dz + 1] + ys[dy + 1]) * int64_t(nx) + xs[dx + 1];
  }
};

}  // namespace lbmb
