// Velocity sets in the reference's direction order
// (crates/lbm-core/src/lattice.rs:295-470). The order is load-bearing:
// OPP[q] = q+1 for odd q and q-1 for even q > 0, D3Q19 is a prefix of D3Q27,
// and TRT pair p is (2p+1, 2p+2). D3Q7 (scalar ADE only) is the first seven
// directions with w0 = 1/4, w1..6 = 1/8, cs^2 = 1/4.
#pragma once
#include <cstdint>

namespace lbmb {

template <int Q>
struct Lat;

template <>
struct Lat<19> {
  static constexpr int Q = 19, NPAIR = 9;
  static constexpr double INV_CS2 = 3.0;
  __host__ __device__ static constexpr int cx(int q) {
    constexpr int8_t t[19] = {0, 1, -1, 0, 0, 0, 0, 1, -1, 1, -1, 0, 0, 1, -1, 1, -1, 0, 0};
    return t[q];
  }
  __host__ __device__ static constexpr int cy(int q) {
    constexpr int8_t t[19] = {0, 0, 0, 1, -1, 0, 0, 1, -1, 0, 0, 1, -1, -1, 1, 0, 0, 1, -1};
    return t[q];
  }
  __host__ __device__ static constexpr int cz(int q) {
    constexpr int8_t t[19] = {0, 0, 0, 0, 0, 1, -1, 0, 0, 1, -1, 1, -1, 0, 0, -1, 1, -1, 1};
    return t[q];
  }
  __host__ __device__ static constexpr double w(int q) {
    return q == 0 ? 1.0 / 3.0 : (q < 7 ? 1.0 / 18.0 : 1.0 / 36.0);
  }
};

template <>
struct Lat<27> {
  static constexpr int Q = 27, NPAIR = 13;
  static constexpr double INV_CS2 = 3.0;
  __host__ __device__ static constexpr int cx(int q) {
    constexpr int8_t t[27] = {0, 1, -1, 0, 0, 0, 0, 1, -1, 1, -1, 0, 0, 1,
                              -1, 1, -1, 0, 0, 1, -1, 1, -1, 1, -1, 1, -1};
    return t[q];
  }
  __host__ __device__ static constexpr int cy(int q) {
    constexpr int8_t t[27] = {0, 0, 0, 1, -1, 0, 0, 1, -1, 0, 0, 1, -1, -1,
                              1, 0, 0, 1, -1, 1, -1, 1, -1, -1, 1, -1, 1};
    return t[q];
  }
  __host__ __device__ static constexpr int cz(int q) {
    constexpr int8_t t[27] = {0, 0, 0, 0, 0, 1, -1, 0, 0, 1, -1, 1, -1, 0,
                              0, -1, 1, -1, 1, 1, -1, -1, 1, 1, -1, -1, 1};
    return t[q];
  }
  __host__ __device__ static constexpr double w(int q) {
    return q == 0 ? 8.0 / 27.0 : (q < 7 ? 2.0 / 27.0 : (q < 19 ? 1.0 / 54.0 : 1.0 / 216.0));
  }
};

template <>
struct Lat<7> {
  static constexpr int Q = 7, NPAIR = 3;
  static constexpr double INV_CS2 = 4.0;
  __host__ __device__ static constexpr int cx(int q) { return Lat<19>::cx(q); }
  __host__ __device__ static constexpr int cy(int q) { return Lat<19>::cy(q); }
  __host__ __device__ static constexpr int cz(int q) { return Lat<19>::cz(q); }
  __host__ __device__ static constexpr double w(int q) { return q == 0 ? 0.25 : 0.125; }
};

__host__ __device__ constexpr int opp(int q) { return q == 0 ? 0 : ((q & 1) ? q + 1 : q - 1); }

// Index of the direction with velocity (cx, cy, cz) (-1 if absent).
template <int Q>
__host__ __device__ constexpr int find_dir(int cx, int cy, int cz) {
  for (int q = 0; q < Q; ++q)
    if (Lat<Q>::cx(q) == cx && Lat<Q>::cy(q) == cy && Lat<Q>::cz(q) == cz) return q;
  return -1;
}
// Mirror of direction q in z: (cx, cy, -cz).
template <int Q>
__host__ __device__ constexpr int mirror_z(int q) {
  return find_dir<Q>(Lat<Q>::cx(q), Lat<Q>::cy(q), -Lat<Q>::cz(q));
}
// Projection of direction q on the xy plane: (cx, cy, 0) (0 = rest).
template <int Q>
__host__ __device__ constexpr int planar(int q) {
  return find_dir<Q>(Lat<Q>::cx(q), Lat<Q>::cy(q), 0);
}

}  // namespace lbmb
