// One cell per thread AA collide-stream with a small register footprint
// (TRT / BGK, no uniform body force, fp32 | fp16 | bf16 storage).
//
// The kernel is built for occupancy: a flat grid over the cells, 32-bit
// element offsets, a branch-free pointer select for directions that bounce
// off a solid neighbour, the pair-folded TRT algebra of hydro_pair.cuh in
// scalar form (S = f_a + f_b and D = f_a - f_b are recomputed where they are
// needed instead of being kept live), and single-instruction reciprocals.
// With 16-bit storage every access is one element, so no direction needs
// alignment handling and the odd step costs the same instructions as the
// even one; latency is hidden by the number of resident warps.
#pragma once
#include "hydro_pair.cuh"

namespace lbmb {

constexpr int LEAN_BLOCK = 128;

// FIELD: take omega+ from the per-cell relaxation field when one is set
// (the window kernel); the lean kernel is never launched with a field.
template <int Q, bool FIELD = false>
__device__ __forceinline__ float trt_lean_collide(float (&f)[Q], const HydroParams<float>& p, int64_t cell,
                                                  const float* omega = nullptr) {
  using L = Lat<Q>;
  constexpr int NP = (Q - 1) / 2;
  static_assert(pair_heads_positive<Q>(), "pair head convention");
  float drho = f[0];
  float jx = 0.f, jy = 0.f, jz = 0.f;
#pragma unroll
  for (int k = 0; k < NP; ++k) {
    const int a = 2 * k + 1, b = a + 1;
    drho += f[a] + f[b];
    const float d = f[a] - f[b];
    if (L::cx(a) == 1) jx += d;
    if (L::cx(a) == -1) jx -= d;
    if (L::cy(a) == 1) jy += d;
    if (L::cy(a) == -1) jy -= d;
    if (L::cz(a) == 1) jz += d;
    if (L::cz(a) == -1) jz -= d;
  }
  const float rho = drho + 1.f;
  const float inv = rcp_fast(rho);
  const float ux = jx * inv, uy = jy * inv, uz = jz * inv;
  const float usq = ux * ux + uy * uy + uz * uz;
  float op = (FIELD && omega) ? omega[cell] : p.omega_p, om = p.omega_m;
  if (p.les_c > 0.f) {
    float s[6] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
#pragma unroll
    for (int k = 0; k < NP; ++k) {
      const int a = 2 * k + 1;
      const int cx = L::cx(a), cy = L::cy(a), cz = L::cz(a);
      const float sv = f[a] + f[a + 1];
      if (cx) s[0] += sv;
      if (cy) s[1] += sv;
      if (cz) s[2] += sv;
      if (cx && cy) s[3] += float(cx * cy) * sv;
      if (cx && cz) s[4] += float(cx * cz) * sv;
      if (cy && cz) s[5] += float(cy * cz) * sv;
    }
    const float te = les_tau_pair<Q>(s, rho, inv, ux, uy, uz, p.les_c, p.tau0);
    op = rcp_fast(te);
    if (p.magic > 0.f) {
      const float l = te - 0.5f;
      om = l * rcp_fast(p.magic + 0.5f * l);
    } else {
      om = op;
    }
  }
  const float base = drho - 1.5f * rho * usq;
  const float nhop = -0.5f * op, hom = 0.5f * om;
  float oA[3], oB[3], nC[3];
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    const int a = k == 0 ? 1 : (k == 1 ? 7 : 19);
    if (a >= Q) continue;
    const float w = float(L::w(a));
    oA[k] = (op * w) * base;
    oB[k] = (op * (4.5f * w)) * rho;
    nC[k] = (om * (-3.f * w)) * rho;
  }
  f[0] = (1.f - op) * f[0] + (op * float(L::w(0))) * base;
#pragma unroll
  for (int k = 0; k < NP; ++k) {
    const int a = 2 * k + 1, b = a + 1;
    const int cl = wclass<Q>(a);
    float cu = L::cx(a) ? ux : (L::cy(a) ? uy : uz);
    if (L::cx(a) && L::cy(a)) cu = L::cy(a) > 0 ? cu + uy : cu - uy;
    if ((L::cx(a) || L::cy(a)) && L::cz(a)) cu = L::cz(a) > 0 ? cu + uz : cu - uz;
    const float t = oB[cl] * (cu * cu) + oA[cl];
    const float pn = nhop * (f[a] + f[b]) + t;     // -rp
    const float m = nC[cl] * cu + hom * (f[a] - f[b]);  // rm
    f[a] = (f[a] + pn) - m;
    f[b] = (f[b] + pn) + m;
  }
  return rho;
}

// Update of one cell (c < number of cells) with the lean kernel's code.
template <int Q, class S, bool ODD>
__device__ __forceinline__ void lean_cell(const HydroParams<float>& p, uint32_t c) {
  using L = Lat<Q>;
  using CD = Codec<S>;
  const uint32_t fl = p.flags[c];
  if (fl & (F_SOLID | F_FORCED)) return;
  const int nx = p.nx, nxy = p.nxy;
  if (fl & (F_WRAP | F_SLIP)) {
    const int z = int(c / uint32_t(nxy));
    const int r = int(c - uint32_t(z) * uint32_t(nxy));
    const int y = r / nx;
    hydro_cell_generic<Q, S, COLL_TRT, ODD, false>(p, r - y * nx, y, z, c, uint8_t(fl));
    return;
  }
  const uint32_t mk = (fl & F_BOUNDARY) ? p.nbr[c] : 0u;
  // Per-thread base pointer plus per-direction offsets that depend on the
  // launch parameters only (uniform across the grid).
  S* cb = static_cast<S*>(p.f) + c;
  const int64_t pl = int64_t(p.plane);
  // P(k): slot k of this cell; T(k): slot k of the neighbour x + c_k. The
  // odd step reads slot opp(q) of x - c_q = T(opp(q)) and writes T(q), so
  // loads and stores share one set of offsets.
  auto P = [&](int k) { return int32_t(int64_t(k) * pl); };
  auto T = [&](int k) { return int32_t(int64_t(k) * pl + (L::cx(k) + L::cy(k) * nx + L::cz(k) * nxy)); };
  // Odd step: a warp whose active cells have no solid neighbour (the bulk
  // of the tank) takes straight neighbour accesses; the others test the
  // solid-neighbour mask per direction. The vote is warp-uniform.
  const bool clear = ODD && __all_sync(__activemask(), mk == 0u);
  float f[Q];
  if (clear) {
#pragma unroll
    for (int q = 0; q < Q; ++q) f[q] = CD::ld(cb + T(opp(q)));
  } else {
#pragma unroll
    for (int q = 0; q < Q; ++q) {
      if (!ODD) {
        f[q] = CD::ld(cb + P(q));
      } else {
        const int o = opp(q);
        f[q] = CD::ld(cb + T(o));
        if ((mk >> o) & 1u) f[q] = CD::ld(cb + P(q));  // neighbour solid: own slot
      }
    }
  }
  const float rho = trt_lean_collide<Q>(f, p, int64_t(c));
  if (fl & F_MOVING) {
#pragma unroll
    for (int q = 0; q < Q; ++q) {
      const int o = opp(q);
      if ((mk >> q) & 1u) {
        const Vec4<float> wu = p.wall_u[int64_t(c) + (T(q) - P(q))];
        f[q] += ((6.f * float(L::w(o))) * rho) *
                ((float(L::cx(o)) * wu.x + float(L::cy(o)) * wu.y) + float(L::cz(o)) * wu.z);
      }
    }
  }
  // even step: a fresh copy of the base pointer keeps the compiler from
  // holding the load addresses (the same offsets) live across the collision
  if constexpr (!ODD) asm volatile("" : "+l"(cb));
  if (clear) {
#pragma unroll
    for (int q = 0; q < Q; ++q) CD::st(cb + T(q), f[q]);
  } else {
#pragma unroll
    for (int q = 0; q < Q; ++q) {
      const int o = opp(q);
      if (!ODD || ((mk >> q) & 1u))
        CD::st(cb + P(o), f[q]);  // even step, or towards a wall: the own slot
      else
        CD::st(cb + T(q), f[q]);
    }
  }
}

// MINB: resident blocks per SM the register allocation is sized for
// (8: 64 registers, 7: 72, 6: 80).
template <int Q, class S, bool ODD, int MINB>
__global__ void __launch_bounds__(LEAN_BLOCK, MINB) hydro_lean_kernel(HydroParams<float> p, uint32_t n) {
  const uint32_t c = blockIdx.x * LEAN_BLOCK + threadIdx.x;
  if (c >= n) return;
  lean_cell<Q, S, ODD>(p, c);
}

}  // namespace lbmb
