// Two cells per thread AA collide-stream with packed fp32x2 arithmetic
// (TRT / BGK or D3Q27 central moment, no uniform body force, fp32 | fp16 |
// bf16 storage).
//
// Thread i owns the x-adjacent cells c = 2i and c + 1 (nx even, so a pair
// never straddles a row and every plane offset q * plane + c is even).
// Both cells' populations of a direction travel as one 2-element access
// whenever the pair's source (or destination) window starts on an even
// cell, which is every direction with c_x = 0 on the odd step and every
// direction on the even step; directions with c_x = +-1 on the odd step
// use two element accesses at consecutive addresses. The collision runs on
// float2 registers with the sm_100 packed FADD2/FMUL2/FFMA2 instructions,
// so one instruction advances both cells.
//
// TRT algebra (collision.rs:123-202 without a force term), per TRT pair
// (a, b = opp(a)) with cu = c_a . u, S = f_a + f_b, D = f_a - f_b and
// weight w of the pair:
//   rp = omega+ (S/2 - w (drho + rho (4.5 cu^2 - 1.5 u^2)))
//   rm = omega- (D/2 - 3 w rho cu)
//   f_a' = f_a - rp - rm,   f_b' = f_b - rp + rm
// i.e. the same operator as the reference with the pair sums folded
// algebraically (rounding differs from the reference's operand order at the
// level of one ulp per operation; the parity tests bound it).
//
// Walls, moving walls and the AA ownership rule follow hydro.cuh; pairs
// with a solid neighbour in a direction fall back to per-cell element
// accesses for that direction only. Cells inside IBM stencils are left to
// hydro_cells_kernel; cells on a periodic face take the generic path.
#pragma once
#include <cuda_fp16.h>
#include "hydro.cuh"

namespace lbmb {

constexpr int PAIR_BLOCK = 128;

__device__ __forceinline__ float2 add2(float2 a, float2 b) { return __fadd2_rn(a, b); }
__device__ __forceinline__ float2 mul2(float2 a, float2 b) { return __fmul2_rn(a, b); }
__device__ __forceinline__ float2 fma2(float2 a, float2 b, float2 c) { return __ffma2_rn(a, b, c); }
__device__ __forceinline__ float2 sub2(float2 a, float2 b) { return __ffma2_rn(b, make_float2(-1.f, -1.f), a); }
__device__ __forceinline__ float2 bc2(float a) { return make_float2(a, a); }

// Single-instruction reciprocal and square root (PTX rcp/sqrt .approx, a few
// ulp). Used for 1/rho and the subgrid model, where the IEEE-rounded forms
// cost a slow-path branch per call; the parity tests bound the difference.
__device__ __forceinline__ float rcp_fast(float x) {
  float r;
  asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
  return r;
}
__device__ __forceinline__ float sqrt_fast(float x) {
  float r;
  asm("sqrt.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
  return r;
}

// Two adjacent storage elements <-> float2.
template <class S>
struct PairIO;

template <>
struct PairIO<float> {
  __device__ __forceinline__ static float2 ld2(const float* p) { return *reinterpret_cast<const float2*>(p); }
  __device__ __forceinline__ static float ld1(const float* p) { return *p; }
  __device__ __forceinline__ static void st2(float* p, float2 v) { *reinterpret_cast<float2*>(p) = v; }
  __device__ __forceinline__ static void st1(float* p, float v) { *p = v; }
};

template <>
struct PairIO<__half> {
  __device__ __forceinline__ static float2 ld2(const __half* p) {
    return __half22float2(*reinterpret_cast<const __half2*>(p));
  }
  __device__ __forceinline__ static float ld1(const __half* p) { return __half2float(*p); }
  __device__ __forceinline__ static void st2(__half* p, float2 v) {
    *reinterpret_cast<__half2*>(p) = __float22half2_rn(v);
  }
  __device__ __forceinline__ static void st1(__half* p, float v) { *p = __float2half_rn(v); }
};

template <>
struct PairIO<__nv_bfloat16> {
  __device__ __forceinline__ static float2 ld2(const __nv_bfloat16* p) {
    return __bfloat1622float2(*reinterpret_cast<const __nv_bfloat162*>(p));
  }
  __device__ __forceinline__ static float ld1(const __nv_bfloat16* p) { return __bfloat162float(*p); }
  __device__ __forceinline__ static void st2(__nv_bfloat16* p, float2 v) {
    *reinterpret_cast<__nv_bfloat162*>(p) = __float22bfloat162_rn(v);
  }
  __device__ __forceinline__ static void st1(__nv_bfloat16* p, float v) { *p = __float2bfloat16_rn(v); }
};

// Every first member a = 2k + 1 of a TRT pair has its first nonzero velocity
// component equal to +1 (lattice.rs direction order), so c_a . u needs no
// negation of its leading term.
template <int Q>
__host__ __device__ constexpr bool pair_heads_positive() {
  using L = Lat<Q>;
  for (int a = 1; a < Q; a += 2) {
    const int lead = L::cx(a) ? L::cx(a) : (L::cy(a) ? L::cy(a) : L::cz(a));
    if (lead != 1) return false;
  }
  return true;
}

// Weight class of a direction: 0 = axis, 1 = face diagonal, 2 = corner.
template <int Q>
__host__ __device__ constexpr int wclass(int q) {
  return (Lat<Q>::cx(q) != 0) + (Lat<Q>::cy(q) != 0) + (Lat<Q>::cz(q) != 0) - 1;
}

// LES-adjusted tau for one cell from the pair sums (Pi uses S only).
template <int Q>
__device__ __forceinline__ float les_tau_pair(const float (&s)[6], float rho, float inv_rho, float ux, float uy,
                                              float uz, float les_c, float tau0) {
  const float d3 = (rho - 1.f) * (1.f / 3.f);
  const float pxx = s[0] - d3 - rho * ux * ux, pyy = s[1] - d3 - rho * uy * uy, pzz = s[2] - d3 - rho * uz * uz;
  const float pxy = s[3] - rho * ux * uy, pxz = s[4] - rho * ux * uz, pyz = s[5] - rho * uy * uz;
  const float pn = sqrt_fast((pxx * pxx + pyy * pyy + pzz * pzz) + 2.f * (pxy * pxy + pxz * pxz + pyz * pyz));
  return 0.5f * (tau0 + sqrt_fast(tau0 * tau0 + les_c * pn * inv_rho));
}

// TRT collision of two cells in float2 lanes in register-lean form: the
// operator of trt_pair_collide (hydro_pair.cuh), with the pair sums
// S = f_a + f_b and differences D = f_a - f_b recomputed where they are used
// instead of being held for all pairs (the form of trt_lean_collide).
template <int Q>
__device__ __forceinline__ float2 trt_pair_lean(float2 (&f)[Q], const HydroParams<float>& p) {
  using L = Lat<Q>;
  constexpr int NP = (Q - 1) / 2;
  static_assert(pair_heads_positive<Q>(), "pair head convention");
  float2 drho = f[0], jx = bc2(0.f), jy = bc2(0.f), jz = bc2(0.f);
#pragma unroll
  for (int k = 0; k < NP; ++k) {
    const int a = 2 * k + 1, b = a + 1;
    drho = add2(drho, add2(f[a], f[b]));
    const float2 d = sub2(f[a], f[b]);
    if (L::cx(a) == 1) jx = add2(jx, d);
    if (L::cx(a) == -1) jx = sub2(jx, d);
    if (L::cy(a) == 1) jy = add2(jy, d);
    if (L::cy(a) == -1) jy = sub2(jy, d);
    if (L::cz(a) == 1) jz = add2(jz, d);
    if (L::cz(a) == -1) jz = sub2(jz, d);
  }
  const float2 rho = add2(drho, bc2(1.f));
  const float2 inv = make_float2(rcp_fast(rho.x), rcp_fast(rho.y));
  const float2 ux = mul2(jx, inv), uy = mul2(jy, inv), uz = mul2(jz, inv);
  const float2 usq = fma2(ux, ux, fma2(uy, uy, mul2(uz, uz)));
  float2 op = bc2(p.omega_p), om = bc2(p.omega_m);
  if (p.les_c > 0.f) {
    // second moments of the pair sums, both lanes at once
    float2 s6[6] = {bc2(0.f), bc2(0.f), bc2(0.f), bc2(0.f), bc2(0.f), bc2(0.f)};
#pragma unroll
    for (int k = 0; k < NP; ++k) {
      const int a = 2 * k + 1;
      const int cx = L::cx(a), cy = L::cy(a), cz = L::cz(a);
      const float2 sv = add2(f[a], f[a + 1]);
      if (cx) s6[0] = add2(s6[0], sv);
      if (cy) s6[1] = add2(s6[1], sv);
      if (cz) s6[2] = add2(s6[2], sv);
      if (cx && cy) s6[3] = cx * cy > 0 ? add2(s6[3], sv) : sub2(s6[3], sv);
      if (cx && cz) s6[4] = cx * cz > 0 ? add2(s6[4], sv) : sub2(s6[4], sv);
      if (cy && cz) s6[5] = cy * cz > 0 ? add2(s6[5], sv) : sub2(s6[5], sv);
    }
    const float sa[6] = {s6[0].x, s6[1].x, s6[2].x, s6[3].x, s6[4].x, s6[5].x};
    const float sb[6] = {s6[0].y, s6[1].y, s6[2].y, s6[3].y, s6[4].y, s6[5].y};
    const float te0 = les_tau_pair<Q>(sa, rho.x, inv.x, ux.x, uy.x, uz.x, p.les_c, p.tau0);
    const float te1 = les_tau_pair<Q>(sb, rho.y, inv.y, ux.y, uy.y, uz.y, p.les_c, p.tau0);
    op = make_float2(rcp_fast(te0), rcp_fast(te1));
    if (p.magic > 0.f) {
      const float l0 = te0 - 0.5f, l1 = te1 - 0.5f;
      om = make_float2(l0 * rcp_fast(p.magic + 0.5f * l0), l1 * rcp_fast(p.magic + 0.5f * l1));
    } else {
      om = op;
    }
  }
  const float2 base = fma2(mul2(rho, bc2(-1.5f)), usq, drho);
  const float2 nhop = mul2(op, bc2(-0.5f)), hom = mul2(om, bc2(0.5f));
  f[0] = fma2(sub2(bc2(1.f), op), f[0], mul2(mul2(op, bc2(float(L::w(0)))), base));
  // the pairs come in weight classes (axis, face diagonal, corner) in
  // direction order; a class's coefficients are formed where it starts
  float2 oA = bc2(0.f), oB = bc2(0.f), nC = bc2(0.f);
#pragma unroll
  for (int k = 0; k < NP; ++k) {
    const int a = 2 * k + 1, b = a + 1;
    if (k == 0 || wclass<Q>(a) != wclass<Q>(a - 2)) {
      const float w = float(L::w(a));
      oA = mul2(mul2(op, bc2(w)), base);
      oB = mul2(mul2(op, bc2(4.5f * w)), rho);
      nC = mul2(mul2(om, bc2(-3.f * w)), rho);
    }
    float2 cu = L::cx(a) ? ux : (L::cy(a) ? uy : uz);
    if (L::cx(a) && L::cy(a)) cu = L::cy(a) > 0 ? add2(cu, uy) : sub2(cu, uy);
    if ((L::cx(a) || L::cy(a)) && L::cz(a)) cu = L::cz(a) > 0 ? add2(cu, uz) : sub2(cu, uz);
    const float2 t = fma2(oB, mul2(cu, cu), oA);
    const float2 pn = fma2(nhop, add2(f[a], f[b]), t);          // -rp
    const float2 m = fma2(nC, cu, mul2(hom, sub2(f[a], f[b])));  // rm
    f[a] = sub2(add2(f[a], pn), m);
    f[b] = add2(add2(f[b], pn), m);
  }
  return rho;
}

// Backward central-moment transform of one line (the values at c = -1, 0,
// +1 from the central moments of order 0, 1, 2 about u; cm_bwd of hydro.cuh)
// on float2 lanes.
__device__ __forceinline__ void cm_bwd2(float2& k0, float2& k1, float2& k2, float2 u) {
  const float2 m1 = fma2(u, k0, k1);
  const float2 m2 = fma2(mul2(u, u), k0, fma2(mul2(u, bc2(2.f)), k1, k2));
  const float2 fm = mul2(bc2(0.5f), sub2(m2, m1));
  const float2 f0 = sub2(k0, m2);
  const float2 fp = mul2(bc2(0.5f), add2(m2, m1));
  k0 = fm;
  k1 = f0;
  k2 = fp;
}

// D3Q27 central-moment collision (kernels.rs:406-533, no force) of two
// cells in float2 lanes, in the regularized form of collide_cm_x2
// (hydro_async.cuh): f' = feq + T^-1 K', where K' holds only the five
// deviatoric order-2 central moments (1 - omega_s)(Pi - tr Pi / 3) of the
// non-equilibrium stress Pi; the backward transform runs on that sparse
// vector (x pass by fixed per-axis shape functions, then the y and z passes
// of the factorised transform). A lane at exact rest (u = 0 and every
// population w (rho - 1), kernels.rs:434-447) keeps its populations.
template <int Q>
__device__ __forceinline__ float2 cm_pair_reg(float2 (&f)[Q], const HydroParams<float>& p) {
  static_assert(Q == 27, "central moments need the full D3Q27 tensor basis");
  using L = Lat<Q>;
  constexpr int NP = (Q - 1) / 2;
  float2 drho = f[0], jx = bc2(0.f), jy = bc2(0.f), jz = bc2(0.f);
  float2 sxx = bc2(0.f), syy = bc2(0.f), szz = bc2(0.f), sxy = bc2(0.f), sxz = bc2(0.f), syz = bc2(0.f);
#pragma unroll
  for (int k = 0; k < NP; ++k) {
    const int a = 2 * k + 1, b = a + 1;
    const int cx = L::cx(a), cy = L::cy(a), cz = L::cz(a);
    const float2 S = add2(f[a], f[b]), D = sub2(f[a], f[b]);
    drho = add2(drho, S);
    if (cx == 1) jx = add2(jx, D);
    if (cx == -1) jx = sub2(jx, D);
    if (cy == 1) jy = add2(jy, D);
    if (cy == -1) jy = sub2(jy, D);
    if (cz == 1) jz = add2(jz, D);
    if (cz == -1) jz = sub2(jz, D);
    if (cx) sxx = add2(sxx, S);
    if (cy) syy = add2(syy, S);
    if (cz) szz = add2(szz, S);
    if (cx && cy) sxy = cx * cy > 0 ? add2(sxy, S) : sub2(sxy, S);
    if (cx && cz) sxz = cx * cz > 0 ? add2(sxz, S) : sub2(sxz, S);
    if (cy && cz) syz = cy * cz > 0 ? add2(syz, S) : sub2(syz, S);
  }
  const float2 rho = add2(drho, bc2(1.f));
  const float2 inv = make_float2(rcp_fast(rho.x), rcp_fast(rho.y));
  const float2 ux = mul2(jx, inv), uy = mul2(jy, inv), uz = mul2(jz, inv);
  // exact rest (per lane)
  bool rest0 = ux.x == 0.f && uy.x == 0.f && uz.x == 0.f;
  bool rest1 = ux.y == 0.f && uy.y == 0.f && uz.y == 0.f;
  if (rest0 || rest1) {
#pragma unroll
    for (int q = 0; q < Q; ++q) {
      rest0 = rest0 && (f[q].x == float(L::w(q) * (double(rho.x) - 1.0)));
      rest1 = rest1 && (f[q].y == float(L::w(q) * (double(rho.y) - 1.0)));
    }
    if (rest0 && rest1) return rho;
  }
  const float2 d3 = mul2(drho, bc2(1.f / 3.f));
  const float2 pxx = sub2(sub2(sxx, d3), mul2(mul2(rho, ux), ux));
  const float2 pyy = sub2(sub2(syy, d3), mul2(mul2(rho, uy), uy));
  const float2 pzz = sub2(sub2(szz, d3), mul2(mul2(rho, uz), uz));
  const float2 pxy = sub2(sxy, mul2(mul2(rho, ux), uy));
  const float2 pxz = sub2(sxz, mul2(mul2(rho, ux), uz));
  const float2 pyz = sub2(syz, mul2(mul2(rho, uy), uz));
  const float2 usq = fma2(ux, ux, fma2(uy, uy, mul2(uz, uz)));
  float2 os = bc2(p.omega_shear);
  if (p.les_c > 0.f) {
    const float2 q2 = fma2(pxx, pxx, fma2(pyy, pyy, mul2(pzz, pzz)));
    const float2 o2 = fma2(pxy, pxy, fma2(pxz, pxz, mul2(pyz, pyz)));
    const float2 n2 = fma2(bc2(2.f), o2, q2);
    const float t0 = p.tau0;
    const float te0 = 0.5f * (t0 + sqrt_fast(t0 * t0 + p.les_c * sqrt_fast(n2.x) * inv.x));
    const float te1 = 0.5f * (t0 + sqrt_fast(t0 * t0 + p.les_c * sqrt_fast(n2.y) * inv.y));
    os = make_float2(rcp_fast(te0), rcp_fast(te1));
  }
  const float2 osc = fma2(os, mul2(usq, bc2(-0.16f)), os);
  const float2 keep = sub2(bc2(1.f), make_float2(fminf(osc.x, 2.f), fminf(osc.y, 2.f)));
  const float2 bulk = mul2(add2(add2(pxx, pyy), pzz), bc2(1.f / 3.f));
  const float2 k200 = mul2(keep, sub2(pxx, bulk)), k020 = mul2(keep, sub2(pyy, bulk));
  const float2 k002 = mul2(keep, sub2(pzz, bulk));
  const float2 k110 = mul2(keep, pxy), k101 = mul2(keep, pxz), k011 = mul2(keep, pyz);
  // x pass: G[a][b][c], a = c_x + 1, on the six order-2 lines (b, c)
  const float2 ux2 = mul2(ux, ux);
  const float2 s0m = mul2(bc2(0.5f), sub2(ux2, ux)), s0p = mul2(bc2(0.5f), add2(ux2, ux));
  const float2 s00 = sub2(bc2(1.f), ux2);
  const float2 s1m = sub2(ux, bc2(0.5f)), s1p = add2(ux, bc2(0.5f));
  const float2 s10 = mul2(ux, bc2(-2.f));
  float2 G[3][3][3];
  auto line0 = [&](int b, int c, float2 k) {  // order 0 along x
    G[0][b][c] = mul2(s0m, k);
    G[1][b][c] = mul2(s00, k);
    G[2][b][c] = mul2(s0p, k);
  };
  auto line1 = [&](int b, int c, float2 k) {  // order 1 along x
    G[0][b][c] = mul2(s1m, k);
    G[1][b][c] = mul2(s10, k);
    G[2][b][c] = mul2(s1p, k);
  };
  G[0][0][0] = mul2(bc2(0.5f), k200);  // order 2 along x
  G[1][0][0] = mul2(bc2(-1.f), k200);
  G[2][0][0] = G[0][0][0];
  line0(2, 0, k020);
  line0(0, 2, k002);
  line0(1, 1, k011);
  line1(1, 0, k110);
  line1(0, 1, k101);
  // y pass over b for each (a, c): c = 0 full, c = 1 without order 2,
  // c = 2 order 0 only
  const float2 uy2 = mul2(uy, uy);
  const float2 t0m = mul2(bc2(0.5f), sub2(uy2, uy)), t0p = mul2(bc2(0.5f), add2(uy2, uy));
  const float2 t00 = sub2(bc2(1.f), uy2);
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    cm_bwd2(G[a][0][0], G[a][1][0], G[a][2][0], uy);
    {
      const float2 k0 = G[a][0][1], k1 = G[a][1][1];
      const float2 m1 = fma2(uy, k0, k1);
      const float2 m2 = mul2(uy, fma2(uy, k0, mul2(bc2(2.f), k1)));
      G[a][0][1] = mul2(bc2(0.5f), sub2(m2, m1));
      G[a][1][1] = sub2(k0, m2);
      G[a][2][1] = mul2(bc2(0.5f), add2(m2, m1));
    }
    {
      const float2 k0 = G[a][0][2];
      G[a][0][2] = mul2(t0m, k0);
      G[a][1][2] = mul2(t00, k0);
      G[a][2][2] = mul2(t0p, k0);
    }
  }
  // z pass over c for each (a, b)
#pragma unroll
  for (int a = 0; a < 3; ++a)
#pragma unroll
    for (int b = 0; b < 3; ++b) cm_bwd2(G[a][b][0], G[a][b][1], G[a][b][2], uz);
  // f' = feq + G: w (drho + rho (3 cu + 4.5 cu^2 - 1.5 u^2))
  const float2 nusq = mul2(bc2(-1.5f), usq);
#pragma unroll
  for (int q = 0; q < Q; ++q) {
    float2 cu = L::cx(q) ? (L::cx(q) > 0 ? ux : mul2(ux, bc2(-1.f))) : bc2(0.f);
    if (L::cy(q)) cu = L::cy(q) > 0 ? add2(cu, uy) : sub2(cu, uy);
    if (L::cz(q)) cu = L::cz(q) > 0 ? add2(cu, uz) : sub2(cu, uz);
    const float2 inner = fma2(cu, fma2(bc2(4.5f), cu, bc2(3.f)), nusq);
    const float2 v = fma2(bc2(float(L::w(q))), fma2(rho, inner, drho), G[L::cx(q) + 1][L::cy(q) + 1][L::cz(q) + 1]);
    f[q].x = rest0 ? f[q].x : v.x;
    f[q].y = rest1 ? f[q].y : v.y;
  }
  return rho;
}

// Collision of a pair in the chosen form.
template <int Q, int COLL>
__device__ __forceinline__ float2 pair_collide(float2 (&f)[Q], const HydroParams<float>& p) {
  if constexpr (COLL == COLL_CM) return cm_pair_reg<Q>(f, p);
  else return trt_pair_lean<Q>(f, p);
}

// The two elements at e and e + 1 of a 16-bit array where e is odd: the two
// aligned 4-byte words that hold them, merged (neighbouring threads load the
// same words, so the second load hits L1).
template <class S>
__device__ __forceinline__ float2 ld2_odd(const S* p) {
  if constexpr (sizeof(S) == 2) {
    const uint32_t* w = reinterpret_cast<const uint32_t*>(p - 1);
    uint32_t v = __byte_perm(w[0], w[1], 0x5432);
    if constexpr (std::is_same<S, __half>::value) return __half22float2(*reinterpret_cast<__half2*>(&v));
    else return __bfloat1622float2(*reinterpret_cast<__nv_bfloat162*>(&v));
  } else {
    return make_float2(PairIO<S>::ld1(p), PairIO<S>::ld1(p + 1));
  }
}

// Pair sweep: two x-adjacent cells per thread, one warp per 64-cell tile of
// a compacted list (tiles with a non-solid cell), direct accesses of at
// least 4 bytes wherever the pair is aligned (TRT / BGK, or the central
// moment on D3Q27; fp32 | fp16 | bf16 storage). With 2-byte storage, warps
// of one-element accesses reach about 0.73 of the copy bandwidth even
// without arithmetic, 4-byte pair accesses reach the copy bandwidth, and
// the packed collisions (trt_pair_lean, cm_pair_reg) halve the arithmetic
// instructions.
//   even step: own slots, aligned pair loads and stores for every direction;
//   odd step:  slot opp(q) of x - c_q and slot q of x + c_q; directions with
//              c_x = 0 stay aligned, the others read the two aligned words
//              around the pair and store two elements.
// The population loads are issued together with the flag load (every
// address is inside the allocation whatever the flags say), so a tile costs
// one memory round trip. A warp of 32 active pairs (and, on the odd step,
// no wall cell) takes straight pair accesses (warp-uniform vote). The other
// warps make every access per element and unconditionally, with the
// address selected per cell and link instead of a predicated access (a
// conditional load or store per link costs more than the access itself):
//   odd-step loads: a link whose upstream cell is solid reads the cell's
//     own slot (bounce-back); the tile list marks the tiles holding such
//     cells (TILE_BND), and the warp loads their solid-neighbour masks one
//     tile ahead, so the selection needs no extra round trip;
//   stores: a link whose downstream cell is solid writes the cell's own
//     slot (odd step), and an inactive cell of the pair (solid, or IBM-forced
//     and updated by hydro_cells_kernel) writes its own word of the scratch
//     plane Q, which nothing reads.
// Cells on a periodic face, under the free-slip top or next to a moving
// wall take the generic path.
constexpr int PAIR_TILE = 64;
constexpr uint32_t TILE_BND = 0x80000000u;  // tile-list bit: a fluid cell of the tile has a solid neighbour

// Per-tile addressing of a lane's pair: element offsets from the pair's
// first cell (own slot k, and slot k of the neighbour x + c_k; uniform across
// the grid).
template <int Q>
struct PairAddr {
  int nx, nxy;
  int64_t pl;
  __device__ __forceinline__ int32_t P(int k) const { return int32_t(int64_t(k) * pl); }
  __device__ __forceinline__ int32_t T(int k) const {
    using L = Lat<Q>;
    return int32_t(int64_t(k) * pl + (L::cx(k) + L::cy(k) * nx + L::cz(k) * nxy));
  }
};

// Source of link q for element e of the lane's pair on a wall tile of the
// odd step: the own slot when the upstream cell is solid, else the
// neighbour's slot.
template <int Q>
__device__ __forceinline__ int32_t pair_src(const PairAddr<Q>& A, uint32_t mk, int q) {
  const int o = opp(q);
  return ((mk >> o) & 1u) ? A.P(q) : A.T(o);
}

// The lane's populations straight from global memory (see the access
// rules above).
template <int Q, class S, bool ODD>
__device__ __forceinline__ void pair_load(const PairAddr<Q>& A, const S* cb, bool bnd_tile, uint32_t mk0,
                                          uint32_t mk1, float2 (&f)[Q]) {
  using L = Lat<Q>;
  using IO = PairIO<S>;
  if (ODD && bnd_tile) {
#pragma unroll
    for (int q = 0; q < Q; ++q) f[q] = make_float2(IO::ld1(cb + pair_src(A, mk0, q)), IO::ld1(cb + pair_src(A, mk1, q) + 1));
  } else {
#pragma unroll
    for (int q = 0; q < Q; ++q) {
      if (!ODD) {
        f[q] = IO::ld2(cb + A.P(q));
      } else {
        const S* src = cb + A.T(opp(q));
        f[q] = (L::cx(q) & 1) ? ld2_odd(src) : IO::ld2(src);
      }
    }
  }
}

__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }

template <int N>
__device__ __forceinline__ void cp_async_wait() {
  asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory");
}

__device__ __forceinline__ void cp_async4(uint32_t dst, const void* src) {
  asm volatile("cp.async.ca.shared.global [%0], [%1], 4;" ::"r"(dst), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_async8(uint32_t dst, const void* src) {
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" ::"r"(dst), "l"(src) : "memory");
}

// Staged form of pair_load: the same bytes copied by cp.async into the
// lane's staging slots (one 8-byte slot per link, slot q at byte offset
// q * 256 + 8 * lane of the stage, so a warp's reads of one link are
// conflict-free), then read back by pair_unstage once the copies landed.
// A slot holds the pair (fp32: 8 bytes; 16-bit: the low 4 bytes), or the two
// 4-byte pieces the pair is made of: two fp32 elements, or the two aligned
// 16-bit words around an odd-offset pair or around each element of a wall
// link.
template <int Q, class S, bool ODD>
__device__ __forceinline__ void pair_stage(const PairAddr<Q>& A, const S* cb, bool bnd_tile, uint32_t mk0,
                                           uint32_t mk1, uint32_t slots) {
  using L = Lat<Q>;
  constexpr bool W16 = sizeof(S) == 2;
#pragma unroll
  for (int q = 0; q < Q; ++q) {
    const uint32_t d = slots + uint32_t(q) * 256u;
    if (ODD && bnd_tile) {
      const S* s0 = cb + pair_src(A, mk0, q);
      const S* s1 = cb + pair_src(A, mk1, q) + 1;
      if (W16) {  // the aligned words holding each element
        s0 = reinterpret_cast<const S*>(reinterpret_cast<uintptr_t>(s0) & ~uintptr_t(3));
        s1 = reinterpret_cast<const S*>(reinterpret_cast<uintptr_t>(s1) & ~uintptr_t(3));
      }
      cp_async4(d, s0);
      cp_async4(d + 4u, s1);
    } else if (!ODD || !(L::cx(q) & 1)) {
      const S* src = cb + (ODD ? A.T(opp(q)) : A.P(q));
      if (W16) cp_async4(d, src);
      else cp_async8(d, src);
    } else {  // odd step, c_x odd: the pair starts at an odd element
      const S* src = cb + A.T(opp(q));
      if (W16) {
        cp_async4(d, src - 1);
        cp_async4(d + 4u, src + 1);
      } else {
        cp_async4(d, src);
        cp_async4(d + 4u, src + 1);
      }
    }
  }
}

template <class S>
__device__ __forceinline__ float2 h2f2(uint32_t v) {
  if constexpr (std::is_same<S, __half>::value) return __half22float2(*reinterpret_cast<__half2*>(&v));
  else return __bfloat1622float2(*reinterpret_cast<__nv_bfloat162*>(&v));
}

template <int Q, class S, bool ODD>
__device__ __forceinline__ void pair_unstage(const PairAddr<Q>& A, bool bnd_tile, uint32_t mk0, uint32_t mk1,
                                             const uint2* slots, float2 (&f)[Q]) {
  using L = Lat<Q>;
#pragma unroll
  for (int q = 0; q < Q; ++q) {
    const uint2 v = slots[q * 32];
    if constexpr (sizeof(S) == 4) {
      f[q] = make_float2(__uint_as_float(v.x), __uint_as_float(v.y));
    } else if (ODD && bnd_tile) {
      // element 0 sits in the high half of its word when its offset is odd
      // (c is even; own slots are even, neighbour slots odd when c_x is)
      const int o = opp(q);
      const bool odd0 = !((mk0 >> o) & 1u) && (L::cx(o) & 1);
      const bool odd1 = ((mk1 >> o) & 1u) || !(L::cx(o) & 1);
      const uint32_t h = __byte_perm(v.x, v.y, (odd0 ? 0x32u : 0x10u) | (odd1 ? 0x7600u : 0x5400u));
      f[q] = h2f2<S>(h);
    } else if (!ODD || !(L::cx(q) & 1)) {
      f[q] = h2f2<S>(v.x);
    } else {
      f[q] = h2f2<S>(__byte_perm(v.x, v.y, 0x5432));
    }
  }
}

// The rest of a lane's tile once its populations are in registers: flags
// (fl2: the pair's two flag bytes), generic cells, collision, stores.
template <int Q, class S, bool ODD, int COLL>
__device__ __forceinline__ void pair_finish(const HydroParams<float>& p, const PairAddr<Q>& A, S* cb, uint32_t c,
                                            bool bnd_tile, uint32_t mk0, uint32_t mk1, uint32_t fl2,
                                            float2 (&f)[Q]) {
  using L = Lat<Q>;
  using IO = PairIO<S>;
  const uint32_t fl0 = fl2 & 0xffu, fl1 = fl2 >> 8;
  const bool act0 = !(fl0 & (F_SOLID | F_FORCED)), act1 = !(fl1 & (F_SOLID | F_FORCED));
  if (!(act0 || act1)) return;
  if ((fl0 | fl1) & (F_WRAP | F_SLIP | F_MOVING)) {
    const int nx = A.nx, nxy = A.nxy;
    const int z = int(c / uint32_t(nxy));
    const int r = int(c - uint32_t(z) * uint32_t(nxy));
    const int y = r / nx, x = r - y * nx;
    if (act0) hydro_cell_generic<Q, S, COLL, ODD, false>(p, x, y, z, c, uint8_t(fl0));
    if (act1) hydro_cell_generic<Q, S, COLL, ODD, false>(p, x + 1, y, z, c + 1, uint8_t(fl1));
    return;
  }
  const bool straight = __all_sync(__activemask(), act0 && act1) && !bnd_tile;
  pair_collide<Q, COLL>(f, p);
  // a fresh copy of the base pointer keeps the compiler from holding the
  // load addresses (the same offsets on the even step) live across the
  // collision
  asm volatile("" : "+l"(cb));
  if (straight) {
#pragma unroll
    for (int q = 0; q < Q; ++q) {
      if (!ODD) {
        IO::st2(cb + A.P(opp(q)), f[q]);
      } else if (L::cx(q) & 1) {
        IO::st1(cb + A.T(q), f[q].x);
        IO::st1(cb + A.T(q) + 1, f[q].y);
      } else {
        IO::st2(cb + A.T(q), f[q]);
      }
    }
    return;
  }
  const int32_t scratch = A.P(Q);
#pragma unroll
  for (int q = 0; q < Q; ++q) {
    const int o = opp(q);
    int32_t d0 = A.P(o), d1 = A.P(o);
    if (ODD) {
      d0 = ((mk0 >> q) & 1u) ? A.P(o) : A.T(q);
      d1 = ((mk1 >> q) & 1u) ? A.P(o) : A.T(q);
    }
    IO::st1(cb + (act0 ? d0 : scratch), f[q].x);
    IO::st1(cb + (act1 ? d1 : scratch) + 1, f[q].y);
  }
}

// The flag bytes of the lane's pair (both solid past the grid's end).
__device__ __forceinline__ uint32_t pair_flags(const HydroParams<float>& p, uint32_t c, uint32_t ncells) {
  return c < ncells ? uint32_t(reinterpret_cast<const uint16_t*>(p.flags)[c >> 1])
                    : uint32_t(F_SOLID | (F_SOLID << 8));
}

// Warps walk the tile list with a grid stride (persistent: a runner step
// sizes the grid to leave block slots free for the IBM chain on the side
// stream), the tile entries ahead of the tile in hand and, on the odd step
// of TILE_BND tiles, the solid-neighbour masks ahead of the populations.
//   STAGED = false: the populations of a tile are loaded when the warp
//     reaches it (entries two tiles ahead, masks one tile ahead);
//   STAGED = true: they are copied by cp.async into the warp's staging
//     slots one tile ahead (two stages of Q x 32 slots of 8 bytes per warp,
//     dynamic shared memory), so their latency overlaps the collision of
//     the tile in hand (entries three tiles ahead, masks two, flags one).
template <int Q, class S, bool ODD, int MINB, int COLL, bool STAGED = false>
__global__ void __launch_bounds__(PAIR_BLOCK, MINB)
    hydro_pair_kernel(HydroParams<float> p, const uint32_t* tiles, int ntiles, uint32_t ncells) {
  const int nwarps = int(gridDim.x) * (PAIR_BLOCK / 32);
  const uint32_t lane = threadIdx.x & 31u;
  const uint32_t lane2 = 2u * lane;
  int w = int((blockIdx.x * PAIR_BLOCK + threadIdx.x) >> 5);
  const PairAddr<Q> A{p.nx, p.nxy, int64_t(p.plane)};
  S* const fb = static_cast<S*>(p.f);
  auto cell0 = [&](uint32_t e) { return (e & ~TILE_BND) * PAIR_TILE + lane2; };
  // the masks of the lane's two cells (c is even, so the pair is one
  // aligned 8-byte word of the mask array)
  auto masks = [&](uint32_t e) {
    uint2 m = make_uint2(0u, 0u);
    if (ODD && (e & TILE_BND)) {
      const uint32_t c = cell0(e);
      if (c < ncells) m = __ldg(reinterpret_cast<const uint2*>(p.nbr) + (c >> 1));
    }
    return m;
  };
  auto entry = [&](int k) { return k < ntiles ? __ldg(tiles + k) : 0u; };
  if constexpr (!STAGED) {
    uint32_t e0 = entry(w);
    uint32_t e1 = entry(w + nwarps);
    uint2 m0 = masks(e0);
    for (; w < ntiles; w += nwarps) {
      const uint32_t e2 = entry(w + 2 * nwarps);
      const uint2 m1 = masks(e1);  // e1 = 0 past the end: no load
      const uint32_t c = cell0(e0);
      S* cb = fb + c;
      const bool bnd = ODD && (e0 & TILE_BND);  // warp-uniform
      float2 f[Q];
      pair_load<Q, S, ODD>(A, cb, bnd, m0.x, m0.y, f);
      pair_finish<Q, S, ODD, COLL>(p, A, cb, c, bnd, m0.x, m0.y, pair_flags(p, c, ncells), f);
      e0 = e1;
      e1 = e2;
      m0 = m1;
    }
  } else {
    extern __shared__ uint2 pair_slots_smem[];
    uint2* const wslots = pair_slots_smem + size_t(threadIdx.x >> 5) * (2 * Q * 32) + lane;
    const uint32_t wsh = static_cast<uint32_t>(__cvta_generic_to_shared(wslots));
    auto stage = [&](uint32_t e, uint2 m, int buf) {
      const uint32_t c = cell0(e);
      pair_stage<Q, S, ODD>(A, fb + c, ODD && (e & TILE_BND), m.x, m.y, wsh + uint32_t(buf) * (Q * 256u));
    };
    uint32_t e0 = entry(w);
    uint32_t e1 = entry(w + nwarps);
    uint32_t e2 = entry(w + 2 * nwarps);
    uint2 m0 = masks(e0);
    if (w < ntiles) stage(e0, m0, 0);
    cp_async_commit();
    uint32_t fl0 = pair_flags(p, cell0(e0), ncells);
    uint2 m1 = masks(e1);
    int buf = 0;
    for (; w < ntiles; w += nwarps) {
      const uint32_t e3 = entry(w + 3 * nwarps);
      const bool more = w + nwarps < ntiles;
      if (more) stage(e1, m1, buf ^ 1);
      cp_async_commit();
      const uint2 m2 = masks(e2);
      const uint32_t fl1 = more ? pair_flags(p, cell0(e1), ncells) : 0u;
      cp_async_wait<1>();  // this tile's copies (only the lane's own slots are read)
      const uint32_t c = cell0(e0);
      S* cb = fb + c;
      const bool bnd = ODD && (e0 & TILE_BND);
      float2 f[Q];
      pair_unstage<Q, S, ODD>(A, bnd, m0.x, m0.y, wslots + size_t(buf) * (Q * 32), f);
      pair_finish<Q, S, ODD, COLL>(p, A, cb, c, bnd, m0.x, m0.y, fl0, f);
      e0 = e1;
      e1 = e2;
      e2 = e3;
      m0 = m1;
      m1 = m2;
      fl0 = fl1;
      buf ^= 1;
    }
    cp_async_wait<0>();
  }
}

template <int Q>
constexpr size_t pair_staged_smem_bytes() {
  return size_t(PAIR_BLOCK / 32) * 2 * Q * 32 * sizeof(uint2);
}

}  // namespace lbmb
