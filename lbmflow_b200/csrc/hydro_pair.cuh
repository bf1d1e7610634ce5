// Two cells per thread AA collide-stream with packed fp32x2 arithmetic
// (TRT / BGK, no uniform body force, fp32 | fp16 | bf16 storage).
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

// TRT collision of two cells held in float2 lanes; returns rho (for the
// moving-wall term).
template <int Q>
__device__ __forceinline__ float2 trt_pair_collide(float2 (&f)[Q], const HydroParams<float>& p) {
  using L = Lat<Q>;
  constexpr int NP = (Q - 1) / 2;
  static_assert(pair_heads_positive<Q>(), "pair head convention");
  float2 S[NP], D[NP];
#pragma unroll
  for (int k = 0; k < NP; ++k) {
    S[k] = add2(f[2 * k + 1], f[2 * k + 2]);
    D[k] = sub2(f[2 * k + 1], f[2 * k + 2]);
  }
  float2 drho = add2(f[0], S[0]);
#pragma unroll
  for (int k = 1; k < NP; ++k) drho = add2(drho, S[k]);
  // pairs 0, 1, 2 are the +x, +y, +z axis links
  float2 jx = D[0], jy = D[1], jz = D[2];
#pragma unroll
  for (int k = 3; k < NP; ++k) {
    const int a = 2 * k + 1;
    if (L::cx(a) == 1) jx = add2(jx, D[k]);
    if (L::cx(a) == -1) jx = sub2(jx, D[k]);
    if (L::cy(a) == 1) jy = add2(jy, D[k]);
    if (L::cy(a) == -1) jy = sub2(jy, D[k]);
    if (L::cz(a) == 1) jz = add2(jz, D[k]);
    if (L::cz(a) == -1) jz = sub2(jz, D[k]);
  }
  const float2 rho = add2(drho, bc2(1.f));
  const float2 inv = make_float2(rcp_fast(rho.x), rcp_fast(rho.y));
  const float2 ux = mul2(jx, inv), uy = mul2(jy, inv), uz = mul2(jz, inv);
  const float2 usq = fma2(ux, ux, fma2(uy, uy, mul2(uz, uz)));
  float2 op = bc2(p.omega_p), om = bc2(p.omega_m);
  if (p.les_c > 0.f) {
    float s[2][6];
#pragma unroll
    for (int h = 0; h < 2; ++h)
#pragma unroll
      for (int i = 0; i < 6; ++i) s[h][i] = 0.f;
#pragma unroll
    for (int k = 0; k < NP; ++k) {
      const int a = 2 * k + 1;
      const int cx = L::cx(a), cy = L::cy(a), cz = L::cz(a);
      const float sv[2] = {S[k].x, S[k].y};
#pragma unroll
      for (int h = 0; h < 2; ++h) {
        if (cx) s[h][0] += sv[h];
        if (cy) s[h][1] += sv[h];
        if (cz) s[h][2] += sv[h];
        if (cx && cy) s[h][3] += float(cx * cy) * sv[h];
        if (cx && cz) s[h][4] += float(cx * cz) * sv[h];
        if (cy && cz) s[h][5] += float(cy * cz) * sv[h];
      }
    }
    const float te0 = les_tau_pair<Q>(s[0], rho.x, inv.x, ux.x, uy.x, uz.x, p.les_c, p.tau0);
    const float te1 = les_tau_pair<Q>(s[1], rho.y, inv.y, ux.y, uy.y, uz.y, p.les_c, p.tau0);
    op = make_float2(rcp_fast(te0), rcp_fast(te1));
    // omega- = 1 / (magic / (tau - 1/2) + 1/2) = (tau - 1/2) / (magic + (tau - 1/2) / 2)
    if (p.magic > 0.f) {
      const float l0 = te0 - 0.5f, l1 = te1 - 0.5f;
      om = make_float2(l0 * rcp_fast(p.magic + 0.5f * l0), l1 * rcp_fast(p.magic + 0.5f * l1));
    } else {
      om = op;
    }
  }
  // base = drho - 1.5 rho u^2 (feq of the rest population is w0 * base)
  const float2 base = fma2(mul2(rho, bc2(-1.5f)), usq, drho);
  const float2 nhop = mul2(op, bc2(-0.5f)), hom = mul2(om, bc2(0.5f));
  float2 oA[3], oB[3], nC[3];
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    const int a = k == 0 ? 1 : (k == 1 ? 7 : 19);
    if (a >= Q) continue;
    const float w = float(L::w(a));
    oA[k] = mul2(mul2(op, bc2(w)), base);
    oB[k] = mul2(mul2(op, bc2(4.5f * w)), rho);
    nC[k] = mul2(mul2(om, bc2(-3.f * w)), rho);
  }
  f[0] = fma2(sub2(bc2(1.f), op), f[0], mul2(mul2(op, bc2(float(L::w(0)))), base));
#pragma unroll
  for (int k = 0; k < NP; ++k) {
    const int a = 2 * k + 1, b = a + 1;
    const int cl = wclass<Q>(a);
    float2 cu = L::cx(a) ? ux : (L::cy(a) ? uy : uz);
    if (L::cx(a) && L::cy(a)) cu = L::cy(a) > 0 ? add2(cu, uy) : sub2(cu, uy);
    if ((L::cx(a) || L::cy(a)) && L::cz(a)) cu = L::cz(a) > 0 ? add2(cu, uz) : sub2(cu, uz);
    const float2 t = fma2(oB[cl], mul2(cu, cu), oA[cl]);
    const float2 pn = fma2(nhop, S[k], t);            // -rp
    const float2 m = fma2(nC[cl], cu, mul2(hom, D[k]));  // rm
    f[a] = sub2(add2(f[a], pn), m);
    f[b] = add2(add2(f[b], pn), m);
  }
  return rho;
}

// Central-moment collision (kernels.rs:406-533, no force term) of two cells
// in float2 lanes, in the form that keeps one set of 27 values live:
//   K = f - feq;  K <- T K (factorised central-moment transform);
//   K <- (I - R) K  (order <= 1 kept, order-2 deviatoric at 1 - w_s, trace
//                    and order >= 3 to zero);
//   f' = feq + T^-1 K
// which is the same operator as f + T^-1[-R T(f - feq)] by linearity. The
// exact-rest skip (kernels.rs:434-447) zeroes K of a lane whose populations
// all equal w (rho - 1), so that lane comes back unchanged.
__device__ __forceinline__ void cm_fwd2(float2& a, float2& b, float2& c, float2 u) {
  const float2 k0 = add2(add2(a, b), c);
  const float2 d = sub2(c, a);
  const float2 s = add2(c, a);
  const float2 k1 = fma2(mul2(u, bc2(-1.f)), k0, d);
  const float2 k2 = fma2(mul2(u, u), k0, fma2(mul2(u, bc2(-2.f)), d, s));
  a = k0;
  b = k1;
  c = k2;
}
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

template <int Q>
__device__ __forceinline__ float2 cm_pair_collide(float2 (&f)[Q], const HydroParams<float>& p) {
  static_assert(Q == 27, "central moments need the full D3Q27 tensor basis");
  using L = Lat<Q>;
  constexpr int NP = (Q - 1) / 2;
  float2 drho = f[0], jx = bc2(0.f), jy = bc2(0.f), jz = bc2(0.f);
  float s6[2][6] = {{0.f, 0.f, 0.f, 0.f, 0.f, 0.f}, {0.f, 0.f, 0.f, 0.f, 0.f, 0.f}};
#pragma unroll
  for (int k = 0; k < NP; ++k) {
    const int a = 2 * k + 1, b = a + 1;
    const float2 S = add2(f[a], f[b]), D = sub2(f[a], f[b]);
    drho = add2(drho, S);
    if (L::cx(a) == 1) jx = add2(jx, D);
    if (L::cx(a) == -1) jx = sub2(jx, D);
    if (L::cy(a) == 1) jy = add2(jy, D);
    if (L::cy(a) == -1) jy = sub2(jy, D);
    if (L::cz(a) == 1) jz = add2(jz, D);
    if (L::cz(a) == -1) jz = sub2(jz, D);
  }
  const float2 rho = add2(drho, bc2(1.f));
  const float2 inv = make_float2(rcp_fast(rho.x), rcp_fast(rho.y));
  const float2 ux = mul2(jx, inv), uy = mul2(jy, inv), uz = mul2(jz, inv);
  const float2 usq = fma2(ux, ux, fma2(uy, uy, mul2(uz, uz)));
  float2 os = bc2(p.omega_shear);
  if (p.les_c > 0.f) {
#pragma unroll
    for (int k = 0; k < NP; ++k) {
      const int a = 2 * k + 1;
      const int cx = L::cx(a), cy = L::cy(a), cz = L::cz(a);
      const float2 S = add2(f[a], f[a + 1]);
      const float sv[2] = {S.x, S.y};
#pragma unroll
      for (int h = 0; h < 2; ++h) {
        if (cx) s6[h][0] += sv[h];
        if (cy) s6[h][1] += sv[h];
        if (cz) s6[h][2] += sv[h];
        if (cx && cy) s6[h][3] += float(cx * cy) * sv[h];
        if (cx && cz) s6[h][4] += float(cx * cz) * sv[h];
        if (cy && cz) s6[h][5] += float(cy * cz) * sv[h];
      }
    }
    const float te0 = les_tau_pair<Q>(s6[0], rho.x, inv.x, ux.x, uy.x, uz.x, p.les_c, p.tau0);
    const float te1 = les_tau_pair<Q>(s6[1], rho.y, inv.y, ux.y, uy.y, uz.y, p.les_c, p.tau0);
    os = make_float2(rcp_fast(te0), rcp_fast(te1));
  }
  // exact rest (per lane): u == 0 and every population == w (rho - 1)
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
  auto feq = [&](int q) {
    float2 cu = L::cx(q) ? (L::cx(q) > 0 ? ux : mul2(ux, bc2(-1.f))) : bc2(0.f);
    if (L::cy(q)) cu = L::cy(q) > 0 ? add2(cu, uy) : sub2(cu, uy);
    if (L::cz(q)) cu = L::cz(q) > 0 ? add2(cu, uz) : sub2(cu, uz);
    // w (drho + rho (3 cu + 4.5 cu^2 - 1.5 u^2))
    const float2 inner = fma2(cu, fma2(bc2(4.5f), cu, bc2(3.f)), mul2(bc2(-1.5f), usq));
    return mul2(bc2(float(L::w(q))), fma2(rho, inner, drho));
  };
  float2 K[3][3][3];
#pragma unroll
  for (int q = 0; q < Q; ++q) K[L::cx(q) + 1][L::cy(q) + 1][L::cz(q) + 1] = sub2(f[q], feq(q));
  if (rest0 || rest1) {
#pragma unroll
    for (int i = 0; i < 27; ++i) {
      float2& k = K[i / 9][(i / 3) % 3][i % 3];
      if (rest0) k.x = 0.f;
      if (rest1) k.y = 0.f;
    }
  }
#pragma unroll
  for (int i = 0; i < 3; ++i)
#pragma unroll
    for (int j = 0; j < 3; ++j) cm_fwd2(K[i][j][0], K[i][j][1], K[i][j][2], uz);
#pragma unroll
  for (int i = 0; i < 3; ++i)
#pragma unroll
    for (int k = 0; k < 3; ++k) cm_fwd2(K[i][0][k], K[i][1][k], K[i][2][k], uy);
#pragma unroll
  for (int j = 0; j < 3; ++j)
#pragma unroll
    for (int k = 0; k < 3; ++k) cm_fwd2(K[0][j][k], K[1][j][k], K[2][j][k], ux);
  // deviatoric rate w_s (1 - 0.16 |u|^2) capped at 2
  const float2 ws = make_float2(fminf(os.x * (1.f - 0.16f * usq.x), 2.f), fminf(os.y * (1.f - 0.16f * usq.y), 2.f));
  const float2 keep = sub2(bc2(1.f), ws);
  const float2 bulk = mul2(bc2(1.f / 3.f), add2(add2(K[2][0][0], K[0][2][0]), K[0][0][2]));
#pragma unroll
  for (int a = 0; a < 3; ++a)
#pragma unroll
    for (int b = 0; b < 3; ++b)
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        const int order = a + b + c;
        const bool diag = order == 2 && (a == 2 || b == 2 || c == 2);
        if (order <= 1) continue;
        if (diag) K[a][b][c] = mul2(keep, sub2(K[a][b][c], bulk));
        else if (order == 2) K[a][b][c] = mul2(keep, K[a][b][c]);
        else K[a][b][c] = bc2(0.f);
      }
#pragma unroll
  for (int j = 0; j < 3; ++j)
#pragma unroll
    for (int k = 0; k < 3; ++k) cm_bwd2(K[0][j][k], K[1][j][k], K[2][j][k], ux);
#pragma unroll
  for (int i = 0; i < 3; ++i)
#pragma unroll
    for (int k = 0; k < 3; ++k) cm_bwd2(K[i][0][k], K[i][1][k], K[i][2][k], uy);
#pragma unroll
  for (int i = 0; i < 3; ++i)
#pragma unroll
    for (int j = 0; j < 3; ++j) cm_bwd2(K[i][j][0], K[i][j][1], K[i][j][2], uz);
#pragma unroll
  for (int q = 0; q < Q; ++q) {
    const float2 v = add2(feq(q), K[L::cx(q) + 1][L::cy(q) + 1][L::cz(q) + 1]);
    // a lane at exact rest keeps its populations bit for bit
    f[q].x = rest0 ? f[q].x : v.x;
    f[q].y = rest1 ? f[q].y : v.y;
  }
  return rho;
}

// Collision of a pair in the chosen form.
template <int Q, int COLL>
__device__ __forceinline__ float2 pair_collide(float2 (&f)[Q], const HydroParams<float>& p) {
  if constexpr (COLL == COLL_CM) return cm_pair_collide<Q>(f, p);
  else return trt_pair_collide<Q>(f, p);
}

template <int Q, class S, bool ODD, int COLL = COLL_TRT>
__global__ void __launch_bounds__(PAIR_BLOCK, COLL == COLL_CM ? 2 : 4) hydro_pair_kernel(HydroParams<float> p, uint32_t npairs) {
  using L = Lat<Q>;
  using IO = PairIO<S>;
  const uint32_t pi = blockIdx.x * PAIR_BLOCK + threadIdx.x;
  if (pi >= npairs) return;
  const uint32_t c = 2 * pi;
  const uint32_t fl2 = reinterpret_cast<const uint16_t*>(p.flags)[pi];
  const uint32_t fl0 = fl2 & 0xffu, fl1 = fl2 >> 8;
  const bool act0 = !(fl0 & (F_SOLID | F_FORCED)), act1 = !(fl1 & (F_SOLID | F_FORCED));
  if (!(act0 || act1)) return;
  const int nx = p.nx, nxy = p.nxy;
  if ((fl0 | fl1) & (F_WRAP | F_SLIP)) {
    const int z = int(c / uint32_t(nxy));
    const int r = int(c - uint32_t(z) * uint32_t(nxy));
    const int y = r / nx, x = r - y * nx;
    if (act0) hydro_cell_generic<Q, S, COLL, ODD, false>(p, x, y, z, c, uint8_t(fl0));
    if (act1) hydro_cell_generic<Q, S, COLL, ODD, false>(p, x + 1, y, z, c + 1, uint8_t(fl1));
    return;
  }
  const uint32_t mk0 = (fl0 & F_BOUNDARY) ? p.nbr[c] : 0u;
  const uint32_t mk1 = (fl1 & F_BOUNDARY) ? p.nbr[c + 1] : 0u;
  const uint32_t mk = mk0 | mk1;
  S* fb = static_cast<S*>(p.f);
  const uint32_t pl = p.plane;
  auto dq = [&](int q) { return L::cx(q) + L::cy(q) * nx + L::cz(q) * nxy; };
  float2 f[Q];
#pragma unroll
  for (int q = 0; q < Q; ++q) {
    if (!ODD) {
      f[q] = IO::ld2(fb + (uint32_t(q) * pl + c));
    } else {
      const int o = opp(q);
      // the neighbour window is always inside the allocation; a direction
      // that bounces off a solid neighbour is then re-read from the own slot
      const S* src = fb + int32_t(uint32_t(o) * pl + c - uint32_t(dq(q)));
      if (L::cx(q) & 1) f[q] = make_float2(IO::ld1(src), IO::ld1(src + 1));
      else f[q] = IO::ld2(src);
      const S* own = fb + (uint32_t(q) * pl + c);
      if ((mk0 >> o) & 1u) f[q].x = IO::ld1(own);
      if ((mk1 >> o) & 1u) f[q].y = IO::ld1(own + 1);
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

}  // namespace lbmb
