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
#include "hydro_pair.cuh"

namespace lbmb {

// D3Q27 central-moment collision of one fp32 cell (no force) with the
// x-opposite populations (-1, j, k) and (+1, j, k) of the 3 x 3 x 3 tensor
// held together in a float2 (FP[j][k] = (f(-1, j-1, k-1), f(+1, j-1, k-1)),
// F1[j][k] = f(0, j-1, k-1)).
//
// The operator is the reference's (kernels.rs:406-533): with K = f - feq in
// central moments about u, the post-collision moments keep order 0 and 1,
// relax the order-2 deviatoric part at omega_s (1 - 0.16 |u|^2) capped at 2,
// and relax the order-2 trace and every higher moment at 1, i.e. set them
// to the equilibrium's. So f' = feq + T^-1 K' where K' holds only the five
// deviatoric order-2 moments (1 - omega_s) (K_ab - tr K / 3 delta_ab); the
// order-0/1 moments of f - feq are zero when u = j / rho (they are dropped
// here: round-off), and the order-2 central moments of f - feq then equal
// its raw ones, the non-equilibrium stress
//   Pi_ab = sum_q c_a c_b f_q - rho u_a u_b - (rho - 1) / 3 delta_ab
// (deviation form, second-order equilibrium). Only the backward transform
// runs, on that sparse K': the x pass maps each of the six order-2 lines to
// the three x velocities with fixed per-axis shape functions, then the y
// and z passes of the factorised transform, packed on the x-opposite pairs
// (FFMA2 / FADD2 / FMUL2). The subgrid rate comes from the same Pi.
__device__ __forceinline__ void collide_cm_x2(float2 (&FP)[3][3], float (&F1)[3][3], float rho, float ux, float uy,
                                              float uz, float omega_shear, float les_c, float tau0) {
  using L = Lat<27>;
  auto wgt = [](int nz) -> float {  // weight of a direction with nz nonzero components
    return nz == 0 ? float(L::w(0)) : (nz == 1 ? float(L::w(1)) : (nz == 2 ? float(L::w(7)) : float(L::w(19))));
  };
  const float drho = rho - 1.f;
  if (ux == 0.f && uy == 0.f && uz == 0.f) {
    // exact-rest skip (kernels.rs:434-447)
    bool exact = true;
#pragma unroll
    for (int j = 0; j < 3; ++j)
#pragma unroll
      for (int k = 0; k < 3; ++k) {
        const int nz = (j != 1) + (k != 1);
        const float e0 = float(double(wgt(nz)) * (double(rho) - 1.0));
        const float e1 = float(double(wgt(nz + 1)) * (double(rho) - 1.0));
        exact = exact && F1[j][k] == e0 && FP[j][k].x == e1 && FP[j][k].y == e1;
      }
    if (exact) return;
  }
  // second moments of the populations
  float sxx = 0.f, syy = 0.f, szz = 0.f, sxy = 0.f, sxz = 0.f, syz = 0.f;
#pragma unroll
  for (int j = 0; j < 3; ++j)
#pragma unroll
    for (int k = 0; k < 3; ++k) {
      const float sp = FP[j][k].x + FP[j][k].y;  // c_x = +-1
      const float dp = FP[j][k].y - FP[j][k].x;  // c_x f over the pair
      const float s3 = sp + F1[j][k];
      sxx += sp;
      if (j != 1) syy += s3;
      if (k != 1) szz += s3;
      if (j == 2) sxy += dp;
      if (j == 0) sxy -= dp;
      if (k == 2) sxz += dp;
      if (k == 0) sxz -= dp;
      if (j != 1 && k != 1) syz = (j == k) ? syz + s3 : syz - s3;
    }
  const float d3 = drho * (1.f / 3.f);
  const float pxx = (sxx - d3) - rho * ux * ux, pyy = (syy - d3) - rho * uy * uy, pzz = (szz - d3) - rho * uz * uz;
  const float pxy = sxy - rho * ux * uy, pxz = sxz - rho * ux * uz, pyz = syz - rho * uy * uz;
  const float usq = (ux * ux + uy * uy) + uz * uz;
  if (les_c > 0.f) {
    const float pn = fast_sqrt((pxx * pxx + pyy * pyy + pzz * pzz) + 2.f * (pxy * pxy + pxz * pxz + pyz * pyz));
    omega_shear = fast_rcp(0.5f * (tau0 + fast_sqrt(tau0 * tau0 + les_c * pn * fast_rcp(rho))));
  }
  const float os = fminf(omega_shear * (1.f + -0.16f * usq), 2.f);
  const float keep = 1.f - os;
  const float bulk = (pxx + pyy + pzz) * (1.f / 3.f);
  const float k200 = keep * (pxx - bulk), k020 = keep * (pyy - bulk), k002 = keep * (pzz - bulk);
  const float k110 = keep * pxy, k101 = keep * pxz, k011 = keep * pyz;
  // x pass: per-axis shape functions of order 0, 1, 2 at c = (-1, +1) and 0
  //   order 0: ((u^2 - u)/2, (u^2 + u)/2), 1 - u^2
  //   order 1: (u - 1/2, u + 1/2), -2u
  //   order 2: (1/2, 1/2), -1
  const float ux2 = ux * ux;
  const float2 s0 = make_float2(0.5f * (ux2 - ux), 0.5f * (ux2 + ux));
  const float m0 = 1.f - ux2;
  const float2 s1 = make_float2(ux - 0.5f, ux + 0.5f);
  const float m1 = -2.f * ux;
  // G[b][c]: the line (b, c) after the x pass, pair (c_x = -1, +1) and mid
  // (c_x = 0); lines (1, 2), (2, 1), (2, 2) are zero
  float2 GP[3][3];
  float G1[3][3];
  GP[0][0] = bc2(0.5f * k200);  G1[0][0] = -k200;            // (2, 0, 0)
  GP[2][0] = mul2(s0, bc2(k020)); G1[2][0] = m0 * k020;      // (0, 2, 0)
  GP[0][2] = mul2(s0, bc2(k002)); G1[0][2] = m0 * k002;      // (0, 0, 2)
  GP[1][1] = mul2(s0, bc2(k011)); G1[1][1] = m0 * k011;      // (0, 1, 1)
  GP[1][0] = mul2(s1, bc2(k110)); G1[1][0] = m1 * k110;      // (1, 1, 0)
  GP[0][1] = mul2(s1, bc2(k101)); G1[0][1] = m1 * k101;      // (1, 0, 1)
  const float2 uy2 = bc2(uy), uz2 = bc2(uz);
  // y pass over b for each c: c = 0 full, c = 1 without order 2, c = 2 order 0 only
  cm_bwd2(GP[0][0], GP[1][0], GP[2][0], uy2);
  cm_bwd(G1[0][0], G1[1][0], G1[2][0], uy);
  {
    // (k0, k1, 0): m1 = k1 + u k0, m2 = u (u k0 + 2 k1)
    const float2 k0 = GP[0][1], k1 = GP[1][1];
    const float2 p1 = fma2(uy2, k0, k1);
    const float2 p2 = mul2(uy2, fma2(uy2, k0, mul2(bc2(2.f), k1)));
    GP[0][1] = mul2(bc2(0.5f), sub2(p2, p1));
    GP[1][1] = sub2(k0, p2);
    GP[2][1] = mul2(bc2(0.5f), add2(p2, p1));
    const float q0 = G1[0][1], q1 = G1[1][1];
    const float r1 = q1 + uy * q0;
    const float r2 = uy * (uy * q0 + 2.f * q1);
    G1[0][1] = 0.5f * (r2 - r1);
    G1[1][1] = q0 - r2;
    G1[2][1] = 0.5f * (r2 + r1);
  }
  {
    const float uy_2 = uy * uy;
    const float t0 = 0.5f * (uy_2 - uy), t1 = 1.f - uy_2, t2 = 0.5f * (uy_2 + uy);
    const float2 k0 = GP[0][2];
    const float q0 = G1[0][2];
    GP[0][2] = mul2(bc2(t0), k0);
    GP[1][2] = mul2(bc2(t1), k0);
    GP[2][2] = mul2(bc2(t2), k0);
    G1[0][2] = t0 * q0;
    G1[1][2] = t1 * q0;
    G1[2][2] = t2 * q0;
  }
  // z pass over c for each b
#pragma unroll
  for (int j = 0; j < 3; ++j) {
    cm_bwd2(GP[j][0], GP[j][1], GP[j][2], uz2);
    cm_bwd(G1[j][0], G1[j][1], G1[j][2], uz);
  }
  // f' = feq + the transformed increment
  const float2 uxpm = make_float2(-ux, ux);
  const float2 drho2 = bc2(drho), rho2 = bc2(rho), nusq2 = bc2(-1.5f * usq);
#pragma unroll
  for (int j = 0; j < 3; ++j)
#pragma unroll
    for (int k = 0; k < 3; ++k) {
      const int nz = (j != 1) + (k != 1);
      const float v = float(j - 1) * uy + float(k - 1) * uz;
      const float inner1 = (3.f * v + (4.5f * v) * v) - 1.5f * usq;
      F1[j][k] = wgt(nz) * (drho + rho * inner1) + G1[j][k];
      const float2 cu = add2(bc2(v), uxpm);
      const float2 inner = fma2(cu, fma2(bc2(4.5f), cu, bc2(3.f)), nusq2);
      FP[j][k] = fma2(bc2(wgt(nz + 1)), fma2(rho2, inner, drho2), GP[j][k]);
    }
}

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
    if constexpr (COLL == COLL_CM && std::is_same<A, float>::value) {
      // packed central-moment path: populations straight into the
      // x-opposite pair layout
      float2 FP[3][3];
      float F1[3][3];
#pragma unroll
      for (int q = 0; q < Q; ++q) {
        const float v = CD::ld(src + q * ASYNC_TILE);
        const int jj = L::cy(q) + 1, kk = L::cz(q) + 1;
        if (L::cx(q) == 0) F1[jj][kk] = v;
        else if (L::cx(q) < 0) FP[jj][kk].x = v;
        else FP[jj][kk].y = v;
      }
      float dr = 0.f, m0 = 0.f, m1 = 0.f, m2 = 0.f;
#pragma unroll
      for (int jj = 0; jj < 3; ++jj)
#pragma unroll
        for (int kk = 0; kk < 3; ++kk) {
          const float s3 = (FP[jj][kk].x + F1[jj][kk]) + FP[jj][kk].y;
          dr += s3;
          m0 += FP[jj][kk].y - FP[jj][kk].x;
          if (jj == 2) m1 += s3;
          if (jj == 0) m1 -= s3;
          if (kk == 2) m2 += s3;
          if (kk == 0) m2 -= s3;
        }
      const float rho = 1.f + dr;
      const float inv = fast_rcp(rho);
      collide_cm_x2(FP, F1, rho, m0 * inv, m1 * inv, m2 * inv, p.omega_shear, p.les_c, p.tau0);
#pragma unroll
      for (int q = 0; q < Q; ++q) {
        const int jj = L::cy(q) + 1, kk = L::cz(q) + 1;
        f[q] = L::cx(q) == 0 ? F1[jj][kk] : (L::cx(q) < 0 ? FP[jj][kk].x : FP[jj][kk].y);
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
      continue;
    }
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
        cell_rates<Q, A, false, false>(p, f, rho, ux, uy, uz, op, om, cp, cm, os, cell);
      }
      collide_cm<Q, false, A, LK>(f, rho, ux, uy, uz, z0, z0, z0, os, p.les_c, p.tau0);
    } else {
      A op, om, cp, cm, os;
      cell_rates<Q, A, true, false>(p, f, rho, ux, uy, uz, op, om, cp, cm, os, cell);
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
