// Fused collide + stream in place (AA pattern), one thread per cell.
//
// Reference operator per step (crates/lbm-core/src/backend.rs:266-328):
// collide with the moments cached at the end of the previous step
// (kernels.rs:129-160 / 406-533), pull-stream with half-way bounce-back and
// the moving-wall term 6 w rho_dest (c . u_wall) (kernels.rs:547-622), then
// refresh the moments (kernels.rs:627-668). Here the cached moments are
// recomputed from the loaded populations (identical arithmetic), and the
// stream is a push into the in-place AA layout:
//
//   even step: read  slot q      of x            (normal layout)
//              write slot opp(q) of x            (swapped layout)
//   odd step:  read  slot opp(q) of x - c_q      (own slot q if x - c_q solid)
//              write slot q      of x + c_q      (own slot opp(q) if solid)
//
// Every location is read and then written by exactly one thread per step,
// so the update needs one population buffer and no barrier. A post-
// collision population aimed at a solid neighbour is written back bounced
// (plus the moving-wall term) into the slot the next step reads for the
// reflected direction, which is exactly the reference's bounce-back value.
//
// Cells are split by their flag byte into three code paths:
//   interior  (no solid neighbour, not on a periodic face): neighbour
//             offsets are compile-time combinations of 1, nx and nx*ny;
//   generic   (solid neighbours and/or periodic wrap): mask and wrap logic;
//   forced    (inside an IBM stencil): handled by hydro_cells_kernel over the
//             compact forced-cell list, after the IBM force update, unless a
//             uniform body force makes every cell forced.
// Element offsets q * plane + cell are 32-bit (checked on the host).
#pragma once
#include <type_traits>

#include "common.cuh"
#include "lattice.cuh"

namespace lbmb {

enum { COLL_TRT = 0, COLL_CM = 1 };

template <class A>
struct HydroParams {
  void* f;                // Q planes of the storage type
  uint32_t plane;         // elements per plane
  const uint8_t* flags;   // per cell
  const uint32_t* nbr;    // per cell: bit q set <=> x + c_q is solid
  const Vec4<A>* wall_u;  // per cell (meaningful on solids)
  const int32_t* fslot;   // per cell (forced cells): force slot
  const Vec4<A>* fprev;   // per slot: field inside the cached moments
  const Vec4<A>* fcur;    // per slot: current field (Guo source)
  int nx, ny, nz;
  int nxy;
  A omega_p, omega_m, cp, cm, omega_shear;
  A gx, gy, gz;  // uniform body force
  int uniform_force;
  A les_c;  // 18 sqrt(2) Cs^2 (0: no LES)
  A tau0;   // 3 nu + 1/2
  A magic;  // TRT magic parameter (<= 0: BGK, omega_m = omega_p)
};

// Smagorinsky LES on the shear rate (no reference counterpart; off unless
// les_c > 0). The non-equilibrium stress comes from the second moments of
// the deviation populations, Pi = sum c c f - (rho - 1)/3 I - rho u u
// (exact for the second-order equilibrium on D3Q19/D3Q27), and
// tau_eff = (tau0 + sqrt(tau0^2 + les_c |Pi| / rho)) / 2.
//
// FAST (fp32 only): single-instruction square roots and reciprocals (PTX
// .approx, a few ulp) instead of the IEEE-rounded forms, which cost a
// slow-path branch each; fp64 keeps the IEEE forms.
template <class A>
__device__ __forceinline__ A fast_rcp(A x) {
  if constexpr (std::is_same<A, float>::value) {
    float r;
    asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
    return r;
  } else {
    return A(1) / x;
  }
}
template <class A>
__device__ __forceinline__ A fast_sqrt(A x) {
  if constexpr (std::is_same<A, float>::value) {
    float r;
    asm("sqrt.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
    return r;
  } else {
    return sqrt(x);
  }
}

template <int Q, class A, bool FAST = false>
__device__ __forceinline__ A les_tau(const A (&f)[Q], A rho, A ux, A uy, A uz, A les_c, A tau0) {
  using L = Lat<Q>;
  A sxx = A(0), syy = A(0), szz = A(0), sxy = A(0), sxz = A(0), syz = A(0);
#pragma unroll
  for (int q = 1; q < Q; ++q) {
    const int cx = L::cx(q), cy = L::cy(q), cz = L::cz(q);
    if (cx) sxx = sxx + f[q];
    if (cy) syy = syy + f[q];
    if (cz) szz = szz + f[q];
    if (cx * cy == 1) sxy = sxy + f[q];
    if (cx * cy == -1) sxy = sxy - f[q];
    if (cx * cz == 1) sxz = sxz + f[q];
    if (cx * cz == -1) sxz = sxz - f[q];
    if (cy * cz == 1) syz = syz + f[q];
    if (cy * cz == -1) syz = syz - f[q];
  }
  const A d3 = (rho - A(1)) * A(1.0 / 3.0);
  const A pxx = sxx - d3 - rho * ux * ux, pyy = syy - d3 - rho * uy * uy, pzz = szz - d3 - rho * uz * uz;
  const A pxy = sxy - rho * ux * uy, pxz = sxz - rho * ux * uz, pyz = syz - rho * uy * uz;
  const A pn2 = (pxx * pxx + pyy * pyy + pzz * pzz) + A(2) * (pxy * pxy + pxz * pxz + pyz * pyz);
  if constexpr (FAST) {
    const A pn = fast_sqrt(pn2);
    return A(0.5) * (tau0 + fast_sqrt(tau0 * tau0 + les_c * pn * fast_rcp(rho)));
  } else {
    const A pn = sqrt(pn2);
    return A(0.5) * (tau0 + sqrt(tau0 * tau0 + les_c * pn / rho));
  }
}

// Relaxation rates of one cell: the configured ones, or the LES-adjusted
// ones (TRT keeps the magic parameter, BGK keeps omega_m = omega_p).
// omega: the per-cell relaxation field (Solver::set_omega_field; null when
// off): TRT takes omega+ = field, c+ = 1 - omega+/2 with omega- unchanged
// (kernels.rs:151-156), the central moment its shear rate (kernels.rs:481).
// It travels beside HydroParams rather than in it: the tuned sweep kernels
// are sensitive to the layout of their parameter block (a changed layout
// cost the cp.async central-moment kernel 8-14% on B200).
template <int Q, class A, bool FAST = false, bool FIELD = true>
__device__ __forceinline__ void cell_rates(const HydroParams<A>& p, const A (&f)[Q], A rho, A ux, A uy, A uz, A& op,
                                           A& om, A& cp, A& cm, A& os, int64_t cell, const A* omega = nullptr) {
  op = p.omega_p;
  om = p.omega_m;
  cp = p.cp;
  cm = p.cm;
  os = p.omega_shear;
  if (FIELD && omega) {
    op = omega[cell];
    cp = A(1) - op / A(2);
    os = op;
    return;
  }
  if (p.les_c > A(0)) {
    const A te = les_tau<Q, A, FAST>(f, rho, ux, uy, uz, p.les_c, p.tau0);
    if constexpr (FAST) {
      op = fast_rcp(te);
      om = p.magic > A(0) ? (te - A(0.5)) * fast_rcp(p.magic + A(0.5) * (te - A(0.5))) : op;
    } else {
      op = A(1) / te;
      om = p.magic > A(0) ? A(1) / (p.magic / (te - A(0.5)) + A(0.5)) : op;
    }
    cp = A(1) - op * A(0.5);
    cm = A(1) - om * A(0.5);
    os = op;
  }
}

// TRT + Guo (crates/lbm-core/src/collision.rs:123-202), BGK when
// omega_m == omega_p. Same operand grouping as the reference; the compiler
// may contract a*b+c into one fused rounding.
template <int Q, bool FORCED, class A>
__device__ __forceinline__ void collide_trt(A (&f)[Q], A rho, A ux, A uy, A uz, A Fx, A Fy, A Fz, A op, A om,
                                            A cp, A cm) {
  using L = Lat<Q>;
  const A usq = (ux * ux + uy * uy) + uz * uz;
  const A uf = (ux * Fx + uy * Fy) + uz * Fz;
  const A drho = rho - A(1);
  auto feq = [&](int q) {
    const A cu = (A(L::cx(q)) * ux + A(L::cy(q)) * uy) + A(L::cz(q)) * uz;
    const A inner = (A(3) * cu + (A(4.5) * cu) * cu) - A(1.5) * usq;
    return A(L::w(q)) * (drho + rho * inner);
  };
  auto src = [&](int q) {
    const A cu = (A(L::cx(q)) * ux + A(L::cy(q)) * uy) + A(L::cz(q)) * uz;
    const A cf = (A(L::cx(q)) * Fx + A(L::cy(q)) * Fy) + A(L::cz(q)) * Fz;
    return A(L::w(q)) * (A(3) * (cf - uf) + (A(9) * cu) * cf);
  };
  {
    const A e0 = feq(0);
    A v = f[0] - op * (f[0] - e0);
    if (FORCED) v = v + cp * src(0);
    f[0] = v;
  }
  const A half = A(0.5);
#pragma unroll
  for (int p = 0; p < L::NPAIR; ++p) {
    const int qa = 2 * p + 1, qb = 2 * p + 2;
    const A fa = f[qa], fb = f[qb];
    const A ea = feq(qa), eb = feq(qb);
    const A fp = half * (fa + fb), fm = half * (fa - fb);
    const A ep = half * (ea + eb), em = half * (ea - eb);
    const A rp = op * (fp - ep), rm = om * (fm - em);
    A va = (fa - rp) - rm, vb = (fb - rp) + rm;
    if (FORCED) {
      const A sa = src(qa), sb = src(qb);
      const A sp = half * (sa + sb), sm = half * (sa - sb);
      const A cps = cp * sp, cms = cm * sm;
      va = va + (cps + cms);
      vb = vb + (cps - cms);
    }
    f[qa] = va;
    f[qb] = vb;
  }
}

// Per-axis central-moment transform of one line (values at c = -1, 0, +1
// along the axis) about the velocity component u (factorised form of the
// reference's raw-moment matrix + binomial shift, kernels.rs:282-392).
template <class A>
__device__ __forceinline__ void cm_fwd(A& a, A& b, A& c, A u) {
  const A k0 = (a + b) + c;
  const A d = c - a;
  const A s = c + a;
  const A k1 = d - u * k0;
  const A k2 = (s - A(2) * u * d) + u * u * k0;
  a = k0;
  b = k1;
  c = k2;
}
template <class A>
__device__ __forceinline__ void cm_bwd(A& k0, A& k1, A& k2, A u) {
  const A m1 = k1 + u * k0;
  const A m2 = (k2 + A(2) * u * k1) + u * u * k0;
  const A fm = A(0.5) * (m2 - m1);
  const A f0 = k0 - m2;
  const A fp = A(0.5) * (m2 + m1);
  k0 = fm;
  k1 = f0;
  k2 = fp;
}

template <class A>
__device__ __forceinline__ void cm_fwd_all(A (&K)[3][3][3], A ux, A uy, A uz) {
#pragma unroll
  for (int i = 0; i < 3; ++i)
#pragma unroll
    for (int j = 0; j < 3; ++j) cm_fwd(K[i][j][0], K[i][j][1], K[i][j][2], uz);
#pragma unroll
  for (int i = 0; i < 3; ++i)
#pragma unroll
    for (int k = 0; k < 3; ++k) cm_fwd(K[i][0][k], K[i][1][k], K[i][2][k], uy);
#pragma unroll
  for (int j = 0; j < 3; ++j)
#pragma unroll
    for (int k = 0; k < 3; ++k) cm_fwd(K[0][j][k], K[1][j][k], K[2][j][k], ux);
}

// D3Q27 central-moment collision with Guo forcing (kernels.rs:406-533), in
// the arithmetic type. Post-collision moments are the reference's: order
// 0/1 keep the population moments (+ the source), order-2 deviatoric
// moments relax at omega_s (1 - 0.16 |u|^2) capped at 2, the order-2 trace
// and all higher moments relax at 1, the source enters with (1 - rate/2).
// By linearity the update is applied to the non-equilibrium part:
//   f_out = f + T^-1 [ -R T(f - feq) + (I - R/2) T(src) ].
//
// LES_K (unforced cells, fp32 fast math): the subgrid rate comes from the
// transformed moments. f - feq has zero raw moments of order 0 and 1 when
// u = j / rho, so its order-2 central moments equal the raw ones, i.e. the
// non-equilibrium stress Pi of les_tau: K200 = Pi_xx, K110 = Pi_xy, ...
// omega_shear = 1 / tau_eff then replaces the configured rate.
template <int Q, bool FORCED, class A, bool LES_K = false>
__device__ __forceinline__ void collide_cm(A (&f)[Q], A rho, A ux, A uy, A uz, A Fx, A Fy, A Fz, A omega_shear,
                                          A les_c = A(0), A tau0 = A(0)) {
  static_assert(!(LES_K && FORCED), "the moment-based subgrid rate needs u = j / rho");
  static_assert(Q == 27, "factorised central-moment collision needs the full D3Q27 tensor basis");
  using L = Lat<Q>;
  if (!FORCED && ux == A(0) && uy == A(0) && uz == A(0)) {
    // Exact-rest skip (kernels.rs:434-447): leave f untouched when every
    // population equals w (rho - 1) bitwise in the storage precision.
    bool exact = true;
#pragma unroll
    for (int q = 0; q < Q; ++q) exact = exact && (f[q] == A(L::w(q) * (double(rho) - 1.0)));
    if (exact) return;
  }
  const A usq = (ux * ux + uy * uy) + uz * uz;
  const A drho = rho - A(1);
  A K[3][3][3];
#pragma unroll
  for (int q = 0; q < Q; ++q) {
    const A cu = (A(L::cx(q)) * ux + A(L::cy(q)) * uy) + A(L::cz(q)) * uz;
    const A inner = (A(3) * cu + (A(4.5) * cu) * cu) - A(1.5) * usq;
    K[L::cx(q) + 1][L::cy(q) + 1][L::cz(q) + 1] = f[q] - A(L::w(q)) * (drho + rho * inner);
  }
  cm_fwd_all(K, ux, uy, uz);
  // K[a][b][c] now holds the non-equilibrium central moment (a, b, c);
  // overwrite it with the post-collision increment.
  if constexpr (LES_K) {
    if (les_c > A(0)) {
      const A pxx = K[2][0][0], pyy = K[0][2][0], pzz = K[0][0][2];
      const A pxy = K[1][1][0], pxz = K[1][0][1], pyz = K[0][1][1];
      const A pn = fast_sqrt((pxx * pxx + pyy * pyy + pzz * pzz) + A(2) * (pxy * pxy + pxz * pxz + pyz * pyz));
      omega_shear = fast_rcp(A(0.5) * (tau0 + fast_sqrt(tau0 * tau0 + les_c * pn * fast_rcp(rho))));
    }
  }
  const A os = fmin(omega_shear * (A(1) + A(-0.16) * usq), A(2));
  const A bulk_neq = (K[2][0][0] + K[0][2][0] + K[0][0][2]) * A(1.0 / 3.0);
#pragma unroll
  for (int a = 0; a < 3; ++a)
#pragma unroll
    for (int b = 0; b < 3; ++b)
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        const int order = a + b + c;
        const bool diag = order == 2 && (a == 2 || b == 2 || c == 2);
        A d;
        if (order <= 1) d = A(0);
        else if (diag) d = -os * (K[a][b][c] - bulk_neq) - bulk_neq;
        else if (order == 2) d = -os * K[a][b][c];
        else d = -K[a][b][c];
        K[a][b][c] = d;
      }
  if (FORCED) {
    A S[3][3][3];
    const A uf = (ux * Fx + uy * Fy) + uz * Fz;
#pragma unroll
    for (int q = 0; q < Q; ++q) {
      const A cu = (A(L::cx(q)) * ux + A(L::cy(q)) * uy) + A(L::cz(q)) * uz;
      const A cf = (A(L::cx(q)) * Fx + A(L::cy(q)) * Fy) + A(L::cz(q)) * Fz;
      S[L::cx(q) + 1][L::cy(q) + 1][L::cz(q) + 1] = A(L::w(q)) * (A(3) * (cf - uf) + (A(9) * cu) * cf);
    }
    cm_fwd_all(S, ux, uy, uz);
    const A bulk_src = (S[2][0][0] + S[0][2][0] + S[0][0][2]) * A(1.0 / 3.0);
#pragma unroll
    for (int a = 0; a < 3; ++a)
#pragma unroll
      for (int b = 0; b < 3; ++b)
#pragma unroll
        for (int c = 0; c < 3; ++c) {
          const int order = a + b + c;
          const bool diag = order == 2 && (a == 2 || b == 2 || c == 2);
          A s;
          if (order <= 1) s = S[a][b][c];
          else if (diag) s = A(0.5) * bulk_src + (A(1) - A(0.5) * os) * (S[a][b][c] - bulk_src);
          else if (order == 2) s = (A(1) - A(0.5) * os) * S[a][b][c];
          else s = A(0.5) * S[a][b][c];
          K[a][b][c] = K[a][b][c] + s;
        }
  }
#pragma unroll
  for (int j = 0; j < 3; ++j)
#pragma unroll
    for (int k = 0; k < 3; ++k) cm_bwd(K[0][j][k], K[1][j][k], K[2][j][k], ux);
#pragma unroll
  for (int i = 0; i < 3; ++i)
#pragma unroll
    for (int k = 0; k < 3; ++k) cm_bwd(K[i][0][k], K[i][1][k], K[i][2][k], uy);
#pragma unroll
  for (int i = 0; i < 3; ++i)
#pragma unroll
    for (int j = 0; j < 3; ++j) cm_bwd(K[i][j][0], K[i][j][1], K[i][j][2], uz);
#pragma unroll
  for (int q = 0; q < Q; ++q) f[q] = f[q] + K[L::cx(q) + 1][L::cy(q) + 1][L::cz(q) + 1];
}

// One cell. GENERIC: solid-neighbour mask, moving walls and periodic wrap;
// otherwise the interior fast path. FORCED: Guo source from the uniform
// force and, on F_FORCED cells, the force slots. FIELD: the per-cell
// relaxation field is read when set (kernels that never run with a field
// compile it out).
template <int Q, class S, int COLL, bool ODD, bool GENERIC, bool FORCED, bool FIELD = false>
__device__ __forceinline__ void hydro_cell(const HydroParams<typename Codec<S>::A>& p, int x, int y, int z,
                                           uint32_t cell, uint8_t fl,
                                           const typename Codec<S>::A* omega = nullptr) {
  using A = typename Codec<S>::A;
  using L = Lat<Q>;
  using CD = Codec<S>;
  S* fb = static_cast<S*>(p.f);
  const uint32_t pl = p.plane;
  const int nx = p.nx, nxy = p.nxy;
  uint32_t mask = 0u;
  int xs[3], ys[3], zs[3];
  if (GENERIC) {
    mask = (fl & F_BOUNDARY) ? p.nbr[cell] : 0u;
    xs[0] = x == 0 ? p.nx - 1 : x - 1;
    xs[1] = x;
    xs[2] = x == p.nx - 1 ? 0 : x + 1;
    ys[0] = y == 0 ? p.ny - 1 : y - 1;
    ys[1] = y;
    ys[2] = y == p.ny - 1 ? 0 : y + 1;
    zs[0] = z == 0 ? p.nz - 1 : z - 1;
    zs[1] = z;
    zs[2] = z == p.nz - 1 ? 0 : z + 1;
  }
  auto nidx = [&](int dx, int dy, int dz) -> uint32_t {
    if (GENERIC) return (uint32_t(zs[dz + 1]) * uint32_t(p.ny) + uint32_t(ys[dy + 1])) * uint32_t(nx) + uint32_t(xs[dx + 1]);
    return cell + uint32_t(dx + dy * nx + dz * nxy);
  };
  A f[Q];
#pragma unroll
  for (int q = 0; q < Q; ++q) {
    if (!ODD) {
      f[q] = CD::ld(fb + (q * pl + cell));
    } else {
      const int o = opp(q);
      if (GENERIC && ((mask >> o) & 1u)) {
        // source solid: bounce-back (own slot q), or under a free-slip top
        // the mirrored population of the partner x - (cx, cy, 0)
        const int d = planar<Q>(o);  // x - (cx, cy, 0) = x + (-cx, -cy, 0)
        if ((mask & NBR_SLIP) && L::cz(q) == -1 && d > 0 && !((mask >> d) & 1u))
          f[q] = CD::ld(fb + (opp(mirror_z<Q>(q)) * pl + nidx(-L::cx(q), -L::cy(q), 0)));
        else
          f[q] = CD::ld(fb + (q * pl + cell));
      } else {
        f[q] = CD::ld(fb + (o * pl + nidx(-L::cx(q), -L::cy(q), -L::cz(q))));
      }
    }
  }
  // Moments (kernels.rs:627-668): rho = 1 + sum f, m = sum c f.
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
  // Force: uniform + per-cell field (KParams::force_at, params.rs:386-405).
  A Fpx = A(0), Fpy = A(0), Fpz = A(0), Fcx = A(0), Fcy = A(0), Fcz = A(0);
  if (FORCED) {
    Fpx = Fcx = p.gx;
    Fpy = Fcy = p.gy;
    Fpz = Fcz = p.gz;
    if (fl & F_FORCED) {
      const int32_t s = p.fslot[cell];
      const Vec4<A> a = p.fprev[s];
      const Vec4<A> b = p.fcur[s];
      Fpx = Fpx + a.x;
      Fpy = Fpy + a.y;
      Fpz = Fpz + a.z;
      Fcx = Fcx + b.x;
      Fcy = Fcy + b.y;
      Fcz = Fcz + b.z;
    }
  }
  const A rho = A(1) + dr;
  const A inv = A(1) / rho;
  const A half = A(0.5);
  const A ux = (m0 + half * Fpx) * inv;
  const A uy = (m1 + half * Fpy) * inv;
  const A uz = (m2 + half * Fpz) * inv;
  A op, om, cp, cm, os;
  cell_rates<Q, A, false, FIELD>(p, f, rho, ux, uy, uz, op, om, cp, cm, os, cell, omega);
  if constexpr (COLL == COLL_CM)
    collide_cm<Q, FORCED, A>(f, rho, ux, uy, uz, Fcx, Fcy, Fcz, os);
  else
    collide_trt<Q, FORCED, A>(f, rho, ux, uy, uz, Fcx, Fcy, Fcz, op, om, cp, cm);
#pragma unroll
  for (int q = 0; q < Q; ++q) {
    A v = f[q];
    const int o = opp(q);
    const bool wall = GENERIC && ((mask >> q) & 1u);
    // free-slip top: specular to the fluid partner x + (cx, cy, 0)
    const int d = planar<Q>(q);
    const bool slip = GENERIC && wall && (mask & NBR_SLIP) && L::cz(q) == 1 && d > 0 && !((mask >> d) & 1u);
    if (GENERIC && wall && !slip && (fl & F_MOVING)) {
      const Vec4<A> wu = p.wall_u[nidx(L::cx(q), L::cy(q), L::cz(q))];
      const A cu = (A(L::cx(o)) * wu.x + A(L::cy(o)) * wu.y) + A(L::cz(o)) * wu.z;
      v = v + ((A(6) * A(L::w(o))) * rho) * cu;
    }
    if (ODD && slip)
      CD::st(fb + (mirror_z<Q>(q) * pl + nidx(L::cx(q), L::cy(q), 0)), v);
    else if (!ODD || wall)
      CD::st(fb + (o * pl + cell), v);
    else
      CD::st(fb + (q * pl + nidx(L::cx(q), L::cy(q), L::cz(q))), v);
  }
}

// Out-of-line generic cell update (periodic wrap, solid neighbours, moving
// walls): compiled once per kernel so the unrolled fast paths keep the
// instruction cache.
template <int Q, class S, int COLL, bool ODD, bool FORCED>
__device__ __noinline__ void hydro_cell_generic(const HydroParams<typename Codec<S>::A> p, int x, int y, int z,
                                                uint32_t cell, uint8_t fl) {
  hydro_cell<Q, S, COLL, ODD, true, FORCED>(p, x, y, z, cell, fl);
}
// The same with the per-cell relaxation field (kernels that take it).
template <int Q, class S, int COLL, bool ODD, bool FORCED>
__device__ __noinline__ void hydro_cell_generic_field(const HydroParams<typename Codec<S>::A> p, int x, int y, int z,
                                                      uint32_t cell, uint8_t fl,
                                                      const typename Codec<S>::A* omega) {
  hydro_cell<Q, S, COLL, ODD, true, FORCED, true>(p, x, y, z, cell, fl, omega);
}

template <class A>
struct HydroOccupancy {
  static constexpr int MIN_BLOCKS = sizeof(A) == 8 ? 2 : 4;  // <= 128 regs (fp32), <= 255 (fp64)
};

// Full-grid sweep: block = one x-row segment, grid = (x tiles, ny, nz).
// FORCED = false skips F_FORCED cells (hydro_cells_kernel updates them after
// the IBM force update); FORCED = true (uniform body force) forces every cell.
template <int Q, class S, int COLL, bool ODD, bool FORCED>
__global__ void __launch_bounds__(128, HydroOccupancy<typename Codec<S>::A>::MIN_BLOCKS)
    hydro_aa_kernel(HydroParams<typename Codec<S>::A> p, const typename Codec<S>::A* omega) {
  const int x = blockIdx.x * blockDim.x + threadIdx.x;
  if (x >= p.nx) return;
  const int y = blockIdx.y, z = blockIdx.z;
  const uint32_t cell = (uint32_t(z) * uint32_t(p.ny) + uint32_t(y)) * uint32_t(p.nx) + uint32_t(x);
  const uint8_t fl = p.flags[cell];
  if (fl & F_SOLID) return;
  if (!FORCED && (fl & F_FORCED)) return;
  if (fl & (F_BOUNDARY | F_WRAP))
    hydro_cell_generic_field<Q, S, COLL, ODD, FORCED>(p, x, y, z, cell, fl, omega);
  else
    hydro_cell<Q, S, COLL, ODD, false, FORCED, true>(p, x, y, z, cell, fl, omega);
}

// Cell-list sweep over the forced cells (after the IBM force update).
template <int Q, class S, int COLL, bool ODD>
__device__ __forceinline__ void forced_cell(const HydroParams<typename Codec<S>::A>& p, uint32_t cell,
                                            const typename Codec<S>::A* omega = nullptr) {
  const uint32_t nxy = uint32_t(p.nxy);
  const int z = int(cell / nxy);
  const uint32_t r = cell - uint32_t(z) * nxy;
  const int y = int(r / uint32_t(p.nx));
  const int x = int(r - uint32_t(y) * uint32_t(p.nx));
  const uint8_t fl = p.flags[cell];
  if (fl & F_SOLID) return;
  hydro_cell<Q, S, COLL, ODD, true, true, true>(p, x, y, z, cell, fl, omega);
}

template <int Q, class S, int COLL, bool ODD>
__global__ void __launch_bounds__(128, HydroOccupancy<typename Codec<S>::A>::MIN_BLOCKS)
    hydro_cells_kernel(HydroParams<typename Codec<S>::A> p, const int64_t* cells, int64_t ncells,
                       const typename Codec<S>::A* omega) {
  const int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
  if (i >= ncells) return;
  forced_cell<Q, S, COLL, ODD>(p, uint32_t(cells[i]), omega);
}

}  // namespace lbmb
