// Discrete adjoint of the stirred-tank runner step (TRT / BGK + Guo forcing,
// half-way bounce-back, direct-forcing IBM with a fixed number of sweeps).
//
// Forward step n (runner.rs:1079-1129 with the IBM of solver.rs:3016-3282):
//   IBM on f^n:   rho_s = 1 + sum f(s), u_s = j_s / rho_s at the stencil cells,
//                 sweeps k = 0..K-1: um = sum_i w_i (u + du^k)_{s_i},
//                 imp^k = rel (t - um) / mob, spread += imp^k w, du += imp^k w / rho,
//                 torque^n = sum_k sum_m (r_m x imp^k_m W_m)_z, F^n = spread
//   hydro:        u = (j + Fp^n / 2) / rho, TRT collision with Guo source F^n,
//                 push stream with bounce-back -> f^{n+1};  Fp^{n+1} = F^n
// Objective J = sum_n Tbar^n torque^n (Tbar^n = 1 / |window| inside the
// averaging window). With lambda^n = dJ/df^n and mu^n = dJ/dFp^n, step n
// backwards is
//   lambda*_q(x) = lambda^{n+1}_q(x + c_q)       (fluid neighbour)
//                = lambda^{n+1}_{opp q}(x)         (solid neighbour)
//   collision adjoint (below), giving lambda^n on every fluid cell, the
//   adjoint of F^n (g_F + mu^{n+1}) and mu^n = dJ/dFp^n at the forced cells
//   IBM adjoint through the sweeps in reverse, adding dJ/df^n at the stencil
//   cells and accumulating dJ/dOmega and dJ/dx_m.
// Collision adjoint of f* = f - (w+ P+ + w- P-)(f - e) + (c+ P+ + c- P-) S
// (P+/P- the TRT pair projectors, c+/- = 1 - w+/- / 2):
//   a = w+ P+ l* + w- P- l*,   b = c+ P+ l* + c- P- l*
//   E_rho = sum_q a_q de_q/drho, E_a = sum_q a_q de_q/du_a, B_a = sum_q b_q dS_q/du_a
//   lambda_p = l*_p - a_p + E_rho + sum_a (E_a + B_a)(c_pa - u_a) / rho
//   g_F,a = sum_q b_q dS_q/dF_a,  g_Fp,a = (E_a + B_a) / (2 rho)
//   dJ/dw+ = -(P+ l*) . (f - e + S/2),  dJ/dw- = -(P- l*) . (f - e + S/2)
// The forward states come from checkpoints (recomputed segment by segment);
// the IBM intermediates of a step are recomputed with the forward kernels.
#pragma once
#include "aux.cuh"
#include "ibm.cuh"

namespace lbmb {

constexpr int ADJ_BLOCK = 128;

// AA storage at a parity -> the logical post-stream layout (same plane
// stride), in the storage type.
template <int Q, class S>
__global__ void snapshot_kernel(const S* fb, int64_t pl, const uint8_t* flags, const uint32_t* nbr, int nx, int ny,
                                int nz, int parity, S* out, int64_t n) {
  using A = typename Codec<S>::A;
  const int64_t cell = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
  if (cell >= n) return;
  const uint8_t fl = flags[cell];
  A f[Q];
  if (fl & F_SOLID) {
#pragma unroll
    for (int q = 0; q < Q; ++q) f[q] = Codec<S>::ld(fb + q * pl + cell);
  } else {
    int x, y, z;
    cell_xyz(cell, nx, ny, x, y, z);
    const uint32_t mask = (fl & F_BOUNDARY) ? nbr[cell] : 0u;
    load_post_stream<Q, S>(fb, pl, cell, x, y, z, nx, ny, nz, mask, parity, f);
  }
#pragma unroll
  for (int q = 0; q < Q; ++q) Codec<S>::st(out + q * pl + cell, f[q]);
}

template <class S>
struct AdjCollide {
  using A = typename Codec<S>::A;
  const S* f;          // logical f^n
  int64_t pl;
  const uint8_t* flags;
  const uint32_t* nbr;
  const Vec4<A>* wall_u;
  const int32_t* fslot;
  const Vec4<A>* F;    // F^n per slot
  const Vec4<A>* Fp;   // Fp^n per slot
  const A* lam_in;     // lambda^{n+1}
  A* lam_out;          // lambda^n (collision part)
  const double* mu_in; // mu^{n+1} per slot (x3)
  double* mu_out;      // mu^n per slot (x3)
  double* Fbar;        // adjoint of F^n per slot (x3)
  double* grad;        // [0] += dJ/dw+, [1] += dJ/dw-
  int nx, ny, nz;
  double op, om;
};

template <int N>
__device__ __forceinline__ void adj_block_add(double (&v)[N], double* out) {
  __shared__ double sh[N][ADJ_BLOCK / 32];
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
#pragma unroll
  for (int k = 0; k < N; ++k)
    for (int o = 16; o > 0; o >>= 1) v[k] += __shfl_down_sync(0xffffffffu, v[k], o);
  if (lane == 0)
#pragma unroll
    for (int k = 0; k < N; ++k) sh[k][wid] = v[k];
  __syncthreads();
  if (threadIdx.x == 0)
    for (int k = 0; k < N; ++k) {
      double s = 0.0;
      for (int w = 0; w < ADJ_BLOCK / 32; ++w) s += sh[k][w];
      atomicAdd(out + k, s);
    }
}

// Collision + stream adjoint of one fluid cell. FORCED: the cell carries an
// IBM force (F, Fp from its slot); otherwise both are zero and the Guo terms
// drop out at compile time.
template <int Q, class S, bool FORCED>
__device__ __forceinline__ void adj_cell(const AdjCollide<S>& p, int64_t cell, uint8_t fl, double (&gsum)[2]) {
  using L = Lat<Q>;
  using A = typename Codec<S>::A;
  const uint32_t mask = (fl & F_BOUNDARY) ? p.nbr[cell] : 0u;
  const int64_t pl = p.pl;
  // lambda*: reverse of the push stream with bounce-back
  A ls[Q];
  if (fl & (F_WRAP | F_SLIP)) {
    int x = 0, y = 0, z = 0;
    cell_xyz(cell, p.nx, p.ny, x, y, z);
    const Nbr nb(x, y, z, p.nx, p.ny, p.nz);
#pragma unroll
    for (int q = 0; q < Q; ++q) {
      if ((mask >> q) & 1u) {
        // free-slip top: the post-collision population went to the mirrored
        // direction of the fluid partner x + (cx, cy, 0)
        const int d = planar<Q>(q);
        if ((mask & NBR_SLIP) && L::cz(q) == 1 && d > 0 && !((mask >> d) & 1u))
          ls[q] = p.lam_in[mirror_z<Q>(q) * pl + nb.at(L::cx(q), L::cy(q), 0)];
        else
          ls[q] = p.lam_in[opp(q) * pl + cell];
      } else {
        ls[q] = p.lam_in[q * pl + nb.at(L::cx(q), L::cy(q), L::cz(q))];
      }
    }
  } else {
    const int64_t nxy = int64_t(p.nx) * p.ny;
#pragma unroll
    for (int q = 0; q < Q; ++q) {
      const int64_t d = int64_t(L::cx(q)) + int64_t(L::cy(q)) * p.nx + int64_t(L::cz(q)) * nxy;
      ls[q] = ((mask >> q) & 1u) ? p.lam_in[opp(q) * pl + cell] : p.lam_in[q * pl + cell + d];
    }
  }
  A f[Q];
#pragma unroll
  for (int q = 0; q < Q; ++q) f[q] = Codec<S>::ld(p.f + q * pl + cell);
  A F[3] = {A(0), A(0), A(0)}, Fp[3] = {A(0), A(0), A(0)};
  int32_t g = -1;
  if (FORCED) {
    g = p.fslot[cell];
    const Vec4<A> a = p.F[g], b = p.Fp[g];
    F[0] = a.x, F[1] = a.y, F[2] = a.z;
    Fp[0] = b.x, Fp[1] = b.y, Fp[2] = b.z;
  }
  A dr = A(0), j[3] = {A(0), A(0), A(0)};
#pragma unroll
  for (int q = 0; q < Q; ++q) {
    dr += f[q];
    j[0] += A(L::cx(q)) * f[q];
    j[1] += A(L::cy(q)) * f[q];
    j[2] += A(L::cz(q)) * f[q];
  }
  const A rho = A(1) + dr, inv = A(1) / rho;
  const A u[3] = {(j[0] + A(0.5) * Fp[0]) * inv, (j[1] + A(0.5) * Fp[1]) * inv, (j[2] + A(0.5) * Fp[2]) * inv};
  const A usq = u[0] * u[0] + u[1] * u[1] + u[2] * u[2];
  const A uF = u[0] * F[0] + u[1] * F[1] + u[2] * F[2];
  const A op = A(p.op), om = A(p.om), cp = A(1) - op * A(0.5), cm = A(1) - om * A(0.5);
  A Er = A(0), E[3] = {A(0), A(0), A(0)}, B[3] = {A(0), A(0), A(0)}, gF[3] = {A(0), A(0), A(0)};
  A dwp = A(0), dwm = A(0);
  A lp[Q], lm[Q];
  lp[0] = ls[0];
  lm[0] = A(0);
#pragma unroll
  for (int k = 0; k < (Q - 1) / 2; ++k) {
    const int a = 2 * k + 1, b = a + 1;
    const A sp = A(0.5) * (ls[a] + ls[b]), sm = A(0.5) * (ls[a] - ls[b]);
    lp[a] = sp, lp[b] = sp, lm[a] = sm, lm[b] = -sm;
  }
#pragma unroll
  for (int q = 0; q < Q; ++q) {
    const A c[3] = {A(L::cx(q)), A(L::cy(q)), A(L::cz(q))};
    const A cu = c[0] * u[0] + c[1] * u[1] + c[2] * u[2];
    const A w = A(L::w(q));
    const A aq = op * lp[q] + om * lm[q];
    const A e = w * (dr + rho * (A(3) * cu + A(4.5) * cu * cu - A(1.5) * usq));
    A r = f[q] - e;
    Er += aq * w * (A(1) + A(3) * cu + A(4.5) * cu * cu - A(1.5) * usq);
#pragma unroll
    for (int d = 0; d < 3; ++d) E[d] += aq * w * rho * (A(3) * c[d] + A(9) * cu * c[d] - A(3) * u[d]);
    if (FORCED) {
      const A cF = c[0] * F[0] + c[1] * F[1] + c[2] * F[2];
      const A bq = cp * lp[q] + cm * lm[q];
      r += A(0.5) * w * (A(3) * (cF - uF) + A(9) * cu * cF);
#pragma unroll
      for (int d = 0; d < 3; ++d) {
        B[d] += bq * w * (A(-3) * F[d] + A(9) * c[d] * cF);
        gF[d] += bq * w * (A(3) * (c[d] - u[d]) + A(9) * cu * c[d]);
      }
    }
    dwp -= lp[q] * r;
    dwm -= lm[q] * r;
  }
  // moving walls: f^{n+1}_{opp q}(x) gets + 6 w_{opp q} rho (c_{opp q} . u_w), rho = 1 + sum f
  A wall = A(0);
  if (fl & F_MOVING) {
    int x = 0, y = 0, z = 0;
    cell_xyz(cell, p.nx, p.ny, x, y, z);
    const Nbr nb(x, y, z, p.nx, p.ny, p.nz);
#pragma unroll
    for (int q = 0; q < Q; ++q)
      if (((mask >> q) & 1u) &&
          !((mask & NBR_SLIP) && L::cz(q) == 1 && planar<Q>(q) > 0 && !((mask >> planar<Q>(q)) & 1u))) {
        const int o = opp(q);
        const Vec4<A> wu = p.wall_u[nb.at(L::cx(q), L::cy(q), L::cz(q))];
        wall += ls[q] * A(6) * A(L::w(o)) * (A(L::cx(o)) * wu.x + A(L::cy(o)) * wu.y + A(L::cz(o)) * wu.z);
      }
  }
  const A G[3] = {(E[0] + B[0]) * inv, (E[1] + B[1]) * inv, (E[2] + B[2]) * inv};
  const A base = Er + wall - (G[0] * u[0] + G[1] * u[1] + G[2] * u[2]);
#pragma unroll
  for (int q = 0; q < Q; ++q) {
    const A aq = op * lp[q] + om * lm[q];
    p.lam_out[q * pl + cell] = ls[q] - aq + base + (G[0] * A(L::cx(q)) + G[1] * A(L::cy(q)) + G[2] * A(L::cz(q)));
  }
  if (FORCED) {
#pragma unroll
    for (int d = 0; d < 3; ++d) {
      p.Fbar[3 * g + d] = double(gF[d]) + p.mu_in[3 * g + d];
      p.mu_out[3 * g + d] = double(G[d] * A(0.5));
    }
  }
  gsum[0] += double(dwp);
  gsum[1] += double(dwm);
}

template <int Q, class S>
__global__ void __launch_bounds__(ADJ_BLOCK) adj_collide_kernel(AdjCollide<S> p, int64_t n) {
  const int64_t cell = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
  double gsum[2] = {0.0, 0.0};
  if (cell < n) {
    const uint8_t fl = p.flags[cell];
    if (!(fl & F_SOLID)) {
      if (fl & F_FORCED) adj_cell<Q, S, true>(p, cell, fl, gsum);
      else adj_cell<Q, S, false>(p, cell, fl, gsum);
    }
  }
  adj_block_add<2>(gsum, p.grad);
}

// Arrays of the IBM adjoint (per global slot / per marker, f64).
struct AdjIbm {
  IbmArgs a;             // forward arrays of the recomputed step (rho, u_now, mob, stencils)
  const double* imp_k;   // sweeps x nm x 3: impulse of each sweep
  const double* du_k;    // sweeps x nslot x 3: du at the start of each sweep
  int64_t nslot;         // global slot count (du_k stride)
  const int64_t* slot_cell;
  int nx, ny;
  int radius;
  double* Fbar;    // per slot x3 (adjoint of the final spread)
  double* dubar;   // per slot x3
  double* ubar;    // per slot x3
  double* rhobar;  // per slot
  double* cksbar;  // per slot
  double* umbar;   // per marker x3
  double* tbar;    // per marker x3
  double* mobbar;  // per marker
  double* xbar;    // per marker x3 (accumulates over steps)
  double* grad;    // [2] += dJ/dOmega_z
  const double* tbar_step;  // dJ/dtorque of this step (device scalar)
};

// d/dp of one axis factor of the marker kernel at distance p - i.
__device__ __forceinline__ void kernel_axis(double d, int radius, double& w, double& dw) {
  const double r = fabs(d), sg = d >= 0.0 ? 1.0 : -1.0;
  if (radius == 1) {
    w = r < 1.0 ? 1.0 - r : 0.0;
    dw = r < 1.0 ? -sg : 0.0;
  } else {
    if (r < 0.5) {
      w = 0.75 - r * r;
      dw = -2.0 * r * sg;
    } else if (r < 1.5) {
      w = 0.5 * (1.5 - r) * (1.5 - r);
      dw = -(1.5 - r) * sg;
    } else {
      w = 0.0;
      dw = 0.0;
    }
  }
}

// Gradient of the stencil weight of marker position pos at cell s.
__device__ __forceinline__ void weight_grad(const AdjIbm& b, const double* pos, int32_t s, double gw[3]) {
  const int64_t cell = b.slot_cell[s];
  const int64_t nxy = int64_t(b.nx) * b.ny;
  const int z = int(cell / nxy);
  const int y = int((cell - int64_t(z) * nxy) / b.nx);
  const int x = int(cell - int64_t(z) * nxy - int64_t(y) * b.nx);
  double w[3], dw[3];
  kernel_axis(pos[0] - double(x), b.radius, w[0], dw[0]);
  kernel_axis(pos[1] - double(y), b.radius, w[1], dw[1]);
  kernel_axis(pos[2] - double(z), b.radius, w[2], dw[2]);
  gw[0] = dw[0] * w[1] * w[2];
  gw[1] = w[0] * dw[1] * w[2];
  gw[2] = w[0] * w[1] * dw[2];
}

// Sweep k in reverse, per marker: impulse adjoint from the spread and the
// torque, then interpolation adjoint (needs dubar = adjoint of du^{k+1}).
static __global__ void __launch_bounds__(ADJ_BLOCK) adj_ibm_marker_kernel(AdjIbm b, int k) {
  const IbmArgs& a = b.a;
  const double Tbar = *b.tbar_step;
  const int64_t m = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
  if (m >= a.nm) return;
  const double* pos = a.pos + 3 * m;
  const double r[3] = {pos[0] - a.center[0], pos[1] - a.center[1], pos[2] - a.center[2]};
  const int32_t k0 = a.st_off[m], k1 = a.st_off[m + 1];
  const double mob = a.mob[m];
  if (k1 <= k0 || mob == 0.0) {
    for (int c = 0; c < 3; ++c) b.umbar[3 * m + c] = 0.0;
    return;
  }
  const double* imp = b.imp_k + (size_t(k) * a.nm + m) * 3;
  const double* du = b.du_k + size_t(k) * b.nslot * 3;
  double W = 0.0, ib[3] = {0.0, 0.0, 0.0};
  for (int32_t i = k0; i < k1; ++i) {
    const int32_t s = a.st_slot[i];
    const double w = a.st_w[i], ir = 1.0 / fmax(a.rho[s], 1.0e-30);
    W += w;
    for (int c = 0; c < 3; ++c) ib[c] += w * (b.Fbar[3 * s + c] + b.dubar[3 * s + c] * ir);
  }
  // torque^k = W (r_x imp_y - r_y imp_x)
  ib[0] += Tbar * W * (-r[1]);
  ib[1] += Tbar * W * r[0];
  const double rel = a.relax;
  double umb[3];
  for (int c = 0; c < 3; ++c) {
    umb[c] = -rel / mob * ib[c];
    b.umbar[3 * m + c] = umb[c];
    b.tbar[3 * m + c] += rel / mob * ib[c];
  }
  b.mobbar[m] += -(ib[0] * imp[0] + ib[1] * imp[1] + ib[2] * imp[2]) / mob;
  double xb[3] = {Tbar * W * imp[1], -Tbar * W * imp[0], 0.0};
  const double tq = r[0] * imp[1] - r[1] * imp[0];
  for (int32_t i = k0; i < k1; ++i) {
    const int32_t s = a.st_slot[i];
    const double ir = 1.0 / fmax(a.rho[s], 1.0e-30);
    double wb = Tbar * tq;
    for (int c = 0; c < 3; ++c)
      wb += imp[c] * (b.Fbar[3 * s + c] + b.dubar[3 * s + c] * ir) +
            umb[c] * (a.u_now[3 * s + c] + du[3 * s + c]);
    double gw[3];
    weight_grad(b, pos, s, gw);
    for (int c = 0; c < 3; ++c) xb[c] += wb * gw[c];
  }
  for (int c = 0; c < 3; ++c) b.xbar[3 * m + c] += xb[c];
}

// Sweep k in reverse, per slot (contributions in marker order): density and
// velocity adjoints, and dubar: adjoint of du^{k+1} -> adjoint of du^k.
static __global__ void __launch_bounds__(ADJ_BLOCK) adj_ibm_slot_kernel(AdjIbm b, int k) {
  const IbmArgs& a = b.a;
  const int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
  if (i >= a.ns) return;
  const int32_t g = a.bslot[i];
  const double rho = fmax(a.rho[g], 1.0e-30);
  const double db[3] = {b.dubar[3 * g], b.dubar[3 * g + 1], b.dubar[3 * g + 2]};
  double su[3] = {0.0, 0.0, 0.0}, sr = 0.0;
  for (int32_t c = a.cs_off[i]; c < a.cs_off[i + 1]; ++c) {
    const int32_t m = a.cs_marker[c];
    const double w = a.cs_w[c];
    const double* imp = b.imp_k + (size_t(k) * a.nm + m) * 3;
    sr += w * (imp[0] * db[0] + imp[1] * db[1] + imp[2] * db[2]);
    for (int d = 0; d < 3; ++d) su[d] += w * b.umbar[3 * m + d];
  }
  b.rhobar[g] += -sr / (rho * rho);
  for (int d = 0; d < 3; ++d) {
    b.ubar[3 * g + d] += su[d];
    b.dubar[3 * g + d] = db[d] + su[d];
  }
}

// Mobility adjoint, per slot: cell-kernel-sum adjoint and its density term.
static __global__ void __launch_bounds__(ADJ_BLOCK) adj_ibm_mob_slot_kernel(AdjIbm b) {
  const IbmArgs& a = b.a;
  const int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
  if (i >= a.ns) return;
  const int32_t g = a.bslot[i];
  const double rho = fmax(a.rho[g], 1.0e-30);
  double cks = 0.0, sm = 0.0;
  for (int32_t c = a.cs_off[i]; c < a.cs_off[i + 1]; ++c) {
    cks += a.cs_w[c];
    sm += a.cs_w[c] * b.mobbar[a.cs_marker[c]];
  }
  b.cksbar[g] = sm / rho;
  b.rhobar[g] += -sm * cks / (rho * rho);
}

// Mobility and target adjoints, per marker; resets the per-step marker
// accumulators; dJ/dOmega partials.
static __global__ void __launch_bounds__(ADJ_BLOCK) adj_ibm_mob_marker_kernel(AdjIbm b) {
  const IbmArgs& a = b.a;
  const int64_t m = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
  double gO[1] = {0.0};
  if (m < a.nm) {
    const double* pos = a.pos + 3 * m;
    const double r[3] = {pos[0] - a.center[0], pos[1] - a.center[1], pos[2] - a.center[2]};
    const double mb = b.mobbar[m];
    double xb[3] = {0.0, 0.0, 0.0};
    for (int32_t i = a.st_off[m]; i < a.st_off[m + 1]; ++i) {
      const int32_t s = a.st_slot[i];
      const double wb = mb * a.st_cks[i] / fmax(a.rho[s], 1.0e-30) + b.cksbar[s];
      double gw[3];
      weight_grad(b, pos, s, gw);
      for (int c = 0; c < 3; ++c) xb[c] += wb * gw[c];
    }
    // t = Omega z x r = (-Omega r_y, Omega r_x, 0)
    const double* tb = b.tbar + 3 * m;
    const double Om = a.omega[2];
    xb[0] += Om * tb[1];
    xb[1] += -Om * tb[0];
    gO[0] = -r[1] * tb[0] + r[0] * tb[1];
    for (int c = 0; c < 3; ++c) {
      b.xbar[3 * m + c] += xb[c];
      b.tbar[3 * m + c] = 0.0;
    }
    b.mobbar[m] = 0.0;
  }
  adj_block_add<1>(gO, b.grad + 2);
}

// dJ/df at the stencil cells from the IBM's rho_s and u_s, added to
// lambda^n; resets the per-slot accumulators.
template <int Q, class A>
__global__ void __launch_bounds__(ADJ_BLOCK) adj_ibm_fbar_kernel(AdjIbm b, A* lam, int64_t pl) {
  using L = Lat<Q>;
  const IbmArgs& a = b.a;
  const int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
  if (i >= a.ns) return;
  const int32_t g = a.bslot[i];
  const int64_t cell = b.slot_cell[g];
  const double rho = fmax(a.rho[g], 1.0e-30);
  const double rb = b.rhobar[g];
  const double ub[3] = {b.ubar[3 * g], b.ubar[3 * g + 1], b.ubar[3 * g + 2]};
  const double* u = a.u_now + 3 * g;
  const double base = rb - (ub[0] * u[0] + ub[1] * u[1] + ub[2] * u[2]) / rho;
#pragma unroll
  for (int q = 0; q < Q; ++q) {
    const double v = base + (ub[0] * L::cx(q) + ub[1] * L::cy(q) + ub[2] * L::cz(q)) / rho;
    lam[q * pl + cell] += A(v);
  }
  b.rhobar[g] = 0.0;
  b.cksbar[g] = 0.0;
  for (int d = 0; d < 3; ++d) {
    b.ubar[3 * g + d] = 0.0;
    b.dubar[3 * g + d] = 0.0;
  }
}

}  // namespace lbmb
