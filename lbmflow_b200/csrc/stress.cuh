// Shear-rate and stress QOIs on the device.
//
// * Native strain rate (Solver::strain_rate_at / gather_shear_rate,
//   solver.rs:5393-5599): Pi_neq = sum c c (f - feq(rho, u)) over the
//   post-stream populations and the cached moments, + 0.5 (uF + Fu) with the
//   current force, times -1 / (2 cs^2 rho tau_eff), tau_eff = 1 / omega_p;
//   in the storage's arithmetic type, like the reference's T.
// * Velocity-gradient stress (stress.rs:32-82 compute_stress_field as the
//   bioprocess runner calls it, runner.rs:1648-1690): f64 central
//   differences of the SI velocity (lattice velocity x dx/dt), one-sided
//   next to a solid or the domain edge, gamma_dot = sqrt(2 S:S), viscous
//   stress mu gamma_dot. The percentile summary (stress.rs:84-100) sorts the
//   finite fluid values on the device (cub radix sort) and interpolates
//   between ranks on the host.
// * Wall-shear proxy (stress.rs:102-294): fluid cells with a solid among
//   their 26 in-domain neighbours, compacted in cell order on the device.
#pragma once
#include <cub/device/device_radix_sort.cuh>
#include <cub/device/device_select.cuh>

#include "aux.cuh"

namespace lbmb {

// Arguments of the native strain rate of a cell.
template <class S>
struct StrainArgs {
  using A = typename Codec<S>::A;
  const S* fb;
  int64_t pl;
  const uint8_t* flags;
  const uint32_t* nbr;
  int nx, ny, nz, parity;
  const int32_t* fslot;
  const Vec4<A>* fprev;
  const Vec4<A>* fcur;
  int field_present;
  A gx, gy, gz, tau_eff;
};

// Native strain rate of fluid cell `cell` into pi (A precision) and its
// cached velocity into u.
template <int Q, class S>
__device__ __forceinline__ void strain_cell(const StrainArgs<S>& a, int64_t cell, typename Codec<S>::A (&pi)[6],
                                            typename Codec<S>::A (&u)[3]) {
  using A = typename Codec<S>::A;
  using L = Lat<Q>;
  const uint8_t fl = a.flags[cell];
  int x, y, z;
  cell_xyz(cell, a.nx, a.ny, x, y, z);
  const uint32_t mask = (fl & F_BOUNDARY) ? a.nbr[cell] : 0u;
  A f[Q];
  load_post_stream<Q, S>(a.fb, a.pl, cell, x, y, z, a.nx, a.ny, a.nz, mask, a.parity, f);
  // cached moments, as moments_kernel (the field inside them is fprev)
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
  A Fx = a.gx, Fy = a.gy, Fz = a.gz;  // force in the cached moments
  A Gx = a.gx, Gy = a.gy, Gz = a.gz;  // current force (KParams::force_at)
  if (fl & F_FORCED) {
    const int32_t sl = a.fslot[cell];
    const Vec4<A> v = a.fprev[sl];
    Fx = Fx + v.x;
    Fy = Fy + v.y;
    Fz = Fz + v.z;
    if (a.field_present) {
      const Vec4<A> b = a.fcur[sl];
      Gx = Gx + b.x;
      Gy = Gy + b.y;
      Gz = Gz + b.z;
    }
  }
  const A r = A(1) + dr;
  const A inv = A(1) / r;
  u[0] = (m0 + A(0.5) * Fx) * inv;
  u[1] = (m1 + A(0.5) * Fy) * inv;
  u[2] = (m2 + A(0.5) * Fz) * inv;
  // equilibrium in deviation form (kernels.rs:103-121)
  const A usq = u[0] * u[0] + u[1] * u[1] + u[2] * u[2];
  const A drho = r - A(1);
#pragma unroll
  for (int k = 0; k < 6; ++k) pi[k] = A(0);
#pragma unroll
  for (int q = 0; q < Q; ++q) {
    const A cx = A(L::cx(q)), cy = A(L::cy(q)), cz = A(L::cz(q));
    const A cu = cx * u[0] + cy * u[1] + cz * u[2];
    const A feq = A(L::w(q)) * (drho + r * (A(3) * cu + A(4.5) * cu * cu - A(1.5) * usq));
    const A fneq = f[q] - feq;
    pi[0] = pi[0] + cx * cx * fneq;
    pi[1] = pi[1] + cy * cy * fneq;
    pi[2] = pi[2] + cz * cz * fneq;
    pi[3] = pi[3] + cx * cy * fneq;
    pi[4] = pi[4] + cx * cz * fneq;
    pi[5] = pi[5] + cy * cz * fneq;
  }
  const A half = A(0.5);
  pi[0] = pi[0] + u[0] * Gx;
  pi[1] = pi[1] + u[1] * Gy;
  pi[2] = pi[2] + u[2] * Gz;
  pi[3] = pi[3] + half * (u[0] * Gy + u[1] * Gx);
  pi[4] = pi[4] + half * (u[0] * Gz + u[2] * Gx);
  pi[5] = pi[5] + half * (u[1] * Gz + u[2] * Gy);
  const A scale = -(A(1) / (A(2.0 / 3.0) * r * a.tau_eff));
#pragma unroll
  for (int k = 0; k < 6; ++k) pi[k] = pi[k] * scale;
}

template <int Q, class S>
__global__ void strain_rate_kernel(StrainArgs<S> a, double* s6, double* gamma, int64_t n) {
  using A = typename Codec<S>::A;
  const int64_t cell = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
  if (cell >= n) return;
  if (a.flags[cell] & F_SOLID) {  // solid cells report zero strain
    if (s6)
      for (int k = 0; k < 6; ++k) s6[6 * cell + k] = 0.0;
    if (gamma) gamma[cell] = 0.0;
    return;
  }
  A pi[6], u[3];
  strain_cell<Q, S>(a, cell, pi, u);
  if (s6)
    for (int k = 0; k < 6; ++k) s6[6 * cell + k] = double(pi[k]);
  if (gamma) {
    const A ss = pi[0] * pi[0] + pi[1] * pi[1] + pi[2] * pi[2] + A(2) * (pi[3] * pi[3] + pi[4] * pi[4] + pi[5] * pi[5]);
    gamma[cell] = double(sqrt(A(2) * ss));
  }
}

// Velocity gradient of a fluid cell (Solver::gather_velocity_gradient,
// solver.rs:5482-5582): symmetric off-diagonal part from the native strain
// rate, diagonal and rotation from differences of the cached velocity
// (u3 = [ux | uy | uz] in f64, exact copies of the A values): central
// between fluid cells, -4/3 w + u + 1/3 u(+1) (mirrored) next to a solid
// whose wall velocity w counts, one-sided at a non-periodic domain edge,
// periodic faces wrapped.
template <int Q, class S>
__device__ __forceinline__ void vel_grad_cell(const StrainArgs<S>& a, const double* u3, const Vec4<typename Codec<S>::A>* wall_u,
                                              int per_x, int per_y, int per_z, int64_t cell,
                                              typename Codec<S>::A (&g)[3][3]) {
  using A = typename Codec<S>::A;
  A st[6], uc[3];
  strain_cell<Q, S>(a, cell, st, uc);
  const int64_t n = int64_t(a.nx) * a.ny * a.nz;
  int x, y, z;
  cell_xyz(cell, a.nx, a.ny, x, y, z);
  const int pos[3] = {x, y, z}, d[3] = {a.nx, a.ny, a.nz}, per[3] = {per_x, per_y, per_z};
  const A own[3] = {A(u3[cell]), A(u3[n + cell]), A(u3[2 * n + cell])};
  A fd[3][3];
  for (int ax = 0; ax < 3; ++ax) {
    // neighbours along ax: 0 none, 1 fluid, 2 solid (wall velocity)
    int kind[2];
    A v[2][3];
    for (int side = 0; side < 2; ++side) {
      int pp[3] = {pos[0], pos[1], pos[2]};
      pp[ax] += side == 0 ? 1 : -1;
      kind[side] = 0;
      if (pp[ax] < 0 || pp[ax] >= d[ax]) {
        if (!per[ax]) continue;
        pp[ax] = (pp[ax] + d[ax]) % d[ax];
      }
      const int64_t j = (int64_t(pp[2]) * a.ny + pp[1]) * a.nx + pp[0];
      if (a.flags[j] & F_SOLID) {
        const Vec4<A> w = wall_u[j];
        v[side][0] = w.x;
        v[side][1] = w.y;
        v[side][2] = w.z;
        kind[side] = 2;
      } else {
        v[side][0] = A(u3[j]);
        v[side][1] = A(u3[n + j]);
        v[side][2] = A(u3[2 * n + j]);
        kind[side] = 1;
      }
    }
    for (int comp = 0; comp < 3; ++comp) {
      const A pv = v[0][comp], mv = v[1][comp];
      A val = A(0);
      if (kind[0] == 1 && kind[1] == 1) val = (pv - mv) * A(0.5);
      else if (kind[0] == 1 && kind[1] == 2) val = -A(4.0 / 3.0) * mv + own[comp] + A(1.0 / 3.0) * pv;
      else if (kind[0] == 2 && kind[1] == 1) val = A(4.0 / 3.0) * pv - own[comp] - A(1.0 / 3.0) * mv;
      else if (kind[0] == 1 && kind[1] == 0) val = pv - own[comp];
      else if (kind[0] == 0 && kind[1] == 1) val = own[comp] - mv;
      fd[comp][ax] = val;
    }
  }
  const A sm[3][3] = {{st[0], st[3], st[4]}, {st[3], st[1], st[5]}, {st[4], st[5], st[2]}};
#pragma unroll
  for (int r = 0; r < 3; ++r)
#pragma unroll
    for (int q = 0; q < 3; ++q) g[r][q] = r == q ? fd[r][q] : sm[r][q] + A(0.5) * (fd[r][q] - fd[q][r]);
}

// Velocity gradient of every cell (g9, n x 9 row-major) and / or WALE
// (les.rs:120-211, Cw 0.325, Delta 1): nu_t and the omega+ field for the
// next collision; clip bound nu_t_max when clip != 0; counts[0] = clipped
// cells, maxbits = bits of the largest nu_t before clipping (non-negative,
// so integer order is value order).
template <int Q, class S>
__global__ void wale_kernel(StrainArgs<S> a, const double* u3, const Vec4<typename Codec<S>::A>* wall_u, int per_x,
                            int per_y, int per_z, typename Codec<S>::A nu0, int clip,
                            typename Codec<S>::A nu_t_max, double* g9, double* nu_t, typename Codec<S>::A* omega,
                            unsigned long long* counts, unsigned long long* maxbits, int64_t n) {
  using A = typename Codec<S>::A;
  const int64_t cell = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
  if (cell >= n) return;
  A g[3][3];
  if (a.flags[cell] & F_SOLID) {
    for (int i = 0; i < 9; ++i) g[i / 3][i % 3] = A(0);
  } else {
    vel_grad_cell<Q, S>(a, u3, wall_u, per_x, per_y, per_z, cell, g);
  }
  if (g9)
    for (int i = 0; i < 9; ++i) g9[9 * cell + i] = double(g[i / 3][i % 3]);
  if (!omega) return;
  A sr[3][3], g2[3][3], sd[3][3];
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) sr[i][j] = A(0.5) * (g[i][j] + g[j][i]);
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) {
      g2[i][j] = A(0);
      for (int k = 0; k < 3; ++k) g2[i][j] = g2[i][j] + g[i][k] * g[k][j];
    }
  const A tr = g2[0][0] + g2[1][1] + g2[2][2];
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) {
      sd[i][j] = A(0.5) * (g2[i][j] + g2[j][i]);
      if (i == j) sd[i][j] = sd[i][j] - tr / A(3);
    }
  A ss = A(0), sdsd = A(0);
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) {
      ss = ss + sr[i][j] * sr[i][j];
      sdsd = sdsd + sd[i][j] * sd[i][j];
    }
  const A cwd = A(0.325) * A(1);
  const A denom = pow(ss, A(2.5)) + pow(sdsd, A(1.25));
  A nut = denom > A(0) ? (cwd * cwd) * pow(sdsd, A(1.5)) / denom : A(0);
  if (nut == nut) {  // the reference's max ignores NaN
    const double nd = double(nut);
    atomicMax(maxbits, (unsigned long long)__double_as_longlong(nd));
  }
  if (clip && nut > nu_t_max) {
    atomicAdd(counts, 1ull);
    nut = nu_t_max;
  }
  if (nu_t) nu_t[cell] = double(nut);
  omega[cell] = A(1) / (A(3) * (nu0 + nut) + A(0.5));
}

// compute_stress_field on the cached velocity moments (lattice units, f64;
// solid entries are never read). key[i]: gamma_dot of a fluid cell when
// finite, else +NaN (solid or non-finite), so that an ascending sort puts
// the values the percentile summary keeps first; *nfinite counts them.
static __global__ void stress_field_kernel(const double* ux, const double* uy, const double* uz, const uint8_t* flags,
                                    int nx, int ny, int nz, double dx, double vscale, double mu, double* s6,
                                    double* gamma, double* viscous, double* key, unsigned long long* nfinite,
                                    int64_t n) {
  const int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
  int finite = 0;
  if (i < n) {
    double gd = __longlong_as_double(0x7ff8000000000000ll);
    if (!(flags[i] & F_SOLID)) {
      int x, y, z;
      cell_xyz(i, nx, ny, x, y, z);
      const int d[3] = {nx, ny, nz};
      const int pos[3] = {x, y, z};
      const double* fld[3] = {ux, uy, uz};
      double g[3][3];
      for (int comp = 0; comp < 3; ++comp)
        for (int axis = 0; axis < 3; ++axis) {
          g[comp][axis] = 0.0;
          if (d[axis] <= 1) continue;
          const int64_t stride = axis == 0 ? 1 : (axis == 1 ? int64_t(nx) : int64_t(nx) * ny);
          const bool hp = pos[axis] + 1 < d[axis] && !(flags[i + stride] & F_SOLID);
          const bool hm = pos[axis] - 1 >= 0 && !(flags[i - stride] & F_SOLID);
          const double own = fld[comp][i] * vscale;
          if (hp && hm) {
            const double pv = fld[comp][i + stride] * vscale, mv = fld[comp][i - stride] * vscale;
            g[comp][axis] = (pv - mv) / (2.0 * dx);
          } else if (hp) {
            g[comp][axis] = (fld[comp][i + stride] * vscale - own) / dx;
          } else if (hm) {
            g[comp][axis] = (own - fld[comp][i - stride] * vscale) / dx;
          }
        }
      const double s[6] = {g[0][0], g[1][1], g[2][2], 0.5 * (g[0][1] + g[1][0]), 0.5 * (g[0][2] + g[2][0]),
                           0.5 * (g[1][2] + g[2][1])};
      const double ss = s[0] * s[0] + s[1] * s[1] + s[2] * s[2] + 2.0 * (s[3] * s[3] + s[4] * s[4] + s[5] * s[5]);
      const double v = sqrt(2.0 * ss);
      if (s6)
        for (int k = 0; k < 6; ++k) s6[6 * i + k] = s[k];
      if (gamma) gamma[i] = v;
      if (viscous) viscous[i] = mu * v;
      if (isfinite(v)) {
        gd = v;
        finite = 1;
      }
    } else {
      if (s6)
        for (int k = 0; k < 6; ++k) s6[6 * i + k] = 0.0;
      if (gamma) gamma[i] = 0.0;
      if (viscous) viscous[i] = 0.0;
    }
    if (key) key[i] = gd;
  }
  if (nfinite) {
    const unsigned b = __ballot_sync(0xffffffffu, finite);
    if ((threadIdx.x & 31) == 0 && b) atomicAdd(nfinite, (unsigned long long)__popc(b));
  }
}

// Values of sorted[0, k) above t (scaled by mul first, as the reference
// forms mu gamma_dot before it counts).
static __global__ void count_above_kernel(const double* sorted, int64_t k, double mul, double t, unsigned long long* out) {
  const int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
  const int above = (i < k) && (mul * sorted[i] > t);
  const unsigned b = __ballot_sync(0xffffffffu, above);
  if ((threadIdx.x & 31) == 0 && b) atomicAdd(out, (unsigned long long)__popc(b));
}

// wall_shear_proxy per cell (dense): flag[i] = 1 for a fluid cell with a
// solid among its 26 in-domain neighbours and a nonzero normal.
template <class A>
__global__ void wall_shear_kernel(const double* ux, const double* uy, const double* uz, const uint8_t* flags,
                                  const Vec4<A>* wall_u, int nx, int ny, int nz, double dx, double vscale, double rho,
                                  double mu, uint8_t* flag, double* tau, double* yplus, double* upar, double* normal,
                                  int64_t n) {
  const int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
  if (i >= n) return;
  flag[i] = 0;
  if (flags[i] & F_SOLID) return;
  int x, y, z;
  cell_xyz(i, nx, ny, x, y, z);
  double nrm[3] = {0.0, 0.0, 0.0}, wu[3] = {0.0, 0.0, 0.0}, count = 0.0;
  for (int dz = -1; dz <= 1; ++dz)
    for (int dy = -1; dy <= 1; ++dy)
      for (int dxo = -1; dxo <= 1; ++dxo) {
        if (!dxo && !dy && !dz) continue;
        const int a = x + dxo, b = y + dy, c = z + dz;
        if (a < 0 || b < 0 || c < 0 || a >= nx || b >= ny || c >= nz) continue;
        const int64_t j = (int64_t(c) * ny + b) * nx + a;
        if (!(flags[j] & F_SOLID)) continue;
        nrm[0] += double(dxo);
        nrm[1] += double(dy);
        nrm[2] += double(dz);
        const Vec4<A> w = wall_u[j];
        wu[0] += double(w.x) * vscale;
        wu[1] += double(w.y) * vscale;
        wu[2] += double(w.z) * vscale;
        count += 1.0;
      }
  if (count == 0.0) return;
  const double mag = sqrt(nrm[0] * nrm[0] + nrm[1] * nrm[1] + nrm[2] * nrm[2]);
  if (mag == 0.0) return;
  for (int k = 0; k < 3; ++k) {
    nrm[k] /= mag;
    wu[k] /= count;
  }
  const double u[3] = {ux[i] * vscale - wu[0], uy[i] * vscale - wu[1], uz[i] * vscale - wu[2]};
  const double un = u[0] * nrm[0] + u[1] * nrm[1] + u[2] * nrm[2];
  const double t[3] = {u[0] - un * nrm[0], u[1] - un * nrm[1], u[2] - un * nrm[2]};
  const double up = sqrt(t[0] * t[0] + t[1] * t[1] + t[2] * t[2]);
  const double y_m = 0.5 * dx;
  const double tw = mu * up / y_m;
  flag[i] = 1;
  tau[i] = tw;
  yplus[i] = y_m * sqrt(tw / rho) / (mu / rho);
  upar[i] = up;
  for (int k = 0; k < 3; ++k) normal[3 * i + k] = nrm[k];
}

static __global__ void iota_kernel(int64_t* out, int64_t n) {
  const int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
  if (i < n) out[i] = i;
}

// Rows of the compacted wall cells: {tau_w, y+, |u_par|, normal x3}.
static __global__ void gather_wall_kernel(const int64_t* sel, int64_t k, const double* tau, const double* yplus,
                                   const double* upar, const double* normal, double* out) {
  const int64_t r = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
  if (r >= k) return;
  const int64_t i = sel[r];
  out[7 * r] = tau[i];
  out[7 * r + 1] = yplus[i];
  out[7 * r + 2] = upar[i];
  for (int a = 0; a < 3; ++a) out[7 * r + 3 + a] = normal[3 * i + a];
  out[7 * r + 6] = 0.0;
}

}  // namespace lbmb
