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

template <int Q, class S>
__global__ void strain_rate_kernel(const S* fb, int64_t pl, const uint8_t* flags, const uint32_t* nbr, int nx,
                                   int ny, int nz, int parity, const int32_t* fslot,
                                   const Vec4<typename Codec<S>::A>* fprev, const Vec4<typename Codec<S>::A>* fcur,
                                   int field_present, typename Codec<S>::A gx, typename Codec<S>::A gy,
                                   typename Codec<S>::A gz, typename Codec<S>::A tau_eff, double* s6, double* gamma,
                                   int64_t n) {
  using A = typename Codec<S>::A;
  using L = Lat<Q>;
  const int64_t cell = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
  if (cell >= n) return;
  const uint8_t fl = flags[cell];
  if (fl & F_SOLID) {  // solid cells report zero strain
    if (s6)
      for (int k = 0; k < 6; ++k) s6[6 * cell + k] = 0.0;
    if (gamma) gamma[cell] = 0.0;
    return;
  }
  int x, y, z;
  cell_xyz(cell, nx, ny, x, y, z);
  const uint32_t mask = (fl & F_BOUNDARY) ? nbr[cell] : 0u;
  A f[Q];
  load_post_stream<Q, S>(fb, pl, cell, x, y, z, nx, ny, nz, mask, parity, f);
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
  A Fx = gx, Fy = gy, Fz = gz;  // force in the cached moments
  A Gx = gx, Gy = gy, Gz = gz;  // current force (KParams::force_at)
  if (fl & F_FORCED) {
    const int32_t sl = fslot[cell];
    const Vec4<A> a = fprev[sl];
    Fx = Fx + a.x;
    Fy = Fy + a.y;
    Fz = Fz + a.z;
    if (field_present) {
      const Vec4<A> b = fcur[sl];
      Gx = Gx + b.x;
      Gy = Gy + b.y;
      Gz = Gz + b.z;
    }
  }
  const A r = A(1) + dr;
  const A inv = A(1) / r;
  const A u[3] = {(m0 + A(0.5) * Fx) * inv, (m1 + A(0.5) * Fy) * inv, (m2 + A(0.5) * Fz) * inv};
  // equilibrium in deviation form (kernels.rs:103-121)
  const A usq = u[0] * u[0] + u[1] * u[1] + u[2] * u[2];
  const A drho = r - A(1);
  A pi[6] = {A(0), A(0), A(0), A(0), A(0), A(0)};
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
  const A scale = -(A(1) / (A(2.0 / 3.0) * r * tau_eff));
#pragma unroll
  for (int k = 0; k < 6; ++k) pi[k] = pi[k] * scale;
  if (s6)
    for (int k = 0; k < 6; ++k) s6[6 * cell + k] = double(pi[k]);
  if (gamma) {
    const A ss = pi[0] * pi[0] + pi[1] * pi[1] + pi[2] * pi[2] + A(2) * (pi[3] * pi[3] + pi[4] * pi[4] + pi[5] * pi[5]);
    gamma[cell] = double(sqrt(A(2) * ss));
  }
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
