// Passive-scalar advection-diffusion (crates/lbm-core/src/solver.rs:
// 2113-2205, scalar.rs:6-15) on the device, AA pattern with its own parity.
//
// Per fluid cell: u = moments of the current hydro state (the reference's
// just-updated cached moments), C = sum h (the concentration after the
// previous scalar stream), BGK collide towards h_eq = w C (1 + c.u/cs^2)
// with omega = 1/(D/cs^2 + 1/2), then push-stream with half-way
// bounce-back. The scalar lattice is D3Q7 (cs^2 = 1/4) or the hydro
// lattice itself (cs^2 = 1/3, the reference's choice).
#pragma once
#include "aux.cuh"
#include "common.cuh"
#include "ibm.cuh"
#include "lattice.cuh"

namespace lbmb {

template <class A>
struct ScalarParams {
  A* h;                 // SQ planes
  int64_t hplane;
  const void* f;        // hydro populations
  int64_t plane;
  const uint8_t* flags;
  const uint32_t* nbr;
  const int32_t* fslot;
  const Vec4<A>* fprev;  // field inside the current moments
  int nx, ny, nz;
  int hparity;           // hydro AA parity of the current state
  A omega;               // scalar relaxation rate
  A gx, gy, gz;
};

template <int HQ, class S>
__device__ __forceinline__ void hydro_velocity(const ScalarParams<typename Codec<S>::A>& p, int64_t cell, int x,
                                               int y, int z, uint8_t fl, uint32_t mask,
                                               typename Codec<S>::A& ux, typename Codec<S>::A& uy,
                                               typename Codec<S>::A& uz) {
  using A = typename Codec<S>::A;
  using L = Lat<HQ>;
  A f[HQ];
  load_post_stream<HQ, S>(static_cast<const S*>(p.f), p.plane, cell, x, y, z, p.nx, p.ny, p.nz, mask, p.hparity,
                          f);
  A dr = A(0), m0 = A(0), m1 = A(0), m2 = A(0);
#pragma unroll
  for (int q = 0; q < HQ; ++q) {
    dr = dr + f[q];
    if (L::cx(q) == 1) m0 = m0 + f[q];
    if (L::cx(q) == -1) m0 = m0 - f[q];
    if (L::cy(q) == 1) m1 = m1 + f[q];
    if (L::cy(q) == -1) m1 = m1 - f[q];
    if (L::cz(q) == 1) m2 = m2 + f[q];
    if (L::cz(q) == -1) m2 = m2 - f[q];
  }
  A Fx = p.gx, Fy = p.gy, Fz = p.gz;
  if (fl & F_FORCED) {
    const Vec4<A> a = p.fprev[p.fslot[cell]];
    Fx = Fx + a.x;
    Fy = Fy + a.y;
    Fz = Fz + a.z;
  }
  const A r = A(1) + dr;
  const A inv = A(1) / r;
  ux = (m0 + A(0.5) * Fx) * inv;
  uy = (m1 + A(0.5) * Fy) * inv;
  uz = (m2 + A(0.5) * Fz) * inv;
}

// scalar_equilibrium (scalar.rs:6-15) with the lattice's 1/cs^2.
template <int SQ, class A>
__device__ __forceinline__ A scalar_feq(int q, A c, A ux, A uy, A uz) {
  using L = Lat<SQ>;
  const A cu = (A(L::cx(q)) * ux + A(L::cy(q)) * uy) + A(L::cz(q)) * uz;
  return (A(L::w(q)) * c) * (A(1) + A(L::INV_CS2) * cu);
}

template <int SQ, int HQ, class S, bool ODD>
__global__ void __launch_bounds__(128) scalar_step_kernel(ScalarParams<typename Codec<S>::A> p) {
  using A = typename Codec<S>::A;
  using L = Lat<SQ>;
  const int x = blockIdx.x * blockDim.x + threadIdx.x;
  if (x >= p.nx) return;
  const int y = blockIdx.y, z = blockIdx.z;
  const int64_t cell = (int64_t(z) * p.ny + y) * p.nx + x;
  const uint8_t fl = p.flags[cell];
  if (fl & F_SOLID) return;
  const uint32_t mask = (fl & F_BOUNDARY) ? p.nbr[cell] : 0u;
  A ux, uy, uz;
  hydro_velocity<HQ, S>(p, cell, x, y, z, fl, mask, ux, uy, uz);
  const Nbr nb(x, y, z, p.nx, p.ny, p.nz);
  A h[SQ];
  A c = A(0);
#pragma unroll
  for (int q = 0; q < SQ; ++q) {
    if (!ODD) {
      h[q] = p.h[q * p.hplane + cell];
    } else {
      const int o = opp(q);
      if ((mask >> o) & 1u)
        h[q] = p.h[q * p.hplane + cell];
      else
        h[q] = p.h[o * p.hplane + nb.at(-L::cx(q), -L::cy(q), -L::cz(q))];
    }
    c = c + h[q];
  }
#pragma unroll
  for (int q = 0; q < SQ; ++q) {
    const A heq = scalar_feq<SQ, A>(q, c, ux, uy, uz);
    const A v = h[q] - p.omega * (h[q] - heq);
    const int o = opp(q);
    const bool wall = (mask >> q) & 1u;
    if (!ODD || wall)
      p.h[o * p.hplane + cell] = v;
    else
      p.h[q * p.hplane + nb.at(L::cx(q), L::cy(q), L::cz(q))] = v;
  }
}

// Concentration C = sum h of the current scalar state; 0 on solids.
template <int SQ, class A>
__device__ __forceinline__ A scalar_conc(const A* hb, int64_t hpl, int64_t cell, int x, int y, int z, int nx,
                                         int ny, int nz, uint32_t mask, int sparity) {
  using L = Lat<SQ>;
  A c = A(0);
  if (sparity == 0) {
#pragma unroll
    for (int q = 0; q < SQ; ++q) c = c + hb[q * hpl + cell];
  } else {
    const Nbr nb(x, y, z, nx, ny, nz);
#pragma unroll
    for (int q = 0; q < SQ; ++q) {
      const int o = opp(q);
      if ((mask >> o) & 1u)
        c = c + hb[q * hpl + cell];
      else
        c = c + hb[o * hpl + nb.at(-L::cx(q), -L::cy(q), -L::cz(q))];
    }
  }
  return c;
}

template <int SQ, class A>
__global__ void scalar_gather_kernel(const A* hb, int64_t hpl, const uint8_t* flags, const uint32_t* nbr, int nx,
                                     int ny, int nz, int sparity, double* out, int64_t n) {
  const int64_t cell = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
  if (cell >= n) return;
  const uint8_t fl = flags[cell];
  if (fl & F_SOLID) {
    out[cell] = 0.0;
    return;
  }
  int x, y, z;
  cell_xyz(cell, nx, ny, x, y, z);
  const uint32_t mask = (fl & F_BOUNDARY) ? nbr[cell] : 0u;
  out[cell] = double(scalar_conc<SQ, A>(hb, hpl, cell, x, y, z, nx, ny, nz, mask, sparity));
}

// Checkpoint image of a scalar's populations (the SCALAR_FIELDS h planes,
// solver.rs:1200-1217): SQ planes over the halo-padded box, halo zero, the
// logical post-stream values (the read of scalar_step_kernel) in the file's
// type T; solid cells report their raw own slots. One thread per padded cell.
template <int SQ, class A, class T>
__global__ void scalar_pack_padded_kernel(const A* hb, int64_t hpl, const uint8_t* flags, const uint32_t* nbr, int nx,
                                          int ny, int nz, int sparity, T* out, int64_t np) {
  using L = Lat<SQ>;
  const int64_t p = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
  if (p >= np) return;
  const int64_t px = nx + 2, pxy = px * (ny + 2);
  const int zz = int(p / pxy);
  const int64_t r = p - zz * pxy;
  const int yy = int(r / px);
  const int x = int(r - yy * px) - 1, y = yy - 1, z = zz - 1;
  if (x < 0 || y < 0 || z < 0 || x >= nx || y >= ny || z >= nz) {
#pragma unroll
    for (int q = 0; q < SQ; ++q) out[q * np + p] = T(0);
    return;
  }
  const int64_t cell = (int64_t(z) * ny + y) * nx + x;
  const uint8_t fl = flags[cell];
  if (sparity == 0 || (fl & F_SOLID)) {
#pragma unroll
    for (int q = 0; q < SQ; ++q) out[q * np + p] = T(hb[q * hpl + cell]);
    return;
  }
  const uint32_t mask = (fl & F_BOUNDARY) ? nbr[cell] : 0u;
  const Nbr nb(x, y, z, nx, ny, nz);
#pragma unroll
  for (int q = 0; q < SQ; ++q) {
    const int o = opp(q);
    const A v = ((mask >> o) & 1u) ? hb[q * hpl + cell] : hb[o * hpl + nb.at(-L::cx(q), -L::cy(q), -L::cz(q))];
    out[q * np + p] = T(v);
  }
}

// Checkpoint image of a scalar -> normal (parity 0) layout.
template <class A, class T>
__global__ void scalar_unpack_padded_kernel(A* hb, int64_t hpl, const T* img, int sq, int nx, int ny, int nz,
                                            int64_t n) {
  const int64_t cell = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
  if (cell >= n) return;
  int x, y, z;
  cell_xyz(cell, nx, ny, x, y, z);
  const int64_t np = int64_t(nx + 2) * (ny + 2) * (nz + 2);
  const int64_t p = (int64_t(z + 1) * (ny + 2) + (y + 1)) * (nx + 2) + (x + 1);
  for (int q = 0; q < sq; ++q) hb[q * hpl + cell] = A(img[q * np + p]);
}

// h = h_eq(C, u) at every cell with u of the current hydro state (solids:
// u from the host-side initial values), normal layout (set_scalar_
// concentration, solver.rs:2910-2966).
template <int SQ, int HQ, class S>
__global__ void scalar_set_kernel(ScalarParams<typename Codec<S>::A> p, const double* conc, const double* usolid,
                                  int64_t n) {
  using A = typename Codec<S>::A;
  const int64_t cell = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
  if (cell >= n) return;
  const uint8_t fl = p.flags[cell];
  A ux, uy, uz;
  if (fl & F_SOLID) {
    ux = A(usolid[3 * cell]);
    uy = A(usolid[3 * cell + 1]);
    uz = A(usolid[3 * cell + 2]);
  } else {
    int x, y, z;
    cell_xyz(cell, p.nx, p.ny, x, y, z);
    const uint32_t mask = (fl & F_BOUNDARY) ? p.nbr[cell] : 0u;
    hydro_velocity<HQ, S>(p, cell, x, y, z, fl, mask, ux, uy, uz);
  }
  const A c = A(conc[cell]);
#pragma unroll
  for (int q = 0; q < SQ; ++q) p.h[q * p.hplane + cell] = scalar_feq<SQ, A>(q, c, ux, uy, uz);
}

// CV of the concentration over fluid cells, two passes like qoi::scalar_cv
// (qoi.rs:507-532): pass 0 sums C, pass 1 sums (C - mean)^2 with the mean
// read back from stats[0] / fluid count.
template <int SQ, class A>
__global__ void __launch_bounds__(RED_BLOCK) scalar_cv_kernel(const A* hb, int64_t hpl, const uint8_t* flags,
                                                              const uint32_t* nbr, int nx, int ny, int nz,
                                                              int sparity, int64_t n, int pass, const double* stats,
                                                              double nfluid, double* part) {
  __shared__ double sh[RED_BLOCK / 32];
  double v[1] = {0.0};
  const double mean = pass ? stats[0] / nfluid : 0.0;
  for (int64_t cell = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; cell < n;
       cell += int64_t(gridDim.x) * blockDim.x) {
    const uint8_t fl = flags[cell];
    if (fl & F_SOLID) continue;
    int x, y, z;
    cell_xyz(cell, nx, ny, x, y, z);
    const uint32_t mask = (fl & F_BOUNDARY) ? nbr[cell] : 0u;
    const double c = double(scalar_conc<SQ, A>(hb, hpl, cell, x, y, z, nx, ny, nz, mask, sparity));
    if (pass == 0) {
      v[0] += c;
    } else {
      const double d = c - mean;
      v[0] += d * d;
    }
  }
  block_sum<1>(v, sh);
  if (threadIdx.x == 0) part[blockIdx.x] = v[0];
}

static __global__ void scalar_cv_finish_kernel(const double* part, int nblk, int pass, double* stats, double nfluid,
                                        double* cv_out) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  double s = 0.0;
  for (int b = 0; b < nblk; ++b) s += part[b];
  if (pass == 0) {
    stats[0] = s;
    return;
  }
  const double mean = stats[0] / nfluid;
  double cv;
  if (!(nfluid > 0.0) || mean == 0.0)
    cv = __longlong_as_double(0x7ff8000000000000LL);
  else
    cv = sqrt(s / nfluid) / fabs(mean);
  if (cv_out) *cv_out = cv;
  stats[1] = cv;
}

// Oxygen transfer (oxygen.rs:124-191) or uptake (reaction.rs:57-137) on a
// gathered concentration array, in place, followed by the negative clip
// (oxygen.rs:193-216). Per block: the f64 sum of the source integral (mol/s
// for the transfer, kmol consumed for the uptake) and the minimum before
// the clip, in a fixed tree order; counts of active interface cells and of
// clipped cells; error bits (1 cell volume, 2 transfer inputs, 4 C_L < 0
// or not finite before the uptake, 8 cell density).
struct OxygenSourceArgs {
  int mode;  // 0 transfer, 1 uptake
  double dt, kl, cstar_u, vol_u;
  const double *cstar, *area, *vol, *density;
  int our_kind;  // 0 constant, 1 Monod, 2 cell-density scaled
  double our, our_max, ks, c_ref, specific_our;
};

constexpr int OXY_BLOCK = 256;

static __global__ void __launch_bounds__(OXY_BLOCK)
    oxygen_source_kernel(double* c, OxygenSourceArgs a, int* err, double* part, unsigned long long* cnt, int64_t n) {
  __shared__ double ssum[OXY_BLOCK], smin[OXY_BLOCK];
  const int64_t i = int64_t(blockIdx.x) * OXY_BLOCK + threadIdx.x;
  double contrib = 0.0, before = INFINITY;
  int active = 0, clipped = 0, e = 0;
  if (i < n) {
    const double v = a.vol ? a.vol[i] : a.vol_u;
    double ci = c[i];
    if (!(isfinite(v) && v > 0.0)) e |= 1;
    if (a.mode == 0) {
      const double cs = a.cstar ? a.cstar[i] : a.cstar_u;
      const double ar = a.area[i];
      if (!(isfinite(ci) && isfinite(cs) && isfinite(ar) && ar >= 0.0)) e |= 2;
      const double source = a.kl * ar * (cs - ci);
      active = ar > 0.0;
      ci += source * a.dt;
      contrib = source * v;
    } else {
      double rate = 0.0;
      if (!(isfinite(ci) && ci >= 0.0)) e |= 4;
      if (a.our_kind == 0) {
        rate = a.our;
      } else if (a.our_kind == 1) {
        const double cs = ci / a.c_ref;
        rate = a.our_max * cs / (a.ks + cs);
      } else {
        const double d = a.density[i];
        if (!(isfinite(d) && d >= 0.0)) e |= 8;
        rate = a.specific_our * d;
      }
      ci -= rate * a.dt;
      contrib = rate * v * a.dt;
    }
    before = ci;
    if (ci < 0.0) {
      ci = 0.0;
      clipped = 1;
    }
    c[i] = ci;
  }
  if (e) atomicOr(err, e);
  ssum[threadIdx.x] = contrib;
  smin[threadIdx.x] = before;
  __syncthreads();
  for (int s = OXY_BLOCK / 2; s > 0; s >>= 1) {
    if (int(threadIdx.x) < s) {
      ssum[threadIdx.x] += ssum[threadIdx.x + s];
      smin[threadIdx.x] = fmin(smin[threadIdx.x], smin[threadIdx.x + s]);
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    part[2 * blockIdx.x] = ssum[0];
    part[2 * blockIdx.x + 1] = smin[0];
  }
  const unsigned ba = __ballot_sync(0xffffffffu, active), bc = __ballot_sync(0xffffffffu, clipped);
  if ((threadIdx.x & 31) == 0) {
    if (ba) atomicAdd(cnt, (unsigned long long)__popc(ba));
    if (bc) atomicAdd(cnt + 1, (unsigned long long)__popc(bc));
  }
}

}  // namespace lbmb
