// Direct-forcing IBM on the device (crates/lbm-core/src/solver.rs:3016-3282).
//
// The reference runs this on the host over full-grid f64 arrays. Here only
// the stencil cells ("slots") are touched:
//   ibm_prep_kernel    per slot:   rho, u_now from the populations
//   ibm_interp_kernel  per marker: um, mobility, impulse, represented force
//   ibm_spread_kernel  per slot:   spread / du gathered in marker order
//   ibm_diag_kernel    per marker: slip statistics; the last block reduces
//                                  all partials in block order and decides
//                                  the early exit on the device
//   ibm_commit_kernel  per slot:   force field += spread (storage precision)
// Every kernel of a sweep returns at once when an earlier sweep converged,
// so a fixed launch sequence reproduces the reference's early exit without
// a host round trip (and can be captured in a CUDA graph).
//
// Summation order: per slot the contributions are gathered in ascending
// marker order (the reference's loop order), so spread, du and the cell
// kernel sum are bit-identical to the reference; the global diagnostics
// are fixed-order tree sums (deterministic run to run).
#pragma once
#include "common.cuh"
#include "lattice.cuh"

namespace lbmb {

constexpr int IBM_BLOCK = 128;

// The chain's kernels are launched with programmatic stream serialization:
// a kernel may be scheduled while its predecessor finishes, and waits here,
// before touching any memory, until the predecessor grid has completed and
// its writes are visible.
__device__ __forceinline__ void pdl_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }

struct IbmDiagDev {
  double slip_max, slip_rms, slip_max_rel, slip_rms_rel;
  double torque[3], fluid_force[3], marker_force[3];
  double momentum_error_rel;
  int iterations;
  int converged;
  unsigned int ticket;
  int pad;
};

struct IbmArgs {
  // markers
  int64_t nm;
  const double* pos;     // nm x 3
  const double* weight;  // nm
  const int32_t* st_off;   // nm + 1
  const int32_t* st_slot;  // active (non-solid) stencil points -> global slot
  const double* st_w;
  const double* st_cks;    // cell kernel sum of the point's cell (this body)
  // slots touched by this body
  int64_t ns;
  const int32_t* bslot;    // body slot -> global slot
  const int32_t* cs_off;   // ns + 1, contributions in marker order
  const int32_t* cs_marker;
  const double* cs_w;
  // per global slot state
  double* rho;       // cached density (f64 view)
  double* u_now;     // x3
  double* du;        // x3
  double* spread;    // x3
  // per marker state
  double* imp;       // x3
  double* mob;
  double* rmf;       // x3 represented marker force of this sweep
  // partials
  double* part_spread;  // gridDim(spread) x 3
  double* part_diag;    // gridDim(diag) x 9
  IbmDiagDev* diag;
  double center[3], omega[3];
  double scale, relax, tol;
};

__device__ __forceinline__ void ibm_target(const IbmArgs& a, int64_t m, double t[3], double r[3]) {
  r[0] = a.pos[3 * m + 0] - a.center[0];
  r[1] = a.pos[3 * m + 1] - a.center[1];
  r[2] = a.pos[3 * m + 2] - a.center[2];
  t[0] = a.omega[1] * r[2] - a.omega[2] * r[1];
  t[1] = a.omega[2] * r[0] - a.omega[0] * r[2];
  t[2] = a.omega[0] * r[1] - a.omega[1] * r[0];
}

// Post-stream populations of one cell in the AA layout of the given parity
// (0: normal, 1: swapped after an even step), as the arithmetic type.
template <int Q, class S>
__device__ __forceinline__ void load_post_stream(const S* fb, int64_t pl, int64_t cell, int x, int y,
                                                 int z, int nx, int ny, int nz, uint32_t mask,
                                                 int parity, typename Codec<S>::A (&f)[Q]) {
  using L = Lat<Q>;
  if (parity == 0) {
#pragma unroll
    for (int q = 0; q < Q; ++q) f[q] = Codec<S>::ld(fb + q * pl + cell);
  } else {
    const Nbr nb(x, y, z, nx, ny, nz);
#pragma unroll
    for (int q = 0; q < Q; ++q) {
      const int o = opp(q);
      if ((mask >> o) & 1u) {
        const int d = planar<Q>(o);
        if ((mask & NBR_SLIP) && L::cz(q) == -1 && d > 0 && !((mask >> d) & 1u))
          f[q] = Codec<S>::ld(fb + opp(mirror_z<Q>(q)) * pl + nb.at(-L::cx(q), -L::cy(q), 0));
        else
          f[q] = Codec<S>::ld(fb + q * pl + cell);
      } else {
        f[q] = Codec<S>::ld(fb + o * pl + nb.at(-L::cx(q), -L::cy(q), -L::cz(q)));
      }
    }
  }
}

// u_now over the body's slots (solver.rs:3036-3087): cached rho (storage
// arithmetic: 1 + sum f) and (sum c f + F/2) / rho in f64 with the force
// field current at call time.
template <int Q, class S>
__device__ __forceinline__ void ibm_prep_body(const IbmArgs& a, int64_t i, const S* fb, int64_t pl,
                                              const int64_t* slot_cell, const uint8_t* flags, const uint32_t* nbr,
                                              int nx, int ny, int nz, int parity,
                                              const Vec4<typename Codec<S>::A>* fcur, int field_present, double gx,
                                              double gy, double gz) {
  using A = typename Codec<S>::A;
  using L = Lat<Q>;
  if (i == 0) {
    IbmDiagDev* d = a.diag;
    d->slip_max = d->slip_rms = d->slip_max_rel = d->slip_rms_rel = 0.0;
    for (int k = 0; k < 3; ++k) d->torque[k] = d->fluid_force[k] = d->marker_force[k] = 0.0;
    d->momentum_error_rel = 0.0;
    d->iterations = 0;
    d->converged = 0;
    d->ticket = 0;
  }
  if (i >= a.ns) return;
  const int32_t g = a.bslot[i];
  const int64_t cell = slot_cell[g];
  const int64_t nxy = int64_t(nx) * ny;
  const int z = int(cell / nxy);
  const int y = int((cell - int64_t(z) * nxy) / nx);
  const int x = int(cell - int64_t(z) * nxy - int64_t(y) * nx);
  const uint32_t mask = (flags[cell] & F_BOUNDARY) ? nbr[cell] : 0u;
  A f[Q];
  load_post_stream<Q, S>(fb, pl, cell, x, y, z, nx, ny, nz, mask, parity, f);
  A dr = A(0);
  double mom[3] = {0.0, 0.0, 0.0};
#pragma unroll
  for (int q = 0; q < Q; ++q) {
    dr = dr + f[q];
    const double fq = double(f[q]);
    mom[0] += double(L::cx(q)) * fq;
    mom[1] += double(L::cy(q)) * fq;
    mom[2] += double(L::cz(q)) * fq;
  }
  const double rho = double(A(1) + dr);
  double force[3] = {gx, gy, gz};
  if (field_present) {
    const Vec4<A> fc = fcur[g];
    force[0] += double(fc.x);
    force[1] += double(fc.y);
    force[2] += double(fc.z);
  }
  const double inv_rho = 1.0 / fmax(rho, 1.0e-30);
  a.rho[g] = rho;
  for (int k = 0; k < 3; ++k) {
    a.u_now[3 * g + k] = (mom[k] + 0.5 * force[k]) * inv_rho;
    a.du[3 * g + k] = 0.0;
    a.spread[3 * g + k] = 0.0;
  }
}

template <int Q, class S>
__global__ void ibm_prep_kernel(IbmArgs a, const S* fb, int64_t pl, const int64_t* slot_cell,
                                const uint8_t* flags, const uint32_t* nbr, int nx, int ny, int nz,
                                int parity, const Vec4<typename Codec<S>::A>* fcur, int field_present,
                                double gx, double gy, double gz) {
  pdl_wait();
  ibm_prep_body<Q, S>(a, int64_t(blockIdx.x) * blockDim.x + threadIdx.x, fb, pl, slot_cell, flags, nbr, nx, ny, nz,
                      parity, fcur, field_present, gx, gy, gz);
}

// Impulse per marker from the current du (solver.rs:3118-3173).
__device__ __forceinline__ void ibm_interp_body(const IbmArgs& a, int64_t m, int sweep) {
  if (m >= a.nm) return;
  if (a.diag->converged) return;
  double t[3], r[3];
  ibm_target(a, m, t, r);
  double um[3] = {0.0, 0.0, 0.0};
  const int32_t k0 = a.st_off[m], k1 = a.st_off[m + 1];
  double mobility = 0.0;
  for (int32_t k = k0; k < k1; ++k) {
    const int32_t s = a.st_slot[k];
    const double w = a.st_w[k];
    um[0] += w * (a.u_now[3 * s + 0] + a.du[3 * s + 0]);
    um[1] += w * (a.u_now[3 * s + 1] + a.du[3 * s + 1]);
    um[2] += w * (a.u_now[3 * s + 2] + a.du[3 * s + 2]);
  }
  if (sweep == 0) {
    for (int32_t k = k0; k < k1; ++k) {
      const int32_t s = a.st_slot[k];
      mobility += a.st_w[k] * a.st_cks[k] / fmax(a.rho[s], 1.0e-30);
    }
    a.mob[m] = mobility;
  } else {
    mobility = a.mob[m];
  }
  double imp[3] = {0.0, 0.0, 0.0};
  if (mobility != 0.0) {
    imp[0] = a.relax * (t[0] - um[0]) / mobility;
    imp[1] = a.relax * (t[1] - um[1]) / mobility;
    imp[2] = a.relax * (t[2] - um[2]) / mobility;
  }
  double rmf[3] = {0.0, 0.0, 0.0};
  for (int32_t k = k0; k < k1; ++k) {
    const double w = a.st_w[k];
    rmf[0] += imp[0] * w;
    rmf[1] += imp[1] * w;
    rmf[2] += imp[2] * w;
  }
  for (int c = 0; c < 3; ++c) {
    a.imp[3 * m + c] = imp[c];
    a.rmf[3 * m + c] = rmf[c];
  }
}

static __global__ void ibm_interp_kernel(IbmArgs a, int sweep) {
  pdl_wait();
  ibm_interp_body(a, int64_t(blockIdx.x) * blockDim.x + threadIdx.x, sweep);
}

template <int N>
__device__ __forceinline__ void block_sum(double (&v)[N], double* sh) {
  // sh: N * (blockDim/32) doubles. Fixed-order warp + block tree.
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = blockDim.x >> 5;
#pragma unroll
  for (int k = 0; k < N; ++k)
    for (int o = 16; o > 0; o >>= 1) v[k] += __shfl_down_sync(0xffffffffu, v[k], o);
  if (lane == 0)
    for (int k = 0; k < N; ++k) sh[k * nw + wid] = v[k];
  __syncthreads();
  if (threadIdx.x == 0)
    for (int k = 0; k < N; ++k) {
      double s = 0.0;
      for (int w = 0; w < nw; ++w) s += sh[k * nw + w];
      v[k] = s;
    }
}

// Spread the impulses into the slots, in marker order (solver.rs:3174-3209).
// bid: block index within this body's spread grid (its partial slot).
__device__ __forceinline__ void ibm_spread_body(const IbmArgs& a, int64_t bid) {
  __shared__ double sh[3 * (IBM_BLOCK / 32)];
  if (a.diag->converged) return;
  const int64_t i = bid * blockDim.x + threadIdx.x;
  double ff[3] = {0.0, 0.0, 0.0};
  if (i < a.ns) {
    const int32_t g = a.bslot[i];
    double sp[3], d[3];
    for (int c = 0; c < 3; ++c) {
      sp[c] = a.spread[3 * g + c];
      d[c] = a.du[3 * g + c];
    }
    const double inv_rho = 1.0 / fmax(a.rho[g], 1.0e-30);
    for (int32_t k = a.cs_off[i]; k < a.cs_off[i + 1]; ++k) {
      const int32_t m = a.cs_marker[k];
      const double w = a.cs_w[k];
      for (int c = 0; c < 3; ++c) {
        const double cf = a.imp[3 * m + c] * w;
        sp[c] += cf;
        d[c] += cf * inv_rho;
        ff[c] += cf;
      }
    }
    for (int c = 0; c < 3; ++c) {
      a.spread[3 * g + c] = sp[c];
      a.du[3 * g + c] = d[c];
    }
  }
  block_sum<3>(ff, sh);
  if (threadIdx.x == 0)
    for (int c = 0; c < 3; ++c) a.part_spread[3 * bid + c] = ff[c];
}

static __global__ void __launch_bounds__(IBM_BLOCK) ibm_spread_kernel(IbmArgs a) {
  pdl_wait();
  ibm_spread_body(a, blockIdx.x);
}

// Slip statistics and the sweep's global reduction (solver.rs:3211-3253).
// bid / nblk: block index and block count of this body's diag grid.
__device__ __forceinline__ void ibm_diag_body(const IbmArgs& a, int sweep, int nblk_spread, unsigned int bid,
                                              unsigned int nblk) {
  __shared__ double sh[9 * (IBM_BLOCK / 32)];
  __shared__ double smax_sh[IBM_BLOCK / 32];
  __shared__ bool last;
  if (a.diag->converged) return;
  const int64_t m = int64_t(bid) * blockDim.x + threadIdx.x;
  double v[8] = {0, 0, 0, 0, 0, 0, 0, 0};  // ssq, wsum, mf[3], tq[3]
  double smax = 0.0;
  if (m < a.nm) {
    double t[3], r[3];
    ibm_target(a, m, t, r);
    const int32_t k0 = a.st_off[m], k1 = a.st_off[m + 1];
    if (k1 > k0) {
      double um[3] = {0.0, 0.0, 0.0};
      for (int32_t k = k0; k < k1; ++k) {
        const int32_t s = a.st_slot[k];
        const double w = a.st_w[k];
        um[0] += w * (a.u_now[3 * s + 0] + a.du[3 * s + 0]);
        um[1] += w * (a.u_now[3 * s + 1] + a.du[3 * s + 1]);
        um[2] += w * (a.u_now[3 * s + 2] + a.du[3 * s + 2]);
      }
      const double sl[3] = {t[0] - um[0], t[1] - um[1], t[2] - um[2]};
      const double mag = sqrt(sl[0] * sl[0] + sl[1] * sl[1] + sl[2] * sl[2]);
      smax = mag;
      v[0] = a.weight[m] * mag * mag;
      v[1] = a.weight[m];
    }
    const double* f = a.rmf + 3 * m;
    v[2] = f[0];
    v[3] = f[1];
    v[4] = f[2];
    v[5] = r[1] * f[2] - r[2] * f[1];
    v[6] = r[2] * f[0] - r[0] * f[2];
    v[7] = r[0] * f[1] - r[1] * f[0];
  }
  for (int o = 16; o > 0; o >>= 1) smax = fmax(smax, __shfl_down_sync(0xffffffffu, smax, o));
  if ((threadIdx.x & 31) == 0) smax_sh[threadIdx.x >> 5] = smax;
  block_sum<8>(v, sh);
  if (threadIdx.x == 0) {
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) smax = fmax(smax, smax_sh[w]);
    double* p = a.part_diag + 9 * bid;
    p[0] = smax;
    for (int k = 0; k < 8; ++k) p[1 + k] = v[k];
    __threadfence();
    const unsigned int t = atomicAdd(&a.diag->ticket, 1u);
    last = (t == nblk - 1);
  }
  __syncthreads();
  if (!last) return;
  __threadfence();
  // The last block reduces every partial: thread t takes blocks t, t + B,
  // ... in order, then a fixed tree (deterministic run to run).
  double acc[11] = {0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0};  // 8 diag sums, 3 spread sums
  double amax = 0.0;
  for (unsigned int b = threadIdx.x; b < nblk; b += blockDim.x) {
    const volatile double* p = a.part_diag + 9 * b;
    amax = fmax(amax, p[0]);
    for (int k = 0; k < 8; ++k) acc[k] += p[1 + k];
  }
  for (int b = threadIdx.x; b < nblk_spread; b += blockDim.x)
    for (int c = 0; c < 3; ++c) acc[8 + c] += ((const volatile double*)a.part_spread)[3 * b + c];
  __syncthreads();
  for (int o = 16; o > 0; o >>= 1) amax = fmax(amax, __shfl_down_sync(0xffffffffu, amax, o));
  if ((threadIdx.x & 31) == 0) smax_sh[threadIdx.x >> 5] = amax;
  __shared__ double sh2[11 * (IBM_BLOCK / 32)];
  block_sum<11>(acc, sh2);
  if (threadIdx.x != 0) return;
  for (int w = 0; w < (int)(blockDim.x >> 5); ++w) amax = fmax(amax, smax_sh[w]);
  double tot[9];
  tot[0] = amax;
  for (int k = 0; k < 8; ++k) tot[1 + k] = acc[k];
  const double ffs[3] = {acc[8], acc[9], acc[10]};
  IbmDiagDev* d = a.diag;
  for (int c = 0; c < 3; ++c) {
    d->fluid_force[c] += ffs[c];
    d->marker_force[c] += tot[3 + c];
    d->torque[c] -= tot[6 + c];
  }
  d->iterations = sweep + 1;
  d->slip_max = tot[0];
  d->slip_rms = tot[2] > 0.0 ? sqrt(tot[1] / tot[2]) : 0.0;
  d->slip_max_rel = d->slip_max / a.scale;
  d->slip_rms_rel = d->slip_rms / a.scale;
  const double e0 = d->fluid_force[0] - d->marker_force[0];
  const double e1 = d->fluid_force[1] - d->marker_force[1];
  const double e2 = d->fluid_force[2] - d->marker_force[2];
  const double mf = sqrt(d->marker_force[0] * d->marker_force[0] + d->marker_force[1] * d->marker_force[1] +
                         d->marker_force[2] * d->marker_force[2]);
  d->momentum_error_rel = sqrt(e0 * e0 + e1 * e1 + e2 * e2) / fmax(mf, 1.0e-12);
  if (d->slip_max_rel <= a.tol) d->converged = 1;
  d->ticket = 0;
}

static __global__ void __launch_bounds__(IBM_BLOCK) ibm_diag_kernel(IbmArgs a, int sweep, int nblk_spread) {
  pdl_wait();
  ibm_diag_body(a, sweep, nblk_spread, blockIdx.x, gridDim.x);
}

// force field += spread in the storage arithmetic (solver.rs:3256-3279),
// and optionally record the diagnostics of this call into per-step series.
template <class A>
__device__ __forceinline__ void ibm_commit_body(const IbmArgs& a, int64_t i, Vec4<A>* fcur, double* series_torque,
                                                double* series_ff, int32_t* series_iters, int64_t* step_counter) {
  if (i < a.ns) {
    const int32_t g = a.bslot[i];
    Vec4<A> v = fcur[g];
    v.x = v.x + A(a.spread[3 * g + 0]);
    v.y = v.y + A(a.spread[3 * g + 1]);
    v.z = v.z + A(a.spread[3 * g + 2]);
    fcur[g] = v;
  }
  if (i == 0 && step_counter) {
    const int64_t s = *step_counter;
    if (series_torque) series_torque[s] = -a.diag->torque[2];
    if (series_ff)
      for (int c = 0; c < 3; ++c) series_ff[3 * s + c] = a.diag->fluid_force[c];
    if (series_iters) series_iters[s] = a.diag->iterations;
    *step_counter = s + 1;
  }
}

template <class A>
__global__ void ibm_commit_kernel(IbmArgs a, Vec4<A>* fcur, double* series_torque, double* series_ff,
                                  int32_t* series_iters, int64_t* step_counter) {
  pdl_wait();
  ibm_commit_body<A>(a, int64_t(blockIdx.x) * blockDim.x + threadIdx.x, fcur, series_torque, series_ff,
                     series_iters, step_counter);
}

}  // namespace lbmb
