// Readback, staging and reduction kernels over the AA population layout.
#pragma once
#include "common.cuh"
#include "ibm.cuh"
#include "lattice.cuh"

namespace lbmb {

constexpr int RED_BLOCK = 256;

__device__ __forceinline__ void cell_xyz(int64_t cell, int nx, int ny, int& x, int& y, int& z) {
  const int64_t nxy = int64_t(nx) * ny;
  z = int(cell / nxy);
  const int64_t r = cell - int64_t(z) * nxy;
  y = int(r / nx);
  x = int(r - int64_t(y) * nx);
}

// Logical post-stream populations -> f64 q-major host layout (stage_out).
// Solid cells report their raw own slots (the reference leaves solid
// populations unspecified: streaming never writes them).
template <int Q, class S>
__global__ void stage_out_kernel(const S* fb, int64_t pl, const uint8_t* flags, const uint32_t* nbr,
                                 int nx, int ny, int nz, int parity, double* out, int64_t n) {
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
  for (int q = 0; q < Q; ++q) out[q * n + cell] = double(f[q]);
}

// f64 q-major host layout -> normal (parity 0) storage layout (stage_in).
template <int Q, class S>
__global__ void stage_in_kernel(S* fb, int64_t pl, const double* in, int64_t n) {
  const int64_t cell = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
  if (cell >= n) return;
#pragma unroll
  for (int q = 0; q < Q; ++q) Codec<S>::stage(fb + q * pl + cell, typename Codec<S>::A(in[q * n + cell]));
}

// Checkpoint image of the populations (solver.rs:4550-4552 over
// fields.rs:3-15): Q planes over the halo-padded box, padded index
// ((z + 1) (ny + 2) + y + 1) (nx + 2) + x + 1, halo cells zero, core cells
// the logical post-stream values in the file's type T (solid cells: their
// raw own slots, as stage_out). One thread per padded cell.
template <int Q, class S, class T>
__global__ void pack_padded_kernel(const S* fb, int64_t pl, const uint8_t* flags, const uint32_t* nbr, int nx,
                                   int ny, int nz, int parity, T* out, int64_t np) {
  using A = typename Codec<S>::A;
  const int64_t p = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
  if (p >= np) return;
  const int64_t px = nx + 2, pxy = px * (ny + 2);
  const int zz = int(p / pxy);
  const int64_t r = p - zz * pxy;
  const int yy = int(r / px);
  const int x = int(r - yy * px) - 1, y = yy - 1, z = zz - 1;
  if (x < 0 || y < 0 || z < 0 || x >= nx || y >= ny || z >= nz) {
#pragma unroll
    for (int q = 0; q < Q; ++q) out[q * np + p] = T(0);
    return;
  }
  const int64_t cell = (int64_t(z) * ny + y) * nx + x;
  const uint8_t fl = flags[cell];
  A f[Q];
  if (fl & F_SOLID) {
#pragma unroll
    for (int q = 0; q < Q; ++q) f[q] = Codec<S>::ld(fb + q * pl + cell);
  } else {
    const uint32_t mask = (fl & F_BOUNDARY) ? nbr[cell] : 0u;
    load_post_stream<Q, S>(fb, pl, cell, x, y, z, nx, ny, nz, mask, parity, f);
  }
#pragma unroll
  for (int q = 0; q < Q; ++q) out[q * np + p] = T(f[q]);
}

// Checkpoint image -> normal (parity 0) storage layout. One thread per cell.
template <int Q, class S, class T>
__global__ void unpack_padded_kernel(S* fb, int64_t pl, const T* img, int nx, int ny, int nz, int64_t n) {
  using A = typename Codec<S>::A;
  const int64_t cell = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
  if (cell >= n) return;
  int x, y, z;
  cell_xyz(cell, nx, ny, x, y, z);
  const int64_t np = int64_t(nx + 2) * (ny + 2) * (nz + 2);
  const int64_t p = (int64_t(z + 1) * (ny + 2) + (y + 1)) * (nx + 2) + (x + 1);
#pragma unroll
  for (int q = 0; q < Q; ++q) Codec<S>::stage(fb + q * pl + cell, A(img[q * np + p]));
}

// Moments of the current state (kernels.rs:627-668) with the force field
// that is inside the cached moments (fprev). Solid cells are skipped.
template <int Q, class S>
__global__ void moments_kernel(const S* fb, int64_t pl, const uint8_t* flags, const uint32_t* nbr,
                               int nx, int ny, int nz, int parity, const int32_t* fslot,
                               const Vec4<typename Codec<S>::A>* fprev, typename Codec<S>::A gx,
                               typename Codec<S>::A gy, typename Codec<S>::A gz, double* rho,
                               double* ux, double* uy, double* uz, int64_t n) {
  using A = typename Codec<S>::A;
  using L = Lat<Q>;
  const int64_t cell = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
  if (cell >= n) return;
  const uint8_t fl = flags[cell];
  if (fl & F_SOLID) return;
  int x, y, z;
  cell_xyz(cell, nx, ny, x, y, z);
  const uint32_t mask = (fl & F_BOUNDARY) ? nbr[cell] : 0u;
  A f[Q];
  load_post_stream<Q, S>(fb, pl, cell, x, y, z, nx, ny, nz, mask, parity, f);
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
  A Fx = gx, Fy = gy, Fz = gz;
  if (fl & F_FORCED) {
    const Vec4<A> a = fprev[fslot[cell]];
    Fx = Fx + a.x;
    Fy = Fy + a.y;
    Fz = Fz + a.z;
  }
  const A r = A(1) + dr;
  const A inv = A(1) / r;
  if (rho) rho[cell] = double(r);
  if (ux) ux[cell] = double((m0 + A(0.5) * Fx) * inv);
  if (uy) uy[cell] = double((m1 + A(0.5) * Fy) * inv);
  if (uz) uz[cell] = double((m2 + A(0.5) * Fz) * inv);
}

// Per-block f64 partials of the backend reductions (backend.rs:920-970):
// out[block] = {fluid cells, sum f_dev, momentum x, y, z (incl. F/2)}.
template <int Q, class S>
__global__ void __launch_bounds__(RED_BLOCK) reduce_kernel(const S* fb, int64_t pl, const uint8_t* flags,
                                                           const uint32_t* nbr, int nx, int ny, int nz,
                                                           int parity, const int32_t* fslot,
                                                           const Vec4<typename Codec<S>::A>* fcur,
                                                           double gx, double gy, double gz, int64_t n,
                                                           double* part) {
  using A = typename Codec<S>::A;
  using L = Lat<Q>;
  __shared__ double sh[5 * (RED_BLOCK / 32)];
  double v[5] = {0, 0, 0, 0, 0};
  for (int64_t cell = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; cell < n;
       cell += int64_t(gridDim.x) * blockDim.x) {
    const uint8_t fl = flags[cell];
    if (fl & F_SOLID) continue;
    int x, y, z;
    cell_xyz(cell, nx, ny, x, y, z);
    const uint32_t mask = (fl & F_BOUNDARY) ? nbr[cell] : 0u;
    A f[Q];
    load_post_stream<Q, S>(fb, pl, cell, x, y, z, nx, ny, nz, mask, parity, f);
    double s = 0.0, m0 = 0.0, m1 = 0.0, m2 = 0.0;
#pragma unroll
    for (int q = 0; q < Q; ++q) {
      const double fq = double(f[q]);
      s += fq;
      m0 += double(L::cx(q)) * fq;
      m1 += double(L::cy(q)) * fq;
      m2 += double(L::cz(q)) * fq;
    }
    double F[3] = {gx, gy, gz};
    if (fl & F_FORCED) {
      const Vec4<A> a = fcur[fslot[cell]];
      F[0] += double(a.x);
      F[1] += double(a.y);
      F[2] += double(a.z);
    }
    v[0] += 1.0;
    v[1] += s;
    v[2] += m0 + 0.5 * F[0];
    v[3] += m1 + 0.5 * F[1];
    v[4] += m2 + 0.5 * F[2];
  }
  block_sum<5>(v, sh);
  if (threadIdx.x == 0)
    for (int k = 0; k < 5; ++k) part[5 * blockIdx.x + k] = v[k];
}

// Sum block partials in block order (single thread: deterministic).
// clear_body_force_field on the device: *nonuniform |= any slot of the
// field differs from the base value (slot 0 when the slots cover every
// cell, else zero), compared component-wise like the host check.
template <class A>
__global__ void field_uniform_kernel(const Vec4<A>* f, int64_t nslots, int full, int* nonuniform) {
  const Vec4<A> base = full ? f[0] : Vec4<A>{A(0), A(0), A(0), A(0)};
  int local = 0;
  for (int64_t s = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; s < nslots; s += int64_t(gridDim.x) * blockDim.x) {
    const Vec4<A> v = f[s];
    if (!(v.x == base.x && v.y == base.y && v.z == base.z)) local = 1;
  }
  if (__syncthreads_or(local) && threadIdx.x == 0) atomicOr(nonuniform, 1);
}

// Zero the field whose value the cached moments hold, when the cleared
// field was uniform (flag from field_uniform_kernel).
template <class A>
__global__ void field_zero_if_uniform_kernel(Vec4<A>* f, int64_t nslots, const int* nonuniform) {
  if (*nonuniform) return;
  for (int64_t s = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; s < nslots; s += int64_t(gridDim.x) * blockDim.x)
    f[s] = Vec4<A>{A(0), A(0), A(0), A(0)};
}

static __global__ void reduce_finish_kernel(const double* part, int nblk, int width, double* out) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  for (int k = 0; k < width; ++k) {
    double s = 0.0;
    for (int b = 0; b < nblk; ++b) s += part[width * b + k];
    out[k] = s;
  }
}

}  // namespace lbmb
