// CPU oracle for the LBMFlow single-GPU time step (test infrastructure only).
//
// This header restates, operand for operand, the reference CPU path
// (lbm-core `CpuScalar` backend + `Solver` orchestration) that the CUDA
// library in lbmflow_b200/ accelerates. It is the CHECKER: only tests/,
// __graft_entry__.smoke() and bench.py's cpu_baseline / reference legs load
// it. Nothing in the product links against it.
//
// Parity is pinned by the reference's own known-answer tests restated in
// tests/test_oracle_kats.py (omega derivation, lattice invariants, bitwise
// equilibrium fixed point, central-moment rest/uniform invariance, scalar
// equilibrium moments, geometry volume/baffle/marker KATs, IBM slip/torque
// KATs, QOI formulas). The reference is Rust and cannot be compiled in this
// environment, so no binary-level comparison against it is possible.
//
// Citations are `path:line` inside the reference project.
#pragma once

#include <algorithm>
#include <array>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <stdexcept>
#include <string>
#include <vector>

namespace lbmo {

// ---------------------------------------------------------------------------
// Lattices (crates/lbm-core/src/lattice.rs:295-470). Direction order is the
// reference's and is load-bearing (OPP[q] == q±1, D3Q19 is a prefix of D3Q27).
// D3Q7 has no reference counterpart: rest + the six axis links (the first 7
// directions of D3Q19), w0 = 1/4, w1..6 = 1/8, cs^2 = 1/4.
// ---------------------------------------------------------------------------
struct D3Q19 {
  static constexpr int D = 3, Q = 19;
  static constexpr int8_t C[19][3] = {
      {0, 0, 0},  {1, 0, 0},  {-1, 0, 0}, {0, 1, 0},  {0, -1, 0}, {0, 0, 1},  {0, 0, -1},
      {1, 1, 0},  {-1, -1, 0}, {1, 0, 1}, {-1, 0, -1}, {0, 1, 1}, {0, -1, -1}, {1, -1, 0},
      {-1, 1, 0}, {1, 0, -1}, {-1, 0, 1}, {0, 1, -1}, {0, -1, 1}};
  static constexpr double W[19] = {
      1.0 / 3.0,  1.0 / 18.0, 1.0 / 18.0, 1.0 / 18.0, 1.0 / 18.0, 1.0 / 18.0, 1.0 / 18.0,
      1.0 / 36.0, 1.0 / 36.0, 1.0 / 36.0, 1.0 / 36.0, 1.0 / 36.0, 1.0 / 36.0, 1.0 / 36.0,
      1.0 / 36.0, 1.0 / 36.0, 1.0 / 36.0, 1.0 / 36.0, 1.0 / 36.0};
  // Scalar-ADE equilibrium factor 1/cs^2 (crates/lbm-core/src/scalar.rs:10-13).
  static constexpr double INV_CS2 = 3.0;
};

struct D3Q27 {
  static constexpr int D = 3, Q = 27;
  static constexpr int8_t C[27][3] = {
      {0, 0, 0},   {1, 0, 0},   {-1, 0, 0}, {0, 1, 0},   {0, -1, 0},  {0, 0, 1},   {0, 0, -1},
      {1, 1, 0},   {-1, -1, 0}, {1, 0, 1},  {-1, 0, -1}, {0, 1, 1},   {0, -1, -1}, {1, -1, 0},
      {-1, 1, 0},  {1, 0, -1},  {-1, 0, 1}, {0, 1, -1},  {0, -1, 1},  {1, 1, 1},   {-1, -1, -1},
      {1, 1, -1},  {-1, -1, 1}, {1, -1, 1}, {-1, 1, -1}, {1, -1, -1}, {-1, 1, 1}};
  static constexpr double W[27] = {
      8.0 / 27.0,  2.0 / 27.0,  2.0 / 27.0,  2.0 / 27.0,  2.0 / 27.0,  2.0 / 27.0,  2.0 / 27.0,
      1.0 / 54.0,  1.0 / 54.0,  1.0 / 54.0,  1.0 / 54.0,  1.0 / 54.0,  1.0 / 54.0,  1.0 / 54.0,
      1.0 / 54.0,  1.0 / 54.0,  1.0 / 54.0,  1.0 / 54.0,  1.0 / 54.0,  1.0 / 216.0, 1.0 / 216.0,
      1.0 / 216.0, 1.0 / 216.0, 1.0 / 216.0, 1.0 / 216.0, 1.0 / 216.0, 1.0 / 216.0};
  static constexpr double INV_CS2 = 3.0;
};

struct D3Q7 {
  static constexpr int D = 3, Q = 7;
  static constexpr int8_t C[7][3] = {{0, 0, 0}, {1, 0, 0},  {-1, 0, 0}, {0, 1, 0},
                                     {0, -1, 0}, {0, 0, 1}, {0, 0, -1}};
  static constexpr double W[7] = {0.25, 0.125, 0.125, 0.125, 0.125, 0.125, 0.125};
  static constexpr double INV_CS2 = 4.0;
};

constexpr int Q_MAX = 27;

// OPP and TRT pairs derived from C exactly as lattice.rs:158-212 does.
template <class L>
struct Tables {
  int opp[L::Q];
  int npairs = 0;
  int pa[L::Q], pb[L::Q];
  Tables() {
    for (int q = 0; q < L::Q; ++q) {
      opp[q] = -1;
      for (int r = 0; r < L::Q; ++r)
        if (L::C[r][0] == -L::C[q][0] && L::C[r][1] == -L::C[q][1] && L::C[r][2] == -L::C[q][2])
          opp[q] = r;
    }
    for (int q = 0; q < L::Q; ++q)
      if (q != 0 && q < opp[q]) {
        pa[npairs] = q;
        pb[npairs] = opp[q];
        ++npairs;
      }
  }
};
template <class L>
inline const Tables<L>& tables() {
  static const Tables<L> t;
  return t;
}

// ---------------------------------------------------------------------------
// Step parameters (crates/lbm-core/src/params.rs).
// ---------------------------------------------------------------------------
enum CollisionKind { BGK = 0, TRT = 1, CENTRAL_MOMENT = 2 };
constexpr double MAGIC_STD = 3.0 / 16.0;  // params.rs:202
constexpr double MAX_SPEED = 0.3;         // params.rs:11

// CollisionKind::omegas (params.rs:205-217).
inline void omegas(int kind, double magic, double nu, double* op, double* om) {
  double tau = 3.0 * nu + 0.5;
  double omega_p = 1.0 / tau;
  double omega_m = omega_p;
  if (kind == TRT) {
    double lam_p = tau - 0.5;
    omega_m = 1.0 / (magic / lam_p + 0.5);
  }
  *op = omega_p;
  *om = omega_m;
}

template <class T>
struct KParams {  // params.rs:322-374
  bool central_moment = false;
  T omega_p, omega_m, omega_shear, cp, cm;
  T force[3];
  T cr[Q_MAX][3];
  T wr[Q_MAX];
};

struct StepParams {  // params.rs:302-320 (subset on the hot path)
  int collision = TRT;
  double magic = MAGIC_STD;
  double omega_shear_cfg = 0.0;  // CentralMoment { omega_shear }
  double omega_p = 1.0, omega_m = 1.0;
  double nu = 1.0 / 6.0;
  double force[3] = {0, 0, 0};
  // Smagorinsky constant (0: off). Not a reference feature: an optional
  // subgrid model of the device library that is restated here so the
  // device path stays checkable with it switched on.
  double smagorinsky_cs = 0.0;
  // Free-slip (specular) top wall: the solid layer z = nz - 1 reflects a
  // population (cx, cy, +1) leaving cell x into (cx, cy, -1) at x + (cx,
  // cy, 0) when that cell is fluid (bounce-back otherwise). Not a reference
  // feature; restated here so the device path stays checkable with it on.
  bool free_slip_top = false;
  // 16-bit population storage (0: off, 1: binary16, 2: bfloat16): every
  // population the step writes is rounded to the 16-bit format (nearest,
  // ties to even) in deviation form, as a device that stores f_i - w_i in 16
  // bits and computes in fp32 (the reference's wgpu f16 design,
  // crates/lbm-core/src/gpu/wgsl.rs:231-243, gpu/backend.rs:160-229).
  int store16 = 0;
};

// ---------------------------------------------------------------------------
// 16-bit storage codecs.
// The reference's host codec (crates/lbm-core/src/gpu/backend.rs:160-213):
// f32 -> binary16 keeps the top 10 mantissa bits and adds one when the
// first dropped bit is set (nearest, ties away from zero), flushes
// magnitudes below 2^-25 to a signed zero, builds subnormals by shifting the
// implicit-bit mantissa, and saturates exponents >= 31 to infinity (NaN
// included). Decoding is exact.
// ---------------------------------------------------------------------------
inline uint16_t f32_to_f16_bits(float value) {
  uint32_t x;
  std::memcpy(&x, &value, 4);
  const uint16_t sign = uint16_t((x >> 16) & 0x8000u);
  const int32_t exp = int32_t((x >> 23) & 0xffu) - 127 + 15;
  const uint32_t mant = x & 0x7fffffu;
  if (exp <= 0) {
    if (exp < -10) return sign;
    const uint32_t m = mant | 0x800000u;
    const uint32_t shift = uint32_t(14 - exp);
    uint16_t half = uint16_t(m >> shift);
    if (((m >> (shift - 1)) & 1u) != 0) half = uint16_t(half + 1);
    return uint16_t(sign | half);
  }
  if (exp >= 31) return uint16_t(sign | 0x7c00u);
  uint16_t half = uint16_t(sign | (uint16_t(exp) << 10) | uint16_t(mant >> 13));
  if ((mant & 0x1000u) != 0) half = uint16_t(half + 1);
  return half;
}

inline float f16_bits_to_f32(uint16_t bits) {
  const uint32_t sign = uint32_t(bits & 0x8000u) << 16;
  const uint32_t exp = (bits >> 10) & 0x1fu;
  const uint32_t mant = bits & 0x03ffu;
  uint32_t out;
  if (exp == 0) {
    if (mant == 0) {
      out = sign;
    } else {
      uint32_t m = mant;
      int32_t e = -14;
      while ((m & 0x400u) == 0) {
        m <<= 1;
        e -= 1;
      }
      m &= 0x3ffu;
      out = sign | (uint32_t(e + 127) << 23) | (m << 13);
    }
  } else if (exp == 31) {
    out = sign | 0x7f800000u | (mant << 13);
  } else {
    out = sign | ((exp - 15 + 127) << 23) | (mant << 13);
  }
  float f;
  std::memcpy(&f, &out, 4);
  return f;
}

// Round to the nearest binary16 value, ties to even (the device-side f16()
// store of the fused step); finite inputs only on this path.
inline float round_f16_rne(float v) { return float(_Float16(v)); }

// Round to the nearest bfloat16 value, ties to even (top 16 bits of the
// binary32 pattern after adding 0x7fff plus the lowest kept bit).
inline float round_bf16_rne(float v) {
  uint32_t x;
  std::memcpy(&x, &v, 4);
  if ((x & 0x7fffffffu) > 0x7f800000u) return v;  // NaN stays NaN
  x += 0x7fffu + ((x >> 16) & 1u);
  x &= 0xffff0000u;
  float f;
  std::memcpy(&f, &x, 4);
  return f;
}

// The stored value of a population in the given 16-bit mode (1: binary16,
// 2: bfloat16).
inline float store16_round(int mode, float v) { return mode == 1 ? round_f16_rne(v) : round_bf16_rne(v); }
// Host staging of a population into 16-bit storage: the reference's codec
// for binary16, nearest-even for bfloat16 (no reference codec).
inline float stage16(int mode, float v) {
  return mode == 1 ? f16_bits_to_f32(f32_to_f16_bits(v)) : round_bf16_rne(v);
}

template <class L, class T>
KParams<T> make_kparams(const StepParams& p) {  // KParams::new, params.rs:350-374
  KParams<T> k{};
  for (int q = 0; q < L::Q; ++q) {
    for (int a = 0; a < 3; ++a) k.cr[q][a] = T(double(L::C[q][a]));
    k.wr[q] = T(L::W[q]);
  }
  k.central_moment = (p.collision == CENTRAL_MOMENT);
  k.omega_p = T(p.omega_p);
  k.omega_m = T(p.omega_m);
  k.omega_shear = T(p.collision == CENTRAL_MOMENT ? p.omega_shear_cfg : p.omega_p);
  k.cp = T(1.0 - p.omega_p / 2.0);
  k.cm = T(1.0 - p.omega_m / 2.0);
  for (int a = 0; a < 3; ++a) k.force[a] = T(p.force[a]);
  return k;
}

// ---------------------------------------------------------------------------
// Equilibrium in deviation form (kernels.rs:103-121).
// ---------------------------------------------------------------------------
template <class L, class T>
inline void equilibrium(const KParams<T>& p, T r, const T u[3], T* feq) {
  const T three = T(3.0), f45 = T(4.5), f15 = T(1.5);
  T usq = u[0] * u[0];
  for (int d = 1; d < L::D; ++d) usq = usq + u[d] * u[d];
  T drho = r - T(1.0);
  for (int q = 0; q < L::Q; ++q) {
    T cu = p.cr[q][0] * u[0];
    for (int d = 1; d < L::D; ++d) cu = cu + p.cr[q][d] * u[d];
    feq[q] = p.wr[q] * (drho + r * (three * cu + f45 * cu * cu - f15 * usq));
  }
}

// ---------------------------------------------------------------------------
// TRT + Guo collision for one cell (collision.rs:81-202 through
// kernels.rs:129-160). `f` points at population q of this cell at f[q*np].
// ---------------------------------------------------------------------------
template <class L, class T>
inline void collide_trt_cell(T* f, size_t np, T rho, const T u[3], const T fv[3], T op, T cp,
                             bool force_on, const KParams<T>& k) {
  const auto& tb = tables<L>();
  const T half = T(0.5);
  auto cval = [&](int q, int d) { return T(double(int8_t(double(k.cr[q][d])))); };
  auto wval = [&](int q) { return T(double(k.wr[q])); };
  auto dot_u = [&](int q) {
    T acc = cval(q, 0) * u[0];
    for (int d = 1; d < L::D; ++d) acc = acc + cval(q, d) * u[d];
    return acc;
  };
  auto dot_f = [&](int q) {
    T acc = cval(q, 0) * fv[0];
    for (int d = 1; d < L::D; ++d) acc = acc + cval(q, d) * fv[d];
    return acc;
  };
  T usq = u[0] * u[0];
  for (int d = 1; d < L::D; ++d) usq = usq + u[d] * u[d];
  T uf = u[0] * fv[0];
  for (int d = 1; d < L::D; ++d) uf = uf + u[d] * fv[d];
  T feq[Q_MAX], src[Q_MAX];
  for (int q = 0; q < L::Q; ++q) {
    T cu = dot_u(q);
    {  // SecondOrderEq::feq (collision.rs:81-102)
      T cu2 = dot_u(q);
      T drho = rho - T(1.0);
      T three_cu = T(3.0) * cu2;
      T f45_cu = T(4.5) * cu2;
      T f45_cu2 = f45_cu * cu2;
      T f15_usq = T(1.5) * usq;
      T sum = three_cu + f45_cu2;
      T inner = sum - f15_usq;
      T rho_inner = rho * inner;
      T body = drho + rho_inner;
      feq[q] = wval(q) * body;
    }
    if (!force_on) {  // GuoForcing::source (collision.rs:104-121)
      src[q] = T(0.0);
    } else {
      T cf = dot_f(q);
      T cf_minus_uf = cf - uf;
      T first = T(3.0) * cf_minus_uf;
      T nine_cu = T(9.0) * cu;
      T second = nine_cu * cf;
      T body = first + second;
      src[q] = wval(q) * body;
    }
  }
  {  // rest population (collision.rs:149-158)
    T f0 = f[0];
    T f0_minus_e = f0 - feq[0];
    T op_delta = op * f0_minus_e;
    T relaxed = f0 - op_delta;
    T cp_src = cp * src[0];
    f[0] = relaxed + cp_src;
  }
  for (int pi = 0; pi < tb.npairs; ++pi) {  // collision.rs:160-200
    int qa = tb.pa[pi], qb = tb.pb[pi];
    T fa = f[qa * np], fb = f[qb * np];
    T fp = half * (fa + fb);
    T fm = half * (fa - fb);
    T ep = half * (feq[qa] + feq[qb]);
    T em = half * (feq[qa] - feq[qb]);
    T sp = half * (src[qa] + src[qb]);
    T sm = half * (src[qa] - src[qb]);
    T rp = op * (fp - ep);
    T rm = k.omega_m * (fm - em);
    T cp_sp = cp * sp;
    T cm_sm = k.cm * sm;
    T va = ((fa - rp) - rm) + (cp_sp + cm_sm);
    T vb = ((fb - rp) + rm) + (cp_sp - cm_sm);
    f[qa * np] = va;
    f[qb * np] = vb;
  }
}

// ---------------------------------------------------------------------------
// Central-moment collision (kernels.rs:162-533): dense f64 transforms exactly
// as the reference builds them (basis order, Gauss-Jordan inverse with
// partial pivoting, binomial shift), applied per cell in f64 then cast to T.
// ---------------------------------------------------------------------------
struct MomentTransform {
  int q = 0;
  uint8_t basis[Q_MAX][3];
  int exp_index[3][3][3];
  double raw_from_pop[Q_MAX][Q_MAX];
  double pop_from_raw[Q_MAX][Q_MAX];
};

template <class L>
inline MomentTransform build_moment_transform() {  // kernels.rs:162-282
  MomentTransform t{};
  t.q = L::Q;
  int n = 0;
  for (int ax = 0; ax <= 2; ++ax)
    for (int ay = 0; ay <= 2; ++ay)
      for (int az = 0; az <= 2; ++az) {
        if (L::Q == 19 && ax > 0 && ay > 0 && az > 0) continue;
        if (n < L::Q) {
          t.basis[n][0] = uint8_t(ax);
          t.basis[n][1] = uint8_t(ay);
          t.basis[n][2] = uint8_t(az);
          ++n;
        }
      }
  for (int a = 0; a < 3; ++a)
    for (int b = 0; b < 3; ++b)
      for (int c = 0; c < 3; ++c) t.exp_index[a][b][c] = -1;
  auto pw = [](double x, int e) { return e == 0 ? 1.0 : (e == 1 ? x : x * x); };
  for (int m = 0; m < L::Q; ++m) {
    const uint8_t* e = t.basis[m];
    t.exp_index[e[0]][e[1]][e[2]] = m;
    for (int q = 0; q < L::Q; ++q) {
      double v = pw(double(L::C[q][0]), e[0]);
      v *= pw(double(L::C[q][1]), e[1]);
      v *= pw(double(L::C[q][2]), e[2]);
      t.raw_from_pop[m][q] = v;
    }
  }
  // invert_raw_moment_matrix (kernels.rs:223-266)
  const int N = L::Q;
  double a[Q_MAX][2 * Q_MAX];
  for (int r = 0; r < N; ++r) {
    for (int c = 0; c < 2 * N; ++c) a[r][c] = 0.0;
    for (int c = 0; c < N; ++c) a[r][c] = t.raw_from_pop[r][c];
    a[r][N + r] = 1.0;
  }
  for (int col = 0; col < N; ++col) {
    int pivot = col;
    for (int row = col + 1; row < N; ++row)
      if (std::fabs(a[row][col]) > std::fabs(a[pivot][col])) pivot = row;
    if (!(std::fabs(a[pivot][col]) > 1.0e-14)) throw std::runtime_error("singular raw-moment basis");
    if (pivot != col)
      for (int j = 0; j < 2 * N; ++j) std::swap(a[pivot][j], a[col][j]);
    double inv = 1.0 / a[col][col];
    for (int j = col; j < 2 * N; ++j) a[col][j] *= inv;
    for (int row = 0; row < N; ++row) {
      if (row == col) continue;
      double factor = a[row][col];
      if (factor == 0.0) continue;
      for (int j = col; j < 2 * N; ++j) a[row][j] -= factor * a[col][j];
    }
  }
  for (int r = 0; r < N; ++r)
    for (int c = 0; c < N; ++c) t.pop_from_raw[r][c] = a[r][N + c];
  return t;
}

template <class L>
inline const MomentTransform& moment_transform() {
  static const MomentTransform t = build_moment_transform<L>();
  return t;
}

// shifted_moments (kernels.rs:311-346)
inline void shifted_moments(const MomentTransform& t, const double u[3], const double* in,
                            bool raw_to_central, double* out) {
  auto pw = [](double x, int e) { return e == 0 ? 1.0 : (e == 1 ? x : x * x); };
  auto binom = [](int n, int k) {
    if (k == 0) return 1.0;
    if (n == 1 && k == 1) return 1.0;
    if (n == 2 && k == 1) return 2.0;
    return 1.0;  // (2,2)
  };
  for (int m = 0; m < t.q; ++m) {
    const uint8_t* e = t.basis[m];
    double acc = 0.0;
    for (int kx = 0; kx <= e[0]; ++kx)
      for (int ky = 0; ky <= e[1]; ++ky)
        for (int kz = 0; kz <= e[2]; ++kz) {
          int idx = t.exp_index[kx][ky][kz];
          double coef = binom(e[0], kx) * binom(e[1], ky) * binom(e[2], kz);
          double sx = raw_to_central ? -u[0] : u[0];
          double sy = raw_to_central ? -u[1] : u[1];
          double sz = raw_to_central ? -u[2] : u[2];
          coef *= pw(sx, e[0] - kx);
          coef *= pw(sy, e[1] - ky);
          coef *= pw(sz, e[2] - kz);
          acc += coef * in[idx];
        }
    out[m] = acc;
  }
}

inline void pops_to_central(const MomentTransform& t, const double u[3], const double* pops,
                            double* out) {  // kernels.rs:296-309
  double raw[Q_MAX];
  for (int m = 0; m < t.q; ++m) {
    raw[m] = 0.0;
    for (int q = 0; q < t.q; ++q) raw[m] += t.raw_from_pop[m][q] * pops[q];
  }
  shifted_moments(t, u, raw, true, out);
}

template <class L, class T>
inline void collide_cm_cell(T* f, size_t np, T rho_t, const T ut[3], const T fv_t[3],
                            const KParams<T>& k) {  // kernels.rs:406-533
  const MomentTransform& tr = moment_transform<L>();
  double r = double(rho_t);
  double u[3] = {double(ut[0]), double(ut[1]), double(ut[2])};
  double fv[3] = {double(fv_t[0]), double(fv_t[1]), double(fv_t[2])};
  bool force_on = fv[0] != 0.0 || fv[1] != 0.0 || fv[2] != 0.0;
  double phys[Q_MAX], src[Q_MAX];
  bool feq_rest = (u[0] == 0.0 && u[1] == 0.0 && u[2] == 0.0) && !force_on;
  bool exact_rest = feq_rest;
  for (int q = 0; q < L::Q; ++q) {
    T fq = f[q * np];
    phys[q] = double(fq) + L::W[q];
    src[q] = 0.0;
    if (exact_rest) {
      T expected = T(L::W[q] * (r - 1.0));
      double a = double(fq), b = double(expected);
      exact_rest = exact_rest && (std::memcmp(&a, &b, sizeof(double)) == 0);
    }
  }
  if (exact_rest) return;
  if (force_on) {
    double uf = u[0] * fv[0];
    for (int d = 1; d < L::D; ++d) uf += u[d] * fv[d];
    for (int q = 0; q < L::Q; ++q) {
      double cu = double(L::C[q][0]) * u[0];
      double cf = double(L::C[q][0]) * fv[0];
      for (int d = 1; d < L::D; ++d) {
        cu += double(L::C[q][d]) * u[d];
        cf += double(L::C[q][d]) * fv[d];
      }
      src[q] = L::W[q] * (3.0 * (cf - uf) + 9.0 * cu * cf);
    }
  }
  double usq = u[0] * u[0];
  for (int d = 1; d < L::D; ++d) usq += u[d] * u[d];
  double feq_phys[Q_MAX];
  for (int q = 0; q < L::Q; ++q) {
    double cu = double(L::C[q][0]) * u[0];
    for (int d = 1; d < L::D; ++d) cu += double(L::C[q][d]) * u[d];
    feq_phys[q] = L::W[q] * r * (1.0 + 3.0 * cu + 4.5 * cu * cu - 1.5 * usq);
  }
  double mom[Q_MAX], eq[Q_MAX], smom[Q_MAX];
  pops_to_central(tr, u, phys, mom);
  pops_to_central(tr, u, feq_phys, eq);
  pops_to_central(tr, u, src, smom);
  double os_base = double(k.omega_shear);
  double usq3 = u[0] * u[0] + u[1] * u[1] + u[2] * u[2];
  double vc = -0.16 * usq3;
  double os = std::min(os_base * (1.0 + vc), 2.0);
  double post[Q_MAX];
  int diag[3] = {-1, -1, -1};
  for (int m = 0; m < L::Q; ++m) {
    const uint8_t* e = tr.basis[m];
    int order = e[0] + e[1] + e[2];
    if (order == 2)
      for (int a = 0; a < L::D; ++a) {
        uint8_t de[3] = {0, 0, 0};
        de[a] = 2;
        if (e[0] == de[0] && e[1] == de[1] && e[2] == de[2]) diag[a] = m;
      }
    double rate = (order <= 1) ? 0.0 : (order == 2 ? os : 1.0);
    post[m] = mom[m] - rate * (mom[m] - eq[m]) + (1.0 - 0.5 * rate) * smom[m];
  }
  double inv_d = 1.0 / double(L::D);
  double trace_neq = 0.0, trace_src = 0.0;
  for (int a = 0; a < L::D; ++a) {
    trace_neq += mom[diag[a]] - eq[diag[a]];
    trace_src += smom[diag[a]];
  }
  double bulk_neq = trace_neq * inv_d, bulk_src = trace_src * inv_d;
  for (int a = 0; a < L::D; ++a) {
    int idx = diag[a];
    double dev_neq = mom[idx] - eq[idx] - bulk_neq;
    double dev_src = smom[idx] - bulk_src;
    post[idx] = eq[idx] + (1.0 - os) * dev_neq + 0.5 * bulk_src + (1.0 - 0.5 * os) * dev_src;
  }
  double raw_post[Q_MAX];
  shifted_moments(tr, u, post, false, raw_post);
  for (int q = 0; q < L::Q; ++q) {
    double o = 0.0;
    for (int m = 0; m < L::Q; ++m) o += tr.pop_from_raw[q][m] * raw_post[m];
    f[q * np] = T(o - L::W[q]);
  }
}

// ---------------------------------------------------------------------------
// Direct-forcing IBM support (crates/lbm-core/src/rotating_ibm.rs).
// ---------------------------------------------------------------------------
struct IbmConfig {  // DirectForcingConfig (rotating_ibm.rs:106-130)
  int max_iterations = 3;
  double slip_tolerance = 1.0e-2;
  int kernel_radius = 1;
  double relaxation = 1.0;
};

struct IbmDiag {  // IbmDiagnostics (rotating_ibm.rs:134-153)
  int iterations = 0;
  double slip_max = 0, slip_rms = 0, slip_max_rel = 0, slip_rms_rel = 0;
  double torque[3] = {0, 0, 0};
  double fluid_force[3] = {0, 0, 0};
  double marker_force[3] = {0, 0, 0};
  double momentum_error_rel = 0;
};

struct StencilPoint {
  int x, y, z;
  double w;
};

inline double linear_kernel(double r) { return std::max(1.0 - r, 0.0); }  // rotating_ibm.rs:212
inline double quadratic_kernel(double r) {                                 // rotating_ibm.rs:216
  if (r < 0.5) return 0.75 - r * r;
  if (r < 1.5) return 0.5 * (1.5 - r) * (1.5 - r);
  return 0.0;
}

// marker_stencil (rotating_ibm.rs:163-210): clipped tensor stencil, cell
// order x outer, z inner.
inline std::vector<StencilPoint> marker_stencil(const double p[3], const int dims[3], int d,
                                                int radius) {
  if (radius != 1 && radius != 2) throw std::runtime_error("IBM kernel radius must be 1 or 2");
  std::vector<std::pair<int, double>> axes[3];
  for (int a = 0; a < 3; ++a) {
    if (a >= d) {
      axes[a].push_back({0, 1.0});
      continue;
    }
    long lo = long(std::floor(p[a])) - radius + 1;
    long hi = long(std::floor(p[a])) + radius;
    for (long i = lo; i <= hi; ++i) {
      if (i < 0 || i >= dims[a]) continue;
      double r = std::fabs(p[a] - double(i));
      double w = radius == 1 ? linear_kernel(r) : quadratic_kernel(r);
      if (w != 0.0) axes[a].push_back({int(i), w});
    }
  }
  std::vector<StencilPoint> out;
  for (auto& ax : axes[0])
    for (auto& ay : axes[1])
      for (auto& az : axes[2]) out.push_back({ax.first, ay.first, az.first, ax.second * ay.second * az.second});
  return out;
}

inline double norm3(const double v[3], int d) {
  double s = 0.0;
  for (int i = 0; i < d; ++i) s += v[i] * v[i];
  return std::sqrt(s);
}

struct Body {  // RotatingBody (rotating_ibm.rs:24-102)
  double center[3];
  double omega[3];
  std::vector<double> pos;  // n x 3
  std::vector<double> weight;
  size_t n() const { return weight.size(); }
  void target(const double* p, double out[3]) const {
    double r[3] = {p[0] - center[0], p[1] - center[1], p[2] - center[2]};
    out[0] = omega[1] * r[2] - omega[2] * r[1];
    out[1] = omega[2] * r[0] - omega[0] * r[2];
    out[2] = omega[0] * r[1] - omega[1] * r[0];
  }
};

// The force-update core of Solver::apply_rotating_ibm (solver.rs:3093-3253),
// over compact global arrays: rho (f64 view of the cached T density), u_now
// (f64). Writes the accumulated f64 spread (n x 3, zero-initialised by the
// caller) and returns the diagnostics.
inline IbmDiag ibm_direct_forcing(const int dims[3], int d, const uint8_t* solid,
                                  const double* rho, const double* u_now, const Body& body,
                                  const IbmConfig& cfg, double* spread) {
  if (cfg.max_iterations <= 0) throw std::runtime_error("IBM max_iterations must be positive");
  if (!(cfg.slip_tolerance >= 0.0 && std::isfinite(cfg.slip_tolerance)))
    throw std::runtime_error("IBM slip_tolerance must be finite and non-negative");
  if (!(cfg.relaxation > 0.0 && cfg.relaxation <= 1.0))
    throw std::runtime_error("IBM relaxation must be finite and in (0, 1]");
  const size_t n = size_t(dims[0]) * dims[1] * dims[2];
  auto gidx = [&](const StencilPoint& sp) { return (size_t(sp.z) * dims[1] + sp.y) * dims[0] + sp.x; };
  std::vector<double> du(3 * n, 0.0);
  IbmDiag diag;
  double max_target = 0.0;
  const size_t nm = body.n();
  for (size_t m = 0; m < nm; ++m) {
    double t[3];
    body.target(&body.pos[3 * m], t);
    max_target = std::max(max_target, norm3(t, d));
  }
  double scale = std::max(max_target, 1.0);
  std::vector<std::vector<StencilPoint>> st(nm);
  for (size_t m = 0; m < nm; ++m) {
    st[m] = marker_stencil(&body.pos[3 * m], dims, d, cfg.kernel_radius);
    if (st[m].empty()) throw std::runtime_error("IBM marker stencil is outside the domain");
  }
  std::vector<double> cks(n, 0.0);
  for (size_t m = 0; m < nm; ++m)
    for (auto& sp : st[m]) {
      size_t gi = gidx(sp);
      if (solid[gi]) continue;
      cks[gi] += sp.w;
    }
  std::vector<double> imp(3 * nm);
  for (int iter = 0; iter < cfg.max_iterations; ++iter) {
    std::fill(imp.begin(), imp.end(), 0.0);
    for (size_t m = 0; m < nm; ++m) {
      double target[3];
      body.target(&body.pos[3 * m], target);
      double um[3] = {0, 0, 0};
      double mobility = 0.0;
      for (auto& sp : st[m]) {
        size_t gi = gidx(sp);
        if (solid[gi]) continue;
        double rc = rho[gi];
        um[0] += sp.w * (u_now[3 * gi + 0] + du[3 * gi + 0]);
        um[1] += sp.w * (u_now[3 * gi + 1] + du[3 * gi + 1]);
        um[2] += sp.w * (u_now[3 * gi + 2] + du[3 * gi + 2]);
        mobility += sp.w * cks[gi] / std::max(rc, 1.0e-30);
      }
      if (mobility == 0.0) continue;
      double slip[3] = {target[0] - um[0], target[1] - um[1], target[2] - um[2]};
      for (int a = 0; a < 3; ++a) imp[3 * m + a] = cfg.relaxation * slip[a] / mobility;
    }
    for (size_t m = 0; m < nm; ++m) {
      double rmf[3] = {0, 0, 0};
      for (auto& sp : st[m]) {
        size_t gi = gidx(sp);
        if (solid[gi]) continue;
        double cf[3] = {imp[3 * m + 0] * sp.w, imp[3 * m + 1] * sp.w, imp[3 * m + 2] * sp.w};
        for (int a = 0; a < 3; ++a) {
          spread[3 * gi + a] += cf[a];
          diag.fluid_force[a] += cf[a];
          rmf[a] += cf[a];
        }
        double inv_rho = 1.0 / std::max(rho[gi], 1.0e-30);
        for (int a = 0; a < 3; ++a) du[3 * gi + a] += cf[a] * inv_rho;
      }
      for (int a = 0; a < 3; ++a) diag.marker_force[a] += rmf[a];
      const double* p = &body.pos[3 * m];
      double r[3] = {p[0] - body.center[0], p[1] - body.center[1], p[2] - body.center[2]};
      double tq[3] = {r[1] * rmf[2] - r[2] * rmf[1], r[2] * rmf[0] - r[0] * rmf[2],
                      r[0] * rmf[1] - r[1] * rmf[0]};
      for (int a = 0; a < 3; ++a) diag.torque[a] -= tq[a];
    }
    diag.iterations = iter + 1;
    diag.slip_max = 0.0;
    double slip_sq_w = 0.0, w_sum = 0.0;
    for (size_t m = 0; m < nm; ++m) {
      double target[3];
      body.target(&body.pos[3 * m], target);
      double um[3] = {0, 0, 0};
      bool active = false;
      for (auto& sp : st[m]) {
        size_t gi = gidx(sp);
        if (solid[gi]) continue;
        active = true;
        um[0] += sp.w * (u_now[3 * gi + 0] + du[3 * gi + 0]);
        um[1] += sp.w * (u_now[3 * gi + 1] + du[3 * gi + 1]);
        um[2] += sp.w * (u_now[3 * gi + 2] + du[3 * gi + 2]);
      }
      if (!active) continue;
      double slip[3] = {target[0] - um[0], target[1] - um[1], target[2] - um[2]};
      double sm = norm3(slip, d);
      diag.slip_max = std::max(diag.slip_max, sm);
      slip_sq_w += body.weight[m] * sm * sm;
      w_sum += body.weight[m];
    }
    diag.slip_rms = w_sum > 0.0 ? std::sqrt(slip_sq_w / w_sum) : 0.0;
    diag.slip_max_rel = diag.slip_max / scale;
    diag.slip_rms_rel = diag.slip_rms / scale;
    double err[3] = {diag.fluid_force[0] - diag.marker_force[0],
                     diag.fluid_force[1] - diag.marker_force[1],
                     diag.fluid_force[2] - diag.marker_force[2]};
    diag.momentum_error_rel = norm3(err, d) / std::max(norm3(diag.marker_force, d), 1.0e-12);
    if (diag.slip_max_rel <= cfg.slip_tolerance) break;
  }
  return diag;
}

// ---------------------------------------------------------------------------
// Solver: single-part CpuScalar orchestration over compact arrays.
// Periodic axes wrap by index arithmetic, which is what the single-part
// LocalPeriodic halo provides (halo.rs:77-104).
// ---------------------------------------------------------------------------
enum ReductionKind { RED_FLUID_CELLS = 0, RED_MASS_DEV = 1, RED_MOMENTUM = 2 };

template <class T>
struct Scalar {  // fields.rs:39-70
  int q = 0;                // scalar lattice size (7, 19 or 27)
  double diffusivity = 0.0;
  std::vector<T> h, htmp, conc;
};

template <class L, class T>
class Solver {
 public:
  int dims[3];
  bool periodic[3];
  size_t n;
  StepParams params;
  KParams<T> kp;
  std::vector<T> f, ftmp;
  std::vector<T> rho, ux, uy, uz;
  std::vector<uint8_t> solid;
  std::vector<T> wall_u;  // n x 3
  bool has_force_field = false;
  std::vector<T> force_field;  // n x 3
  // Per-cell relaxation field (Solver::set_omega_field, solver.rs:4443-4473):
  // TRT takes omega+ = field, c+ = 1 - omega+/2 (omega- unchanged,
  // kernels.rs:151-156); the central moment takes its shear rate from it
  // (kernels.rs:481).
  bool has_omega_field = false;
  std::vector<T> omega_field;
  std::vector<Scalar<T>> scalars;
  uint64_t time = 0;

  // Solver::build (solver.rs:1754-1900): quiescent f = 0, rho = 1, u = 0,
  // then one update_moments.
  Solver(const int d[3], const bool per[3], const StepParams& p, const uint8_t* solid_in,
         const double* wall_u_in) {
    for (int a = 0; a < 3; ++a) {
      dims[a] = d[a];
      periodic[a] = per[a];
    }
    n = size_t(d[0]) * d[1] * d[2];
    params = p;
    kp = make_kparams<L, T>(params);
    f.assign(L::Q * n, T(0));
    ftmp.assign(L::Q * n, T(0));
    rho.assign(n, T(1));
    ux.assign(n, T(0));
    uy.assign(n, T(0));
    uz.assign(n, T(0));
    solid.assign(n, 0);
    wall_u.assign(3 * n, T(0));
    if (solid_in)
      for (size_t i = 0; i < n; ++i) solid[i] = solid_in[i] ? 1 : 0;
    if (wall_u_in)
      for (size_t i = 0; i < 3 * n; ++i) wall_u[i] = T(wall_u_in[i]);
    update_moments();
  }

  size_t idx(long x, long y, long z) const { return (size_t(z) * dims[1] + size_t(y)) * dims[0] + size_t(x); }

  void force_at(size_t c, T out[3]) const {  // KParams::force_at, params.rs:386-405
    if (has_force_field) {
      for (int a = 0; a < 3; ++a) out[a] = kp.force[a] + force_field[3 * c + a];
    } else {
      for (int a = 0; a < 3; ++a) out[a] = kp.force[a];
    }
  }
  bool force_on() const {
    return kp.force[0] != T(0) || kp.force[1] != T(0) || kp.force[2] != T(0) || has_force_field;
  }

  void collide() {  // CpuScalar::collide (backend.rs:417-474)
    bool fon = force_on();
    const bool les = params.smagorinsky_cs > 0.0;
#pragma omp parallel for schedule(static)
    for (long c = 0; c < long(n); ++c) {
      if (solid[c]) continue;
      T u[3] = {ux[c], uy[c], uz[c]};
      T fv[3];
      force_at(size_t(c), fv);
      if (has_omega_field) {
        const T op = omega_field[c];
        if (kp.central_moment) {
          KParams<T> kc = kp;
          kc.omega_shear = op;
          collide_cm_cell<L, T>(&f[c], n, rho[c], u, fv, kc);
        } else {
          collide_trt_cell<L, T>(&f[c], n, rho[c], u, fv, op, T(1) - op / T(2.0), fon, kp);
        }
        continue;
      }
      if (les) {
        const KParams<T> kc = les_kparams(&f[c], rho[c], u);
        if (kc.central_moment)
          collide_cm_cell<L, T>(&f[c], n, rho[c], u, fv, kc);
        else
          collide_trt_cell<L, T>(&f[c], n, rho[c], u, fv, kc.omega_p, kc.cp, fon, kc);
        continue;
      }
      if (kp.central_moment)
        collide_cm_cell<L, T>(&f[c], n, rho[c], u, fv, kp);
      else
        collide_trt_cell<L, T>(&f[c], n, rho[c], u, fv, kp.omega_p, kp.cp, fon, kp);
    }
  }

  // Smagorinsky-adjusted rates of one cell: Pi_neq from the second moments
  // of the deviation populations, Pi_neq = sum c c f_dev - (rho - 1)/3 I -
  // rho u u; tau_eff = (tau0 + sqrt(tau0^2 + 18 sqrt(2) Cs^2 |Pi_neq| /
  // rho)) / 2; TRT keeps its magic parameter, BGK and the central-moment
  // shear rate take omega = 1 / tau_eff.
  KParams<T> les_kparams(const T* fc, T rho_c, const T u[3]) const {
    T s[6] = {T(0), T(0), T(0), T(0), T(0), T(0)};  // xx yy zz xy xz yz
    for (int q = 1; q < L::Q; ++q) {
      const int cx = L::C[q][0], cy = L::C[q][1], cz = L::C[q][2];
      const T fq = fc[size_t(q) * n];
      if (cx) s[0] = s[0] + fq;
      if (cy) s[1] = s[1] + fq;
      if (cz) s[2] = s[2] + fq;
      if (cx && cy) s[3] = cx * cy > 0 ? s[3] + fq : s[3] - fq;
      if (cx && cz) s[4] = cx * cz > 0 ? s[4] + fq : s[4] - fq;
      if (cy && cz) s[5] = cy * cz > 0 ? s[5] + fq : s[5] - fq;
    }
    const T d3 = (rho_c - T(1)) * T(1.0 / 3.0);
    const T pxx = s[0] - d3 - rho_c * u[0] * u[0], pyy = s[1] - d3 - rho_c * u[1] * u[1];
    const T pzz = s[2] - d3 - rho_c * u[2] * u[2];
    const T pxy = s[3] - rho_c * u[0] * u[1], pxz = s[4] - rho_c * u[0] * u[2];
    const T pyz = s[5] - rho_c * u[1] * u[2];
    const T pn = std::sqrt((pxx * pxx + pyy * pyy + pzz * pzz) + T(2) * (pxy * pxy + pxz * pxz + pyz * pyz));
    const double cs = params.smagorinsky_cs;
    const T les_c = T(18.0 * std::sqrt(2.0) * cs * cs);
    const T tau0 = T(params.collision == CENTRAL_MOMENT ? 1.0 / params.omega_shear_cfg : 3.0 * params.nu + 0.5);
    const T te = T(0.5) * (tau0 + std::sqrt(tau0 * tau0 + les_c * pn / rho_c));
    KParams<T> kc = kp;
    kc.omega_p = T(1) / te;
    kc.omega_m = params.collision == TRT ? T(1) / (T(params.magic) / (te - T(0.5)) + T(0.5)) : kc.omega_p;
    kc.cp = T(1) - kc.omega_p * T(0.5);
    kc.cm = T(1) - kc.omega_m * T(0.5);
    kc.omega_shear = kc.omega_p;
    return kc;
  }

  void stream() {  // stream_row (kernels.rs:547-622) over the full core
    const auto& tb = tables<L>();
    const T six = T(6.0);
#pragma omp parallel for schedule(static)
    for (long zz = 0; zz < dims[2]; ++zz)
      for (long y = 0; y < dims[1]; ++y)
        for (long x = 0; x < dims[0]; ++x) {
          size_t i = idx(x, y, zz);
          if (solid[i]) continue;
          for (int q = 0; q < L::Q; ++q) {
            long s[3] = {x - L::C[q][0], y - L::C[q][1], zz - L::C[q][2]};
            bool skip = false;
            for (int a = 0; a < 3; ++a) {
              if (s[a] < 0) {
                if (!periodic[a]) skip = true;
                else s[a] += dims[a];
              } else if (s[a] >= dims[a]) {
                if (!periodic[a]) skip = true;
                else s[a] -= dims[a];
              }
            }
            if (skip) continue;
            size_t si = idx(s[0], s[1], s[2]);
            if (solid[si] && params.free_slip_top && L::C[q][2] == -1 && zz + 1 == dims[2] - 1) {
              // pull form of the specular rule: the population arriving with
              // (cx, cy, -1) left the partner x - (cx, cy, 0) with (cx, cy, +1)
              long px = x - L::C[q][0], py = y - L::C[q][1];
              bool in = true;
              if (px < 0 || px >= dims[0]) {
                if (periodic[0]) px = (px + dims[0]) % dims[0];
                else in = false;
              }
              if (py < 0 || py >= dims[1]) {
                if (periodic[1]) py = (py + dims[1]) % dims[1];
                else in = false;
              }
              if (in && !solid[idx(px, py, zz)]) {
                int m = 0;
                for (int k = 0; k < L::Q; ++k)
                  if (L::C[k][0] == L::C[q][0] && L::C[k][1] == L::C[q][1] && L::C[k][2] == 1) m = k;
                ftmp[q * n + i] = f[size_t(m) * n + idx(px, py, zz)];
                continue;
              }
            }
            if (solid[si]) {
              T fout = f[tb.opp[q] * n + i];
              const T* wu = &wall_u[3 * si];
              T cu = kp.cr[q][0] * wu[0];
              for (int d = 1; d < L::D; ++d) cu = cu + kp.cr[q][d] * wu[d];
              ftmp[q * n + i] = fout + six * kp.wr[q] * rho[i] * cu;
            } else {
              ftmp[q * n + i] = f[q * n + si];
            }
          }
        }
  }

  void update_moments() {  // moments_row (kernels.rs:627-668)
    const T half = T(0.5);
#pragma omp parallel for schedule(static)
    for (long c = 0; c < long(n); ++c) {
      if (solid[c]) continue;
      T dr = T(0), m0 = T(0), m1 = T(0), m2 = T(0);
      for (int q = 0; q < L::Q; ++q) {
        T fq = f[q * n + c];
        dr = dr + fq;
        m0 = m0 + kp.cr[q][0] * fq;
        m1 = m1 + kp.cr[q][1] * fq;
        m2 = m2 + kp.cr[q][2] * fq;
      }
      T r = T(1) + dr;
      T fv[3];
      force_at(size_t(c), fv);
      rho[c] = r;
      T inv = T(1) / r;
      ux[c] = (m0 + half * fv[0]) * inv;
      uy[c] = (m1 + half * fv[1]) * inv;
      uz[c] = (m2 + half * fv[2]) * inv;
    }
  }

  // One Solver::step (solver.rs:2237-2280): run_span(1) = collide, stream,
  // swap, update_moments; then the scalar ADE.
  // 16-bit storage: round every population of the fluid cells that the
  // stream just wrote.
  void round_stored(std::vector<T>& g) {
    if (!params.store16) return;
    const int mode = params.store16;
#pragma omp parallel for schedule(static)
    for (long c = 0; c < long(n); ++c) {
      if (solid[c]) continue;
      for (int q = 0; q < L::Q; ++q) g[q * n + c] = T(store16_round(mode, float(g[q * n + c])));
    }
  }

  void step() {
    collide();
    stream();
    round_stored(ftmp);
    std::swap(f, ftmp);
    update_moments();
    ++time;
    step_scalars();
  }

  void run(int steps) {
    for (int s = 0; s < steps; ++s) step();
  }

  // reduce_impl (backend.rs:920-970), z,y,x order, f64 accumulation.
  double reduce(int kind, int axis) const {
    double acc = 0.0;
    for (size_t c = 0; c < n; ++c) {
      if (solid[c]) continue;
      if (kind == RED_FLUID_CELLS) {
        acc += 1.0;
      } else if (kind == RED_MASS_DEV) {
        for (int q = 0; q < L::Q; ++q) acc += double(f[q * n + c]);
      } else {
        double m = 0.0;
        for (int q = 0; q < L::Q; ++q) m += double(L::C[q][axis]) * double(f[q * n + c]);
        double fa = has_force_field ? double(kp.force[axis]) + double(force_field[3 * c + axis])
                                    : double(kp.force[axis]);
        acc += m + 0.5 * fa;
      }
    }
    return acc;
  }
  double total_mass_f64() const { return reduce(RED_FLUID_CELLS, 0) + reduce(RED_MASS_DEV, 0); }

  // Solver::init_with (solver.rs:2474-2605) with the init closure sampled
  // into compact arrays (init is pure, so sampling at a neighbour equals the
  // array value there).
  void init_with(const double* r_in, const double* u_in) {
    const T three = T(3.0), half = T(0.5);
    const T tau = T(3.0 * params.nu + 0.5);
    for (size_t c = 0; c < n; ++c) {
      rho[c] = T(r_in[c]);
      ux[c] = T(u_in[3 * c + 0]);
      uy[c] = T(u_in[3 * c + 1]);
      uz[c] = T(u_in[3 * c + 2]);
    }
    for (long z = 0; z < dims[2]; ++z)
      for (long y = 0; y < dims[1]; ++y)
        for (long x = 0; x < dims[0]; ++x) {
          size_t c = idx(x, y, z);
          T u[3] = {ux[c], uy[c], uz[c]};
          T feq[Q_MAX];
          equilibrium<L, T>(kp, rho[c], u, feq);
          for (int q = 0; q < L::Q; ++q) f[q * n + c] = feq[q];
          if (solid[c]) continue;
          auto sample = [&](int a, int dlt, T out[3]) -> bool {
            long g[3] = {x, y, z};
            g[a] += dlt;
            if (g[a] < 0 || g[a] >= dims[a]) {
              if (a < L::D && periodic[a]) g[a] = (g[a] + dims[a]) % dims[a];
              else return false;
            }
            size_t gi = idx(g[0], g[1], g[2]);
            if (solid[gi]) return false;
            out[0] = T(u_in[3 * gi + 0]);
            out[1] = T(u_in[3 * gi + 1]);
            out[2] = T(u_in[3 * gi + 2]);
            return true;
          };
          T grad[3][3] = {{T(0), T(0), T(0)}, {T(0), T(0), T(0)}, {T(0), T(0), T(0)}};
          for (int a = 0; a < L::D; ++a) {
            T pv[3] = {T(0), T(0), T(0)}, mv[3] = {T(0), T(0), T(0)};
            bool hp = sample(a, 1, pv), hm = sample(a, -1, mv);
            for (int b = 0; b < L::D; ++b) {
              if (hp && hm) grad[a][b] = (pv[b] - mv[b]) * half;
              else if (hp) grad[a][b] = pv[b] - u[b];
              else if (hm) grad[a][b] = u[b] - mv[b];
              else grad[a][b] = T(0);
            }
          }
          T div = grad[0][0];
          for (int a = 1; a < L::D; ++a) div = div + grad[a][a];
          for (int q = 0; q < L::Q; ++q) {
            const T* cq = kp.cr[q];
            T ccgu = cq[0] * cq[0] * grad[0][0];
            for (int a = 0; a < L::D; ++a)
              for (int b = a; b < L::D; ++b) {
                if (a == 0 && b == 0) continue;
                if (a == b) ccgu = ccgu + cq[a] * cq[a] * grad[a][a];
                else ccgu = ccgu + cq[a] * cq[b] * (grad[a][b] + grad[b][a]);
              }
            T fneq = -kp.wr[q] * rho[c] * tau * (three * ccgu - div);
            f[q * n + c] = f[q * n + c] + fneq;
          }
        }
    update_moments();
  }

  // --- force field / IBM (solver.rs:2805-2822, 3016-3282) ---
  // Native strain rate of one cell (Solver::strain_rate_at, solver.rs:5393-
  // 5447): Pi_neq = sum c c (f - feq(rho, u)) over the post-stream
  // populations and the cached moments, corrected by +0.5 (uF + Fu) with
  // the current force, scaled by -1 / (2 cs^2 rho tau_eff), tau_eff =
  // 1 / omega_p. Order [S_xx, S_yy, S_zz, S_xy, S_xz, S_yz]; solids: zeros.
  void strain_rate_at(size_t c, T out[6]) const {
    for (int k = 0; k < 6; ++k) out[k] = T(0);
    if (solid[c]) return;
    const T r = rho[c];
    const T u[3] = {ux[c], uy[c], uz[c]};
    T feq[Q_MAX];
    equilibrium<L, T>(kp, r, u, feq);
    T pi[6] = {T(0), T(0), T(0), T(0), T(0), T(0)};
    for (int q = 0; q < L::Q; ++q) {
      const T fneq = f[q * n + c] - feq[q];
      const T cx = kp.cr[q][0], cy = kp.cr[q][1], cz = kp.cr[q][2];
      pi[0] = pi[0] + cx * cx * fneq;
      pi[1] = pi[1] + cy * cy * fneq;
      pi[2] = pi[2] + cz * cz * fneq;
      pi[3] = pi[3] + cx * cy * fneq;
      pi[4] = pi[4] + cx * cz * fneq;
      pi[5] = pi[5] + cy * cz * fneq;
    }
    T fv[3];
    force_at(c, fv);
    const T half = T(0.5);
    pi[0] = pi[0] + u[0] * fv[0];
    pi[1] = pi[1] + u[1] * fv[1];
    pi[2] = pi[2] + u[2] * fv[2];
    pi[3] = pi[3] + half * (u[0] * fv[1] + u[1] * fv[0]);
    pi[4] = pi[4] + half * (u[0] * fv[2] + u[2] * fv[0]);
    pi[5] = pi[5] + half * (u[1] * fv[2] + u[2] * fv[1]);
    const T tau_eff = T(1.0 / params.omega_p);
    const T scale = -(T(1) / (T(2.0 / 3.0) * r * tau_eff));
    for (int k = 0; k < 6; ++k) out[k] = pi[k] * scale;
  }
  void set_omega_field(const double* v) {
    if (!v) {
      has_omega_field = false;
      omega_field.clear();
      return;
    }
    omega_field.assign(n, T(0));
    for (size_t i = 0; i < n; ++i) omega_field[i] = T(v[i]);
    has_omega_field = true;
  }

  // Velocity gradient g[i][j] = du_i/dx_j of one cell
  // (Solver::gather_velocity_gradient, solver.rs:5482-5582): symmetric
  // off-diagonal part from the native strain rate, diagonal and rotation
  // from velocity differences: central between fluid cells, the half-way
  // wall stencil -4/3 w + u + 1/3 u(+1) (mirrored) next to a solid (whose
  // wall velocity counts), one-sided at a non-periodic domain edge,
  // periodic faces wrapped. Solid cells: zeros.
  void velocity_gradient_at(size_t c, T out[3][3]) const {
    for (int i = 0; i < 3; ++i)
      for (int j = 0; j < 3; ++j) out[i][j] = T(0);
    if (solid[c]) return;
    T st[6];
    strain_rate_at(c, st);
    T sm[3][3];
    sm[0][0] = st[0];
    sm[1][1] = st[1];
    sm[2][2] = st[2];
    sm[0][1] = sm[1][0] = st[3];
    sm[0][2] = sm[2][0] = st[4];
    sm[1][2] = sm[2][1] = st[5];
    const long x = long(c % size_t(dims[0])), y = long((c / size_t(dims[0])) % size_t(dims[1])),
               z = long(c / (size_t(dims[0]) * size_t(dims[1])));
    const T own[3] = {ux[c], uy[c], uz[c]};
    // neighbour along axis a by da: 0 none, 1 fluid (v), 2 solid (wall velocity v)
    auto nb = [&](int a, int da, T v[3]) {
      long pp[3] = {x, y, z};
      pp[a] += da;
      if (pp[a] < 0 || pp[a] >= dims[a]) {
        if (!periodic[a]) return 0;
        pp[a] = (pp[a] + dims[a]) % dims[a];
      }
      const size_t j = idx(pp[0], pp[1], pp[2]);
      if (solid[j]) {
        for (int k = 0; k < 3; ++k) v[k] = wall_u[3 * j + k];
        return 2;
      }
      v[0] = ux[j];
      v[1] = uy[j];
      v[2] = uz[j];
      return 1;
    };
    T fd[3][3];
    for (int comp = 0; comp < 3; ++comp)
      for (int a = 0; a < 3; ++a) {
        T pv[3], mv[3];
        const int hp = nb(a, 1, pv), hm = nb(a, -1, mv);
        T v = T(0);
        if (hp == 1 && hm == 1) v = (pv[comp] - mv[comp]) * T(0.5);
        else if (hp == 1 && hm == 2) v = -T(4.0 / 3.0) * mv[comp] + own[comp] + T(1.0 / 3.0) * pv[comp];
        else if (hp == 2 && hm == 1) v = T(4.0 / 3.0) * pv[comp] - own[comp] - T(1.0 / 3.0) * mv[comp];
        else if (hp == 1 && hm == 0) v = pv[comp] - own[comp];
        else if (hp == 0 && hm == 1) v = own[comp] - mv[comp];
        fd[comp][a] = v;
      }
    for (int r = 0; r < 3; ++r)
      for (int q = 0; q < 3; ++q)
        out[r][q] = r == q ? fd[r][q] : sm[r][q] + T(0.5) * (fd[r][q] - fd[q][r]);
  }

  // WaleLes::update (les.rs:120-211), Cw = 0.325, Delta = 1: nu_t from the
  // velocity gradient, optional tau_eff bound, omega+ field installed for
  // the next collision. diag = {clipped cells, clipped fraction, max nu_t
  // before clipping, tau_eff_max (NaN), nu_t_max (NaN)}.
  void wale_update(bool has_max, double tau_eff_max, std::vector<T>& nu_t, double diag[5]) {
    const T cwd = T(0.325) * T(1.0);
    const T cw_delta_sq = cwd * cwd;
    const T nu0 = T(params.nu);
    const T tau0 = T(0.5) + T(3.0) * nu0;
    const T nu_t_max = has_max ? (T(tau_eff_max) - tau0) / T(3.0) : T(0);
    nu_t.assign(n, T(0));
    std::vector<double> om(n);
    size_t clipped = 0;
    T max_before = T(0);
    for (size_t i = 0; i < n; ++i) {
      T g[3][3];
      velocity_gradient_at(i, g);
      T sr[3][3], g2[3][3], sd[3][3];
      for (int a = 0; a < 3; ++a)
        for (int b = 0; b < 3; ++b) sr[a][b] = T(0.5) * (g[a][b] + g[b][a]);
      for (int a = 0; a < 3; ++a)
        for (int b = 0; b < 3; ++b) {
          g2[a][b] = T(0);
          for (int k = 0; k < 3; ++k) g2[a][b] = g2[a][b] + g[a][k] * g[k][b];
        }
      const T tr = g2[0][0] + g2[1][1] + g2[2][2];
      for (int a = 0; a < 3; ++a)
        for (int b = 0; b < 3; ++b) {
          sd[a][b] = T(0.5) * (g2[a][b] + g2[b][a]);
          if (a == b) sd[a][b] = sd[a][b] - tr / T(3.0);
        }
      T ss = T(0), sdsd = T(0);
      for (int a = 0; a < 3; ++a)
        for (int b = 0; b < 3; ++b) {
          ss = ss + sr[a][b] * sr[a][b];
          sdsd = sdsd + sd[a][b] * sd[a][b];
        }
      const T denom = std::pow(ss, T(2.5)) + std::pow(sdsd, T(1.25));
      T nut = denom > T(0) ? cw_delta_sq * std::pow(sdsd, T(1.5)) / denom : T(0);
      max_before = std::max(max_before, nut);
      if (has_max && nut > nu_t_max) {
        ++clipped;
        nut = nu_t_max;
      }
      nu_t[i] = nut;
      om[i] = double(T(1) / (T(3.0) * (nu0 + nut) + T(0.5)));
    }
    set_omega_field(om.data());
    diag[0] = double(clipped);
    diag[1] = n == 0 ? 0.0 : double(T(double(clipped)) / T(double(n)));
    diag[2] = double(max_before);
    diag[3] = has_max ? tau_eff_max : std::nan("");
    diag[4] = has_max ? double(nu_t_max) : std::nan("");
  }

  // gamma_dot = sqrt(2 S:S) (Solver::gather_shear_rate, solver.rs:5588-5599)
  T shear_rate_at(size_t c) const {
    T s[6];
    strain_rate_at(c, s);
    const T ss = s[0] * s[0] + s[1] * s[1] + s[2] * s[2] + T(2.0) * (s[3] * s[3] + s[4] * s[4] + s[5] * s[5]);
    return std::sqrt(T(2.0) * ss);
  }

  void clear_body_force_field() {
    if (!has_force_field) return;
    bool uniform = true;
    for (size_t i = 3; i < 3 * n && uniform; ++i)
      if (force_field[i] != force_field[i % 3]) uniform = false;
    has_force_field = false;
    force_field.clear();
    if (uniform) update_moments();
  }

  IbmDiag apply_rotating_ibm(const Body& body, const IbmConfig& cfg) {
    std::vector<double> r64(n), u_now(3 * n, 0.0);
    for (size_t c = 0; c < n; ++c) {
      r64[c] = double(rho[c]);
      if (solid[c]) continue;
      double mom[3] = {0, 0, 0};
      for (int q = 0; q < L::Q; ++q) {
        double fq = double(f[q * n + c]);
        for (int a = 0; a < L::D; ++a) mom[a] += double(L::C[q][a]) * fq;
      }
      double force[3] = {double(kp.force[0]), double(kp.force[1]), double(kp.force[2])};
      if (has_force_field)
        for (int a = 0; a < 3; ++a) force[a] += double(force_field[3 * c + a]);
      double inv_rho = 1.0 / std::max(double(rho[c]), 1.0e-30);
      for (int a = 0; a < L::D; ++a) u_now[3 * c + a] = (mom[a] + 0.5 * force[a]) * inv_rho;
    }
    std::vector<double> spread(3 * n, 0.0);
    IbmDiag diag = ibm_direct_forcing(dims, L::D, solid.data(), r64.data(), u_now.data(), body, cfg,
                                      spread.data());
    if (!has_force_field) {
      force_field.assign(3 * n, T(0));
      has_force_field = true;
    }
    for (size_t i = 0; i < 3 * n; ++i) force_field[i] = force_field[i] + T(spread[i]);
    return diag;
  }

  // --- passive scalar (solver.rs:2113-2205, 2856-2966; scalar.rs:6-15) ---
  template <class SL>
  void scalar_equilibrium(T conc, const T u[3], T* out) const {
    const T fac = T(SL::INV_CS2);
    for (int q = 0; q < SL::Q; ++q) {
      T cu = T(double(SL::C[q][0])) * u[0] + T(double(SL::C[q][1])) * u[1] + T(double(SL::C[q][2])) * u[2];
      out[q] = T(SL::W[q]) * conc * (T(1) + fac * cu);
    }
  }

  void enable_scalar(int q, double diffusivity) {
    if (!(std::isfinite(diffusivity) && diffusivity > 0.0))
      throw std::runtime_error("scalar diffusivity must be finite > 0");
    if (q != 7 && q != 19 && q != 27) throw std::runtime_error("scalar lattice must be 7, 19 or 27");
    Scalar<T> s;
    s.q = q;
    s.diffusivity = diffusivity;
    s.h.assign(size_t(q) * n, T(0));
    s.htmp.assign(size_t(q) * n, T(0));
    s.conc.assign(n, T(0));
    scalars.push_back(std::move(s));
  }

  template <class SL>
  void set_scalar_impl(Scalar<T>& s, const double* values) {
    for (size_t c = 0; c < n; ++c) {
      T v = T(values[c]);
      s.conc[c] = v;
      T u[3] = {ux[c], uy[c], uz[c]};
      T heq[Q_MAX];
      scalar_equilibrium<SL>(v, u, heq);
      for (int q = 0; q < SL::Q; ++q) {
        s.h[q * n + c] = heq[q];
        s.htmp[q * n + c] = T(0);
      }
    }
  }
  void set_scalar(int k, const double* values) {
    Scalar<T>& s = scalars.at(k);
    if (s.q == 7) set_scalar_impl<D3Q7>(s, values);
    else if (s.q == 19) set_scalar_impl<D3Q19>(s, values);
    else set_scalar_impl<D3Q27>(s, values);
  }

  template <class SL>
  void step_scalar_impl(Scalar<T>& s) {
    const auto& tb = tables<SL>();
    T omega = T(1.0 / (SL::INV_CS2 * s.diffusivity + 0.5));
    for (size_t c = 0; c < n; ++c) {
      if (solid[c]) continue;
      T u[3] = {ux[c], uy[c], uz[c]};
      T heq[Q_MAX];
      scalar_equilibrium<SL>(s.conc[c], u, heq);
      for (int q = 0; q < SL::Q; ++q) {
        size_t k = q * n + c;
        s.h[k] = s.h[k] - omega * (s.h[k] - heq[q]);
      }
    }
    std::fill(s.htmp.begin(), s.htmp.end(), T(0));
    for (long z = 0; z < dims[2]; ++z)
      for (long y = 0; y < dims[1]; ++y)
        for (long x = 0; x < dims[0]; ++x) {
          size_t c = idx(x, y, z);
          if (solid[c]) {
            s.conc[c] = T(0);
            continue;
          }
          for (int q = 0; q < SL::Q; ++q) {
            long sx[3] = {x - SL::C[q][0], y - SL::C[q][1], z - SL::C[q][2]};
            for (int a = 0; a < 3; ++a) {
              if (sx[a] < 0 || sx[a] >= dims[a]) {
                if (!periodic[a]) throw std::runtime_error("scalar stream left a non-periodic domain");
                sx[a] = (sx[a] + dims[a]) % dims[a];
              }
            }
            size_t src = idx(sx[0], sx[1], sx[2]);
            s.htmp[q * n + c] = solid[src] ? s.h[tb.opp[q] * n + c] : s.h[q * n + src];
          }
        }
    std::swap(s.h, s.htmp);
    for (size_t c = 0; c < n; ++c) {
      if (solid[c]) {
        s.conc[c] = T(0);
        continue;
      }
      T sum = T(0);
      for (int q = 0; q < SL::Q; ++q) sum = sum + s.h[q * n + c];
      s.conc[c] = sum;
    }
  }
  void step_scalars() {
    for (auto& s : scalars) {
      if (s.q == 7) step_scalar_impl<D3Q7>(s);
      else if (s.q == 19) step_scalar_impl<D3Q19>(s);
      else step_scalar_impl<D3Q27>(s);
    }
  }
};

// ---------------------------------------------------------------------------
// Walls and stirred-tank geometry.
// ---------------------------------------------------------------------------

// build_wall_rims (solver.rs:1357-1404). Face order XNeg,XPos,YNeg,YPos,ZNeg,ZPos.
inline void build_wall_rims(int d, const int dims[3], const bool is_wall[6], const double u[6][3],
                            uint8_t* solid, double* wall_u) {
  const size_t n = size_t(dims[0]) * dims[1] * dims[2];
  std::vector<double> best(n, -1.0);
  for (size_t i = 0; i < n; ++i) {
    solid[i] = 0;
    wall_u[3 * i] = wall_u[3 * i + 1] = wall_u[3 * i + 2] = 0.0;
  }
  const int order[6] = {2, 3, 0, 1, 4, 5};  // YNeg, YPos, XNeg, XPos, ZNeg, ZPos
  for (int oi = 0; oi < 6; ++oi) {
    int face = order[oi];
    int a = face / 2;
    if (a >= d || !is_wall[face]) continue;
    double speed = u[face][0] * u[face][0] + u[face][1] * u[face][1];
    if (d == 3) speed += u[face][2] * u[face][2];
    int fixed = (face % 2 == 0) ? 0 : dims[a] - 1;
    int t1 = a == 0 ? 1 : 0, t2 = a == 2 ? 1 : 2;
    for (int c2 = 0; c2 < dims[t2]; ++c2)
      for (int c1 = 0; c1 < dims[t1]; ++c1) {
        int pos[3];
        pos[a] = fixed;
        pos[t1] = c1;
        pos[t2] = c2;
        size_t i = (size_t(pos[2]) * dims[1] + pos[1]) * dims[0] + pos[0];
        solid[i] = 1;
        if (speed > best[i]) {
          best[i] = speed;
          for (int k = 0; k < 3; ++k) wall_u[3 * i + k] = u[face][k];
        }
      }
  }
}

// geometry.rs constants (10-16).
constexpr double RUSHTON_BLADE_THICKNESS_FRACTION = 0.04;
constexpr double RUSHTON_DISC_DIAMETER_FRACTION = 0.65;
constexpr double PITCHED_BLADE_ANGLE_DEG = 45.0;
constexpr double PITCHED_BLADE_THICKNESS_FRACTION = 0.035;
constexpr double TAU = 6.283185307179586476925286766559;

struct TankGeometry {  // StirredTankGeometry (geometry.rs:167-176), spargers out of scope
  int dims[3];
  double dx_m;
  std::vector<uint8_t> solid, baffle_mask;
  std::vector<double> wall_velocity;  // n x 3
  // one impeller: markers in lattice coordinates
  double center[3];
  double omega[3];
  std::vector<double> marker_pos;  // m x 3
  std::vector<double> marker_weight;
  std::vector<double> marker_wall_velocity;  // m x 3 (SI)
};

inline double cell_z_m(double dx, int z) { return (double(z) + 0.5) * dx; }  // geometry.rs:941

// apply_cylindrical_tank_mask (geometry.rs:657-679)
inline void apply_cylindrical_tank_mask(const int dims[3], double dx, double vessel_d,
                                        double liquid_h, uint8_t* solid) {
  double radius = 0.5 * vessel_d;
  double cx = 0.5 * dims[0] * dx, cy = 0.5 * dims[1] * dx;
  for (int z = 0; z < dims[2]; ++z) {
    double z_m = cell_z_m(dx, z);
    for (int y = 0; y < dims[1]; ++y)
      for (int x = 0; x < dims[0]; ++x) {
        double px = (double(x) + 0.5) * dx, py = (double(y) + 0.5) * dx;
        double r = std::sqrt((px - cx) * (px - cx) + (py - cy) * (py - cy));
        bool rim = x == 0 || y == 0 || z == 0 || x + 1 == dims[0] || y + 1 == dims[1] || z + 1 == dims[2];
        bool outside = r >= radius || z_m >= liquid_h;
        if (rim || outside) solid[(size_t(z) * dims[1] + y) * dims[0] + x] = 1;
      }
  }
}

// apply_baffle_mask (geometry.rs:681-723), count = 4, wall attached.
inline void apply_baffle_mask(const int dims[3], double dx, double vessel_d, double liquid_h,
                              double width_m, double thickness_m, uint8_t* solid, uint8_t* baffle) {
  double radius = 0.5 * vessel_d;
  double cx = 0.5 * dims[0] * dx, cy = 0.5 * dims[1] * dx;
  double radial_inner = radius - width_m;
  for (int z = 1; z < std::max(dims[2] - 1, 0); ++z) {
    double z_m = cell_z_m(dx, z);
    if (z_m >= liquid_h) continue;
    for (int y = 1; y < std::max(dims[1] - 1, 0); ++y)
      for (int x = 1; x < std::max(dims[0] - 1, 0); ++x) {
        double px = (double(x) + 0.5) * dx, py = (double(y) + 0.5) * dx;
        double rx = px - cx, ry = py - cy;
        double r = std::sqrt(rx * rx + ry * ry);
        if (r >= radius || r < radial_inner) continue;
        bool near_x_wall = std::fabs(ry) <= 0.5 * thickness_m;
        bool near_y_wall = std::fabs(rx) <= 0.5 * thickness_m;
        if (near_x_wall || near_y_wall) {
          size_t i = (size_t(z) * dims[1] + y) * dims[0] + x;
          solid[i] = 1;
          baffle[i] = 1;
        }
      }
  }
}

// build_radial_impeller (geometry.rs:815-906): kind 0 = Rushton, 1 = pitched blade.
inline void build_radial_impeller(const int dims[3], double dx, double vessel_d, double liquid_h,
                                  int kind, double diameter_m, double clearance_m, int blade_count,
                                  double omega_z, TankGeometry& out) {
  double blade_angle_deg = kind == 0 ? 0.0 : PITCHED_BLADE_ANGLE_DEG;
  double thickness_fraction = kind == 0 ? RUSHTON_BLADE_THICKNESS_FRACTION : PITCHED_BLADE_THICKNESS_FRACTION;
  double center_xy[2] = {0.5 * dims[0] * dx, 0.5 * dims[1] * dx};
  double radius = 0.5 * diameter_m;
  double center[3] = {center_xy[0], center_xy[1], clearance_m};
  double radial_inner = kind == 0 ? RUSHTON_DISC_DIAMETER_FRACTION * radius : 0.35 * radius;
  double dr = std::max(dx, radius / 20.0);
  double dz = dx;
  double tangential_step = dx;
  double thickness = std::max(thickness_fraction * diameter_m, dx);
  out.marker_pos.clear();
  out.marker_weight.clear();
  out.marker_wall_velocity.clear();
  for (int b = 0; b < blade_count; ++b) {
    double th = TAU * double(b) / double(blade_count);
    double er[3] = {std::cos(th), std::sin(th), 0.0};
    double et[3] = {-std::sin(th), std::cos(th), 0.0};
    double pitch = blade_angle_deg * (3.14159265358979323846264338327950288 / 180.0);
    double z_span = blade_angle_deg == 0.0 ? thickness
                                           : thickness + (radius - radial_inner) * std::sin(pitch) * 0.18;
    size_t nr = size_t(std::max(std::ceil((radius - radial_inner) / dr), 1.0));
    size_t nt = size_t(std::max(std::ceil(thickness / tangential_step), 1.0));
    size_t nz = size_t(std::max(std::ceil(z_span / dz), 1.0));
    for (size_t ir = 0; ir <= nr; ++ir) {
      double rr = radial_inner + (radius - radial_inner) * double(ir) / double(nr);
      for (size_t it = 0; it <= nt; ++it) {
        double offset_t = -0.5 * thickness + thickness * double(it) / double(nt);
        for (size_t iz = 0; iz <= nz; ++iz) {
          double offset_z = -0.5 * z_span + z_span * double(iz) / double(nz);
          double pitched_z = offset_z + (rr - radial_inner) * std::sin(pitch) * 0.18;
          double p[3] = {center[0] + rr * er[0] + offset_t * et[0],
                         center[1] + rr * er[1] + offset_t * et[1], center[2] + pitched_z};
          double rel_r = std::sqrt(std::pow(p[0] - center_xy[0], 2) + std::pow(p[1] - center_xy[1], 2));
          if (rel_r >= 0.5 * vessel_d || p[2] <= 0.0 || p[2] >= liquid_h) continue;
          double rvec[3] = {p[0] - center[0], p[1] - center[1], p[2] - center[2]};
          double uu[3] = {0.0 * rvec[2] - omega_z * rvec[1], omega_z * rvec[0] - 0.0 * rvec[2],
                          0.0 * rvec[1] - 0.0 * rvec[0]};
          out.marker_pos.push_back(p[0] / dx);
          out.marker_pos.push_back(p[1] / dx);
          out.marker_pos.push_back(p[2] / dx);
          out.marker_weight.push_back(dx * dx);
          for (int a = 0; a < 3; ++a) out.marker_wall_velocity.push_back(uu[a]);
        }
      }
    }
  }
  if (out.marker_weight.empty()) throw std::runtime_error("impeller marker generation produced no markers");
  out.center[0] = center[0] / dx;
  out.center[1] = center[1] / dx;
  out.center[2] = center[2] / dx;
  out.omega[0] = 0.0;
  out.omega[1] = 0.0;
  out.omega[2] = omega_z;
}

// stamp_impeller_wall_velocity (geometry.rs:908-920)
inline void stamp_impeller_wall_velocity(TankGeometry& g) {
  auto nearest = [](double v, int nn) {
    double r = std::round(v);
    r = std::max(r, 0.0);
    r = std::min(r, double(nn - 1));
    return size_t(r);
  };
  size_t m = g.marker_weight.size();
  for (size_t k = 0; k < m; ++k) {
    size_t x = nearest(g.marker_pos[3 * k], g.dims[0]);
    size_t y = nearest(g.marker_pos[3 * k + 1], g.dims[1]);
    size_t z = nearest(g.marker_pos[3 * k + 2], g.dims[2]);
    size_t i = (z * g.dims[1] + y) * g.dims[0] + x;
    for (int a = 0; a < 3; ++a) g.wall_velocity[3 * i + a] = g.marker_wall_velocity[3 * k + a];
  }
}

// Flat-blade (disc) turbine of the device library's tank builder
// (lbmflow_b200/csrc/host_geometry.cpp, kind "flat_blade"; the reference has
// no such generator). Restated here so that a tank built with it needs only
// the oracle: markers on the analytic surfaces at a uniform spacing h cells
// (disc of diameter 0.75 D as concentric rings on both faces, blades of
// radial length D/4 and height D/5 at the rim on both faces of a plate of
// thickness max(0.04 D, 1 cell)); weights are the face area per marker.
// The target velocity of each marker, for the wall-velocity stamp, is
// Omega_z x (p - c) in SI with c = (nx/2, ny/2, clearance) dx.
inline void build_flat_blade_turbine(const int dims[3], double dx, double diameter_m, double clearance_m,
                                     int blade_count, double spacing_cells, double omega_z, TankGeometry& out) {
  const double h = spacing_cells;
  const double D = diameter_m / dx, R = 0.5 * D;
  const double cx = 0.5 * dims[0], cy = 0.5 * dims[1], cz = clearance_m / dx;
  const double t = std::max(0.04 * D, 1.0);
  const double blade_len = 0.25 * D, blade_h = 0.2 * D, r_in = R - blade_len;
  const double r_disc = 0.375 * D;
  const double cxs = 0.5 * dims[0] * dx, cys = 0.5 * dims[1] * dx;
  out.marker_pos.clear();
  out.marker_weight.clear();
  out.marker_wall_velocity.clear();
  auto add = [&](double x, double y, double z, double w) {
    out.marker_pos.push_back(x);
    out.marker_pos.push_back(y);
    out.marker_pos.push_back(z);
    out.marker_weight.push_back(w);
    const double p[3] = {x * dx, y * dx, z * dx};
    const double r[3] = {p[0] - cxs, p[1] - cys, p[2] - clearance_m};
    out.marker_wall_velocity.push_back(0.0 * r[2] - omega_z * r[1]);
    out.marker_wall_velocity.push_back(omega_z * r[0] - 0.0 * r[2]);
    out.marker_wall_velocity.push_back(0.0 * r[1] - 0.0 * r[0]);
  };
  const int rings = int(std::ceil(r_disc / h));
  std::vector<double> rr;
  std::vector<int> rn;
  int total = 0;
  for (int k = 0; k <= rings; ++k) {
    const double r = r_disc * double(k) / double(rings);
    const int m = k == 0 ? 1 : std::max(1, int(std::lround(TAU * r / h)));
    rr.push_back(r);
    rn.push_back(m);
    total += m;
  }
  const double w_disc = 3.14159265358979323846264338327950288 * r_disc * r_disc / double(total);
  for (int face = 0; face < 2; ++face) {
    const double z = cz + (face ? 0.5 : -0.5) * t;
    for (size_t k = 0; k < rr.size(); ++k)
      for (int j = 0; j < rn[k]; ++j) {
        const double th = TAU * (double(j) + 0.5 * double(k & 1)) / double(rn[k]);
        add(cx + rr[k] * std::cos(th), cy + rr[k] * std::sin(th), z, w_disc);
      }
  }
  const int nr = std::max(1, int(std::ceil(blade_len / h)));
  const int nzb = std::max(1, int(std::ceil(blade_h / h)));
  const double w_blade = blade_len * blade_h / double((nr + 1) * (nzb + 1));
  for (int b = 0; b < blade_count; ++b) {
    const double th = TAU * double(b) / double(blade_count);
    const double er[2] = {std::cos(th), std::sin(th)}, et[2] = {-std::sin(th), std::cos(th)};
    for (int face = 0; face < 2; ++face) {
      const double off = (face ? 0.5 : -0.5) * t;
      for (int i = 0; i <= nr; ++i) {
        const double r = r_in + blade_len * double(i) / double(nr);
        for (int k = 0; k <= nzb; ++k) {
          const double z = cz - 0.5 * blade_h + blade_h * double(k) / double(nzb);
          add(cx + r * er[0] + off * et[0], cy + r * er[1] + off * et[1], z, w_blade);
        }
      }
    }
  }
  out.center[0] = cxs / dx;
  out.center[1] = cys / dx;
  out.center[2] = clearance_m / dx;
  out.omega[0] = 0.0;
  out.omega[1] = 0.0;
  out.omega[2] = omega_z;
}

// ---------------------------------------------------------------------------
// Runner QOIs and set-up helpers (crates/lbm-cli/src/runner.rs,
// crates/lbm-scenario/src/units.rs).
// ---------------------------------------------------------------------------
// f64::powi for the small exponents used here: binary exponentiation from
// the low bits (x^3 = x * x^2, x^5 = x * x^4).
inline double powi(double x, int k) {
  double r = 1.0, sq = x;
  bool first = true;
  while (k) {
    if (k & 1) {
      r = first ? sq : r * sq;
      first = false;
    }
    k >>= 1;
    if (k) sq = sq * sq;
  }
  return r;
}

// torque_record_from_ibm (runner.rs:1396-1425): N m per lattice torque unit.
inline double torque_scale(double rho, double dx, double dt) { return rho * powi(dx, 5) / powi(dt, 2); }

// write_power_qois averaging (runner.rs:1514-1543) over the runner's
// records: records at steps s (1-based) with s % probe_every == 0 or
// s == run_steps among the executed steps; mean torque (N m) over records
// with s >= run_steps / 2, or over all records when none is that late.
// Returns NaN when there is no record.
inline double runner_mean_torque(const double* torque_lu, long executed, long run_steps, long probe_every, double rho,
                                 double dx, double dt, long* used) {
  if (probe_every <= 0) probe_every = 1;
  const double sc = torque_scale(rho, dx, dt);
  std::vector<std::pair<long, double>> recs;
  for (long s = 1; s <= executed; ++s)
    if (s % probe_every == 0 || s == run_steps) recs.push_back({s, torque_lu[s - 1] * sc});
  if (recs.empty()) return NAN;
  const long start = run_steps / 2;
  std::vector<double> win;
  for (auto& r : recs)
    if (r.first >= start) win.push_back(r.second);
  if (win.empty())
    for (auto& r : recs) win.push_back(r.second);
  double sum = 0.0;
  for (double v : win) sum += v;
  if (used) *used = long(win.size());
  return sum / double(win.size());
}

// bioprocess_unit_report_unchecked (units.rs:116-325), single-phase
// stirred tank with an optional passive scalar (d_scalar <= 0: none).
// out: dx, dt, u_ref_lu, nu_lu, tau_lu, cs2, Re, Fr, Ma, Sc, Pe, D_lu,
// grid Re; warn/rej bits: 1 MA_LATTICE_HIGH, 2 MA_LATTICE_TOO_HIGH, 4
// TAU_NEAR_HALF, 8 TAU_NON_POSITIVE_VISCOSITY, 16 GRID_REYNOLDS_HIGH, 32
// SCALAR_DIFFUSION_UNSTABLE. Returns false for a non-positive input.
inline bool unit_report(double vessel_d, double liquid_h, double imp_d, double rpm, double rho, double mu, double dt,
                        const int grid[3], double d_scalar, double out[13], unsigned* warn, unsigned* rej) {
  for (double v : {vessel_d, liquid_h, imp_d, rpm, rho, mu, dt})
    if (!(std::isfinite(v) && v > 0.0)) return false;
  if (grid[0] == 0 || grid[1] == 0 || grid[2] == 0) return false;
  const double n_hz = rpm / 60.0;
  const double u_ref_m_s = n_hz * imp_d;
  const double nu_m2_s = mu / rho;
  const double dx_m = vessel_d / double(grid[0]);
  const double u_ref_lu = u_ref_m_s * dt / dx_m;
  const double nu_lu = nu_m2_s * dt / (dx_m * dx_m);
  const double tau_lu = 3.0 * nu_lu + 0.5;
  const double cs2 = 1.0 / 3.0;
  const double mach = u_ref_lu / std::sqrt(cs2);
  const double re = rho * n_hz * powi(imp_d, 2) / mu;
  const double fr = powi(n_hz, 2) * imp_d / 9.80665;
  const bool has_d = d_scalar > 0.0;
  const double sc = has_d ? nu_m2_s / d_scalar : NAN;
  const double pe = has_d ? u_ref_m_s * vessel_d / d_scalar : NAN;
  const double d_lu = has_d ? d_scalar * dt / (dx_m * dx_m) : NAN;
  unsigned w = 0, r = 0;
  if (mach > 0.30)
    r |= 2;
  else if (mach > 0.10)
    w |= 1;
  if (tau_lu <= 0.5)
    r |= 8;
  else if (tau_lu <= 0.55)
    w |= 4;
  const double grid_re = u_ref_lu / nu_lu;
  if (grid_re > 15.0) w |= 16;
  if (has_d && nu_lu / d_lu > 25.0) w |= 32;
  const double vals[13] = {dx_m, dt, u_ref_lu, nu_lu, tau_lu, cs2, re, fr, mach, sc, pe, d_lu, grid_re};
  for (int i = 0; i < 13; ++i) out[i] = vals[i];
  *warn = w;
  *rej = r;
  return true;
}

// scalar_initial_condition, pulse branch (runner.rs:1317-1377): the pulse
// concentration on fluid cells whose centre lies within the radius.
inline void top_hat_pulse(const int dims[3], const uint8_t* solid, double dx, const double center[3], double radius,
                          double conc, double* values) {
  for (int z = 0; z < dims[2]; ++z)
    for (int y = 0; y < dims[1]; ++y)
      for (int x = 0; x < dims[0]; ++x) {
        const size_t i = (size_t(z) * dims[1] + y) * dims[0] + x;
        values[i] = 0.0;
        if (solid && solid[i]) continue;
        const double p[3] = {(double(x) + 0.5) * dx, (double(y) + 0.5) * dx, (double(z) + 0.5) * dx};
        const double r = std::sqrt(powi(p[0] - center[0], 2) + powi(p[1] - center[1], 2) + powi(p[2] - center[2], 2));
        if (r <= radius) values[i] = conc;
      }
}

// ---------------------------------------------------------------------------
// QOI formulas (crates/lbm-core/src/qoi.rs:477-556).
// ---------------------------------------------------------------------------
struct PowerQoi {
  double torque_n_m, power_w, rotational_speed_hz, np, p_over_v_w_m3;
};

inline PowerQoi power_qois(double torque, double omega, double rho, double d, double volume) {
  if (!(std::isfinite(omega) && std::isfinite(rho) && std::isfinite(d) && std::isfinite(volume) &&
        rho > 0.0 && d > 0.0 && volume > 0.0))
    throw std::runtime_error("power QOI inputs must be finite and positive where dimensional");
  double n_hz = omega / TAU;
  if (!(n_hz > 0.0)) throw std::runtime_error("rotational speed must be positive for Np/Nq");
  double power = omega * torque;
  double denom = rho * powi(n_hz, 3) * powi(d, 5);
  return {torque, power, n_hz, power / denom, power / volume};
}

// scalar_cv: returns NaN for the reference's None.
inline double scalar_cv(const double* v, const uint8_t* include, size_t n) {
  size_t cnt = 0;
  double sum = 0.0;
  for (size_t i = 0; i < n; ++i)
    if (include[i]) {
      ++cnt;
      sum += v[i];
    }
  if (cnt == 0) return NAN;
  double mean = sum / double(cnt);
  if (mean == 0.0) return NAN;
  double var = 0.0;
  for (size_t i = 0; i < n; ++i)
    if (include[i]) {
      double dd = v[i] - mean;
      var += dd * dd;
    }
  return std::sqrt(var / double(cnt)) / std::fabs(mean);
}

// mixing_time_from_cv: out = {cv0, t95, t99}; NaN for None. Returns false
// when no finite positive CV exists.
inline bool mixing_time_from_cv(const double* t, const double* cv, size_t n, double out[3]) {
  size_t k = 0;
  for (; k < n; ++k)
    if (std::isfinite(cv[k]) && cv[k] > 0.0) break;
  if (k == n) return false;
  double cv0 = cv[k];
  double t95 = NAN, t99 = NAN;
  for (size_t i = 0; i < n; ++i) {
    if (!std::isfinite(cv[i])) continue;
    if (std::isnan(t95) && cv[i] <= 0.05 * cv0) t95 = t[i];
    if (std::isnan(t99) && cv[i] <= 0.01 * cv0) t99 = t[i];
  }
  out[0] = cv0;
  out[1] = t95;
  out[2] = t99;
  return true;
}

// ---------------------------------------------------------------------------
// Velocity-gradient stress QOIs (crates/lbm-core/src/stress.rs), f64 over
// f64 velocity fields in SI units. Cell index (z ny + y) nx + x.
// ---------------------------------------------------------------------------
struct StressCell {  // stress.rs:3-10
  double s[6];
  double gamma_dot, viscous_stress_pa, second_invariant_s2, von_mises_proxy_pa;
};

// velocity_gradient + neighbor_value (stress.rs:178-226): central
// differences, one-sided next to a solid or the domain edge, zero when both
// neighbours are missing, zero along an axis of extent 1. Not periodic.
inline void stress_velocity_gradient(const int d[3], const double* const f[3], const uint8_t* solid, double dx,
                                     long x, long y, long z, double g[3][3]) {
  const long pos[3] = {x, y, z};
  auto id = [&](long a, long b, long c) { return size_t((c * d[1] + b) * d[0] + a); };
  for (int comp = 0; comp < 3; ++comp)
    for (int axis = 0; axis < 3; ++axis) {
      g[comp][axis] = 0.0;
      if (d[axis] <= 1) continue;
      auto nb = [&](int delta, double& v) {
        long p[3] = {pos[0], pos[1], pos[2]};
        p[axis] += delta;
        if (p[axis] < 0 || p[axis] >= d[axis]) return false;
        const size_t i = id(p[0], p[1], p[2]);
        if (solid[i]) return false;
        v = f[comp][i];
        return true;
      };
      double pv = 0.0, mv = 0.0;
      const bool hp = nb(1, pv), hm = nb(-1, mv);
      const double own = f[comp][id(x, y, z)];
      if (hp && hm) g[comp][axis] = (pv - mv) / (2.0 * dx);
      else if (hp) g[comp][axis] = (pv - own) / dx;
      else if (hm) g[comp][axis] = (own - mv) / dx;
    }
}

// compute_stress_field (stress.rs:32-82); mu per cell.
inline std::vector<StressCell> compute_stress_field(const int d[3], const double* ux, const double* uy,
                                                    const double* uz, const uint8_t* solid, double dx,
                                                    const double* mu) {
  const size_t n = size_t(d[0]) * d[1] * d[2];
  std::vector<StressCell> out(n, StressCell{{0, 0, 0, 0, 0, 0}, 0, 0, 0, 0});
  const double* f[3] = {ux, uy, uz};
  for (long z = 0; z < d[2]; ++z)
    for (long y = 0; y < d[1]; ++y)
      for (long x = 0; x < d[0]; ++x) {
        const size_t i = size_t((z * d[1] + y) * d[0] + x);
        if (solid[i]) continue;
        double g[3][3];
        stress_velocity_gradient(d, f, solid, dx, x, y, z, g);
        const double s[6] = {g[0][0], g[1][1], g[2][2], 0.5 * (g[0][1] + g[1][0]), 0.5 * (g[0][2] + g[2][0]),
                             0.5 * (g[1][2] + g[2][1])};
        const double ss = s[0] * s[0] + s[1] * s[1] + s[2] * s[2] + 2.0 * (s[3] * s[3] + s[4] * s[4] + s[5] * s[5]);
        const double gd = std::sqrt(2.0 * ss);
        StressCell& o = out[i];
        for (int k = 0; k < 6; ++k) o.s[k] = s[k];
        o.gamma_dot = gd;
        o.viscous_stress_pa = mu[i] * gd;
        o.second_invariant_s2 = ss;
        o.von_mises_proxy_pa = std::sqrt(3.0) * mu[i] * gd;
      }
  return out;
}

// percentile_sorted (stress.rs:296-309): linear interpolation between the
// ranks floor / ceil of p (len - 1).
inline double percentile_sorted(const std::vector<double>& s, double p) {
  if (s.size() == 1) return s[0];
  const double rank = p * double(s.size() - 1);
  const size_t lo = size_t(std::floor(rank)), hi = size_t(std::ceil(rank));
  if (lo == hi) return s[lo];
  const double t = rank - double(lo);
  return s[lo] * (1.0 - t) + s[hi] * t;
}

// percentile_summary (stress.rs:84-100): finite values only; false when
// there is none. out = {p50, p90, p95, p99, max, fraction above threshold
// (NaN without a threshold)}.
inline bool percentile_summary(const double* v, size_t n, bool has_threshold, double threshold, double out[6]) {
  std::vector<double> fin;
  fin.reserve(n);
  for (size_t i = 0; i < n; ++i)
    if (std::isfinite(v[i])) fin.push_back(v[i]);
  if (fin.empty()) return false;
  std::sort(fin.begin(), fin.end());
  double frac = std::nan("");
  if (has_threshold) {
    size_t above = 0;
    for (double x : fin) above += x > threshold ? 1 : 0;
    frac = double(above) / double(fin.size());
  }
  out[0] = percentile_sorted(fin, 0.50);
  out[1] = percentile_sorted(fin, 0.90);
  out[2] = percentile_sorted(fin, 0.95);
  out[3] = percentile_sorted(fin, 0.99);
  out[4] = fin.back();
  out[5] = frac;
  return true;
}

struct WallShear {  // WallShearProxy (stress.rs:22-30)
  size_t cell_index;
  double tau_w_pa, y_plus, u_parallel_m_s, y_m;
  double normal[3];
};

// wall_shear_proxy + adjacent_wall_normal_and_velocity (stress.rs:102-294):
// fluid cells with a solid among their 26 in-domain neighbours; normal =
// normalised sum of the offsets to them, wall velocity = their mean; tau_w
// = mu |u_parallel| / (dx / 2), y+ = y u_tau / nu. In cell order.
inline std::vector<WallShear> wall_shear_proxy(const int d[3], const double* ux, const double* uy, const double* uz,
                                               const uint8_t* solid, const double* wall_u, double dx, double rho,
                                               double mu) {
  std::vector<WallShear> out;
  const double y_m = 0.5 * dx, nu = mu / rho;
  for (long z = 0; z < d[2]; ++z)
    for (long y = 0; y < d[1]; ++y)
      for (long x = 0; x < d[0]; ++x) {
        const size_t i = size_t((z * d[1] + y) * d[0] + x);
        if (solid[i]) continue;
        double nrm[3] = {0, 0, 0}, wu[3] = {0, 0, 0}, count = 0.0;
        for (long dz = -1; dz <= 1; ++dz)
          for (long dy = -1; dy <= 1; ++dy)
            for (long dxo = -1; dxo <= 1; ++dxo) {
              if (!dxo && !dy && !dz) continue;
              const long a = x + dxo, b = y + dy, c = z + dz;
              if (a < 0 || b < 0 || c < 0 || a >= d[0] || b >= d[1] || c >= d[2]) continue;
              const size_t j = size_t((c * d[1] + b) * d[0] + a);
              if (!solid[j]) continue;
              nrm[0] += double(dxo);
              nrm[1] += double(dy);
              nrm[2] += double(dz);
              for (int k = 0; k < 3; ++k) wu[k] += wall_u[3 * j + k];
              count += 1.0;
            }
        if (count == 0.0) continue;
        const double mag = std::sqrt(nrm[0] * nrm[0] + nrm[1] * nrm[1] + nrm[2] * nrm[2]);
        if (mag == 0.0) continue;
        for (int k = 0; k < 3; ++k) {
          nrm[k] /= mag;
          wu[k] /= count;
        }
        const double u[3] = {ux[i] - wu[0], uy[i] - wu[1], uz[i] - wu[2]};
        const double un = u[0] * nrm[0] + u[1] * nrm[1] + u[2] * nrm[2];
        const double t[3] = {u[0] - un * nrm[0], u[1] - un * nrm[1], u[2] - un * nrm[2]};
        const double up = std::sqrt(t[0] * t[0] + t[1] * t[1] + t[2] * t[2]);
        const double tau = mu * up / y_m;
        const double u_tau = std::sqrt(tau / rho);
        out.push_back(WallShear{i, tau, y_m * u_tau / nu, up, y_m, {nrm[0], nrm[1], nrm[2]}});
      }
  return out;
}

// ---------------------------------------------------------------------------
// Oxygen transfer and uptake sources (crates/lbm-core/src/oxygen.rs:72-216,
// reaction.rs:57-137) over flat f64 arrays. Each returns 0 on success or an
// error code (the reference's Err variants): 1 invalid cell volume, 2
// invalid transfer inputs / kL, 3 invalid time step, 4 negative or
// non-finite C_L before the uptake, 5 invalid uptake-model parameters.
// ---------------------------------------------------------------------------
struct OxygenDiag {  // OxygenDiagnostics (oxygen.rs:18-23)
  size_t clipped_cells = 0;
  double clipped_fraction = 0.0, min_before_clip = 0.0;
};

inline OxygenDiag clip_negative_concentrations(double* v, size_t n) {  // oxygen.rs:193-216
  OxygenDiag d;
  double mn = INFINITY;
  for (size_t i = 0; i < n; ++i) {
    const double before = v[i];
    if (before < mn) mn = before;
    if (v[i] < 0.0) {
      v[i] = 0.0;
      ++d.clipped_cells;
    }
  }
  d.clipped_fraction = n == 0 ? 0.0 : double(d.clipped_cells) / double(n);
  d.min_before_clip = std::isfinite(mn) ? mn : 0.0;
  return d;
}

// henry_equilibrium (oxygen.rs:72-87); NaN on invalid input
inline double henry_equilibrium(double h, double p) {
  if (!(std::isfinite(h) && h > 0.0) || !(std::isfinite(p) && p >= 0.0)) return std::nan("");
  return h * p;
}

// interfacial_area_density (oxygen.rs:89-115); NaN on invalid input
inline double interfacial_area_density(double phi, const double g[3], double width) {
  if (!(std::isfinite(phi) && phi >= 0.0 && phi <= 1.0) || !(std::isfinite(width) && width > 0.0))
    return std::nan("");
  const double ga = std::sqrt(g[0] * g[0] + g[1] * g[1] + g[2] * g[2]);
  if (!std::isfinite(ga)) return std::nan("");
  return 6.0 * ga * phi * (1.0 - phi) * (4.0 / width);
}

struct OxygenLedger {  // OxygenFluxLedger (oxygen.rs:25-31)
  double cumulative_mol = 0.0, last_step_mol = 0.0, source_integral_mol_s = 0.0;
  size_t active_interface_cells = 0;
};

// apply_interfacial_flux_sources + oxygen_source_step (oxygen.rs:124-191);
// kL of a Constant / Calibrated model.
inline int apply_interfacial_flux_sources(double* c, const double* c_star, const double* area, const double* vol,
                                          size_t n, double dt, double kl, OxygenLedger& ledger, OxygenDiag& diag) {
  if (!(std::isfinite(dt) && dt >= 0.0)) return 3;
  double integral = 0.0;
  size_t active = 0;
  for (size_t i = 0; i < n; ++i) {
    if (!(std::isfinite(vol[i]) && vol[i] > 0.0)) return 1;
    if (!(std::isfinite(c[i]) && std::isfinite(c_star[i]) && std::isfinite(area[i]) && area[i] >= 0.0)) return 2;
    if (!(std::isfinite(kl) && kl > 0.0)) return 2;
    const double source = kl * area[i] * (c_star[i] - c[i]);
    if (area[i] > 0.0) ++active;
    c[i] += source * dt;
    integral += source * vol[i];
  }
  diag = clip_negative_concentrations(c, n);
  ledger.source_integral_mol_s = integral;
  ledger.last_step_mol = integral * dt;
  ledger.cumulative_mol += ledger.last_step_mol;
  ledger.active_interface_cells = active;
  return 0;
}

struct OurModel {  // OurModel (reaction.rs:7-21); kind 0 Constant, 1 Monod, 2 CellDensityScaled
  int kind = 0;
  double our = 0.0, our_max = 0.0, ks = 0.0, c_ref = 0.0, specific_our = 0.0;
};

// oxygen_uptake_rate (reaction.rs:57-93): 0 and the rate, or an error code
inline int oxygen_uptake_rate(const OurModel& m, double c, const double* density, double& rate) {
  if (!(std::isfinite(c) && c >= 0.0)) return 4;
  auto nonneg = [](double v) { return std::isfinite(v) && v >= 0.0; };
  if (m.kind == 0) {
    if (!nonneg(m.our)) return 5;
    rate = m.our;
  } else if (m.kind == 1) {
    if (!nonneg(m.our_max)) return 5;
    if (!(std::isfinite(m.ks) && m.ks > 0.0 && std::isfinite(m.c_ref) && m.c_ref > 0.0)) return 5;
    const double cs = c / m.c_ref;
    rate = m.our_max * cs / (m.ks + cs);
  } else {
    if (!nonneg(m.specific_our)) return 5;
    if (!density || !nonneg(*density)) return 5;
    rate = m.specific_our * *density;
  }
  return 0;
}

struct OurLedger {  // OurLedger (reaction.rs:23-27)
  double cumulative_kmol_consumed = 0.0, last_step_kmol_consumed = 0.0;
};

// apply_oxygen_reaction_source (reaction.rs:95-137)
inline int apply_oxygen_reaction_source(double* c, const double* vol, size_t n, double dt, const OurModel& m,
                                        const double* density, OurLedger& ledger, OxygenDiag& diag) {
  if (!(std::isfinite(dt) && dt >= 0.0)) return 3;
  double consumed = 0.0;
  for (size_t i = 0; i < n; ++i) {
    if (!(std::isfinite(vol[i]) && vol[i] > 0.0)) return 1;
    double rate = 0.0;
    const int e = oxygen_uptake_rate(m, c[i], density ? density + i : nullptr, rate);
    if (e) return e;
    c[i] -= rate * dt;
    consumed += rate * vol[i] * dt;
  }
  diag = clip_negative_concentrations(c, n);
  ledger.last_step_kmol_consumed = consumed;
  ledger.cumulative_kmol_consumed += consumed;
  return 0;
}

}  // namespace lbmo
