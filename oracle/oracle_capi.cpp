// C entry points over the CPU oracle (test infrastructure only; see
// lbm_oracle.hpp). Loaded by tests/ through ctypes via oracle/oracle.py and
// timed as the CPU baseline by bench.py. Never linked into the product.
#include <memory>
#include <type_traits>

#include "lbm_oracle.hpp"

using namespace lbmo;

namespace {

struct AnySolver {
  virtual ~AnySolver() = default;
  virtual void step(int n) = 0;
  virtual void stage_in(const double* f) = 0;
  virtual void stage_out(double* f) const = 0;
  virtual void init_with(const double* rho, const double* u) = 0;
  virtual void read_moments(double* r, double* ux, double* uy, double* uz) const = 0;
  virtual double reduce(int kind, int axis) const = 0;
  virtual IbmDiag ibm(const Body& b, const IbmConfig& c) = 0;
  virtual void clear_force() = 0;
  virtual void get_force(double* out) const = 0;
  virtual int scalar_enable(int q, double d) = 0;
  virtual void scalar_set(int k, const double* v) = 0;
  virtual void scalar_get(int k, double* v) const = 0;
  virtual size_t cells() const = 0;
  virtual const uint8_t* solid() const = 0;
  virtual int q() const = 0;
  virtual void set_smagorinsky(double cs) = 0;
  virtual void set_free_slip_top(bool on) = 0;
  virtual bool set_store16(int mode) = 0;
  virtual void strain_rate(double* s6, double* gamma) const = 0;
  virtual void set_omega_field(const double* v) = 0;
  virtual void velocity_gradient(double* g9) const = 0;
  virtual void wale(bool has_max, double tau_max, double* nu_t, double* diag) = 0;
  // Raw solver state for the checkpoint restatement (fields.rs SoaFields:
  // f, ftmp, rho/ux/uy/uz, force_field, scalars; Solver::time).
  virtual void state_get(double* f, double* ftmp, double* mom, int* has_ff, double* ff, uint64_t* time) const = 0;
  virtual void state_set(const double* f, const double* ftmp, const double* mom, int has_ff, const double* ff,
                         uint64_t time) = 0;
  virtual int scalar_count() const = 0;
  virtual void scalar_raw_get(int k, int* q, double* d, double* h, double* htmp, double* conc) const = 0;
  virtual void scalar_raw_set(int k, double d, const double* h, const double* htmp, const double* conc) = 0;
};

template <class L, class T>
struct Impl final : AnySolver {
  Solver<L, T> s;
  Impl(const int d[3], const bool p[3], const StepParams& sp, const uint8_t* so, const double* wu)
      : s(d, p, sp, so, wu) {}
  void step(int n) override { s.run(n); }
  void set_smagorinsky(double cs) override { s.params.smagorinsky_cs = cs; }
  void set_free_slip_top(bool on) override { s.params.free_slip_top = on; }
  // 16-bit storage mode (fp32 arithmetic only).
  bool set_store16(int mode) override {
    if (mode != 0 && !std::is_same<T, float>::value) return false;
    if (mode < 0 || mode > 2) return false;
    s.params.store16 = mode;
    return true;
  }
  void stage_in(const double* f) override {
    const int m = s.params.store16;
    for (size_t i = 0; i < s.f.size(); ++i) s.f[i] = m ? T(stage16(m, float(f[i]))) : T(f[i]);
    s.update_moments();
  }
  void stage_out(double* f) const override {
    for (size_t i = 0; i < s.f.size(); ++i) f[i] = double(s.f[i]);
  }
  void init_with(const double* r, const double* u) override {
    s.init_with(r, u);
    if (const int m = s.params.store16) {  // staged into 16-bit storage
      for (auto& v : s.f) v = T(stage16(m, float(v)));
      s.update_moments();
    }
  }
  void read_moments(double* r, double* ux, double* uy, double* uz) const override {
    for (size_t c = 0; c < s.n; ++c) {
      if (r) r[c] = double(s.rho[c]);
      if (ux) ux[c] = double(s.ux[c]);
      if (uy) uy[c] = double(s.uy[c]);
      if (uz) uz[c] = double(s.uz[c]);
    }
  }
  double reduce(int kind, int axis) const override { return s.reduce(kind, axis); }
  IbmDiag ibm(const Body& b, const IbmConfig& c) override { return s.apply_rotating_ibm(b, c); }
  void clear_force() override { s.clear_body_force_field(); }
  void get_force(double* out) const override {
    for (size_t i = 0; i < 3 * s.n; ++i) out[i] = s.has_force_field ? double(s.force_field[i]) : 0.0;
  }
  int scalar_enable(int q, double d) override {
    s.enable_scalar(q, d);
    return int(s.scalars.size()) - 1;
  }
  void scalar_set(int k, const double* v) override { s.set_scalar(k, v); }
  void scalar_get(int k, double* v) const override {
    const auto& sc = s.scalars.at(k);
    for (size_t c = 0; c < s.n; ++c) v[c] = double(sc.conc[c]);
  }
  size_t cells() const override { return s.n; }
  const uint8_t* solid() const override { return s.solid.data(); }
  int q() const override { return L::Q; }
  void set_omega_field(const double* v) override { s.set_omega_field(v); }
  void velocity_gradient(double* g9) const override {
    for (size_t c = 0; c < s.n; ++c) {
      T g[3][3];
      s.velocity_gradient_at(c, g);
      for (int i = 0; i < 9; ++i) g9[9 * c + i] = double(g[i / 3][i % 3]);
    }
  }
  void wale(bool has_max, double tau_max, double* nu_t, double* diag) override {
    std::vector<T> v;
    s.wale_update(has_max, tau_max, v, diag);
    if (nu_t)
      for (size_t c = 0; c < s.n; ++c) nu_t[c] = double(v[c]);
  }
  void state_get(double* f, double* ftmp, double* mom, int* has_ff, double* ff, uint64_t* time) const override {
    for (size_t i = 0; i < s.f.size(); ++i) {
      f[i] = double(s.f[i]);
      ftmp[i] = double(s.ftmp[i]);
    }
    for (size_t c = 0; c < s.n; ++c) {
      mom[c] = double(s.rho[c]);
      mom[s.n + c] = double(s.ux[c]);
      mom[2 * s.n + c] = double(s.uy[c]);
      mom[3 * s.n + c] = double(s.uz[c]);
    }
    *has_ff = s.has_force_field ? 1 : 0;
    for (size_t i = 0; i < 3 * s.n; ++i) ff[i] = s.has_force_field ? double(s.force_field[i]) : 0.0;
    *time = s.time;
  }
  void state_set(const double* f, const double* ftmp, const double* mom, int has_ff, const double* ff,
                 uint64_t time) override {
    for (size_t i = 0; i < s.f.size(); ++i) {
      s.f[i] = T(f[i]);
      s.ftmp[i] = T(ftmp[i]);
    }
    for (size_t c = 0; c < s.n; ++c) {
      s.rho[c] = T(mom[c]);
      s.ux[c] = T(mom[s.n + c]);
      s.uy[c] = T(mom[2 * s.n + c]);
      s.uz[c] = T(mom[3 * s.n + c]);
    }
    s.has_force_field = has_ff != 0;
    s.force_field.assign(has_ff ? 3 * s.n : 0, T(0));
    if (has_ff)
      for (size_t i = 0; i < 3 * s.n; ++i) s.force_field[i] = T(ff[i]);
    s.time = time;
  }
  int scalar_count() const override { return int(s.scalars.size()); }
  void scalar_raw_get(int k, int* q, double* d, double* h, double* htmp, double* conc) const override {
    const auto& sc = s.scalars.at(size_t(k));
    *q = sc.q;
    *d = sc.diffusivity;
    if (h)
      for (size_t i = 0; i < sc.h.size(); ++i) h[i] = double(sc.h[i]);
    if (htmp)
      for (size_t i = 0; i < sc.htmp.size(); ++i) htmp[i] = double(sc.htmp[i]);
    if (conc)
      for (size_t c = 0; c < sc.conc.size(); ++c) conc[c] = double(sc.conc[c]);
  }
  void scalar_raw_set(int k, double d, const double* h, const double* htmp, const double* conc) override {
    auto& sc = s.scalars.at(size_t(k));
    sc.diffusivity = d;
    for (size_t i = 0; i < sc.h.size(); ++i) sc.h[i] = T(h[i]);
    for (size_t i = 0; i < sc.htmp.size(); ++i) sc.htmp[i] = T(htmp[i]);
    for (size_t c = 0; c < sc.conc.size(); ++c) sc.conc[c] = T(conc[c]);
  }
  void strain_rate(double* s6, double* gamma) const override {
    for (size_t c = 0; c < s.n; ++c) {
      T v[6];
      s.strain_rate_at(c, v);
      if (s6)
        for (int k = 0; k < 6; ++k) s6[6 * c + k] = double(v[k]);
      if (gamma) gamma[c] = double(s.shear_rate_at(c));
    }
  }
};

void set_err(char* err, int len, const char* msg) {
  if (err && len > 0) {
    std::strncpy(err, msg, size_t(len) - 1);
    err[len - 1] = 0;
  }
}

void fill_diag(const IbmDiag& d, double* out) {
  // layout: iterations, slip_max, slip_rms, slip_max_rel, slip_rms_rel,
  // torque[3], fluid_force[3], marker_force[3], momentum_error_rel
  out[0] = d.iterations;
  out[1] = d.slip_max;
  out[2] = d.slip_rms;
  out[3] = d.slip_max_rel;
  out[4] = d.slip_rms_rel;
  for (int a = 0; a < 3; ++a) {
    out[5 + a] = d.torque[a];
    out[8 + a] = d.fluid_force[a];
    out[11 + a] = d.marker_force[a];
  }
  out[14] = d.momentum_error_rel;
}

Body make_body(const double* pos, const double* w, long nm, const double* center,
               const double* omega) {
  Body b;
  for (int a = 0; a < 3; ++a) {
    b.center[a] = center[a];
    b.omega[a] = omega[a];
  }
  b.pos.assign(pos, pos + 3 * nm);
  b.weight.assign(w, w + nm);
  return b;
}

}  // namespace

extern "C" {

void* lbmo_create(int q, int real_bits, const int* dims, const int* periodic, int collision,
                  double magic, double omega_shear, double nu, const double* force,
                  const uint8_t* solid, const double* wall_u, char* err, int errlen) {
  try {
    StepParams sp;
    sp.collision = collision;
    sp.magic = magic;
    sp.omega_shear_cfg = omega_shear;
    sp.nu = nu;
    omegas(collision, magic, nu, &sp.omega_p, &sp.omega_m);
    for (int a = 0; a < 3; ++a) sp.force[a] = force ? force[a] : 0.0;
    bool per[3] = {periodic[0] != 0, periodic[1] != 0, periodic[2] != 0};
    if (q == 19 && real_bits == 64) return new Impl<D3Q19, double>(dims, per, sp, solid, wall_u);
    if (q == 19 && real_bits == 32) return new Impl<D3Q19, float>(dims, per, sp, solid, wall_u);
    if (q == 27 && real_bits == 64) return new Impl<D3Q27, double>(dims, per, sp, solid, wall_u);
    if (q == 27 && real_bits == 32) return new Impl<D3Q27, float>(dims, per, sp, solid, wall_u);
    set_err(err, errlen, "unsupported lattice/precision");
  } catch (const std::exception& e) {
    set_err(err, errlen, e.what());
  }
  return nullptr;
}

void lbmo_destroy(void* h) { delete static_cast<AnySolver*>(h); }
// Switch the optional Smagorinsky subgrid model on (cs > 0) or off (0).
void lbmo_set_smagorinsky(void* h, double cs) { static_cast<AnySolver*>(h)->set_smagorinsky(cs); }
// Free-slip (specular) top wall on (nonzero) or off.
void lbmo_set_free_slip_top(void* h, int on) { static_cast<AnySolver*>(h)->set_free_slip_top(on != 0); }
void lbmo_step(void* h, int n) { static_cast<AnySolver*>(h)->step(n); }
void lbmo_stage_in(void* h, const double* f) { static_cast<AnySolver*>(h)->stage_in(f); }
void lbmo_stage_out(void* h, double* f) { static_cast<AnySolver*>(h)->stage_out(f); }
void lbmo_init_with(void* h, const double* r, const double* u) { static_cast<AnySolver*>(h)->init_with(r, u); }
void lbmo_read_moments(void* h, double* r, double* ux, double* uy, double* uz) {
  static_cast<AnySolver*>(h)->read_moments(r, ux, uy, uz);
}
double lbmo_reduce(void* h, int kind, int axis) { return static_cast<AnySolver*>(h)->reduce(kind, axis); }
void lbmo_clear_force_field(void* h) { static_cast<AnySolver*>(h)->clear_force(); }
void lbmo_get_force_field(void* h, double* out) { static_cast<AnySolver*>(h)->get_force(out); }

int lbmo_ibm_apply(void* h, const double* pos, const double* w, long nm, const double* center,
                   const double* omega, int max_it, double tol, int radius, double relax,
                   double* diag_out, char* err, int errlen) {
  try {
    Body b = make_body(pos, w, nm, center, omega);
    IbmConfig c{max_it, tol, radius, relax};
    fill_diag(static_cast<AnySolver*>(h)->ibm(b, c), diag_out);
    return 0;
  } catch (const std::exception& e) {
    set_err(err, errlen, e.what());
    return -1;
  }
}

// The IBM force update alone, on caller-provided rho / u_now (d = 2 or 3).
int lbmo_ibm_direct_forcing(const int* dims, int d, const uint8_t* solid, const double* rho,
                            const double* u_now, const double* pos, const double* w, long nm,
                            const double* center, const double* omega, int max_it, double tol,
                            int radius, double relax, double* spread, double* diag_out, char* err,
                            int errlen) {
  try {
    Body b = make_body(pos, w, nm, center, omega);
    IbmConfig c{max_it, tol, radius, relax};
    fill_diag(ibm_direct_forcing(dims, d, solid, rho, u_now, b, c, spread), diag_out);
    return 0;
  } catch (const std::exception& e) {
    set_err(err, errlen, e.what());
    return -1;
  }
}

// Marker stencil (x, y, z, w) rows; returns the point count.
int lbmo_marker_stencil(const double* p, const int* dims, int d, int radius, double* out) {
  auto st = marker_stencil(p, dims, d, radius);
  for (size_t i = 0; i < st.size(); ++i) {
    out[4 * i + 0] = st[i].x;
    out[4 * i + 1] = st[i].y;
    out[4 * i + 2] = st[i].z;
    out[4 * i + 3] = st[i].w;
  }
  return int(st.size());
}

int lbmo_scalar_enable(void* h, int q, double diffusivity) {
  try {
    return static_cast<AnySolver*>(h)->scalar_enable(q, diffusivity);
  } catch (...) {
    return -1;
  }
}
void lbmo_scalar_set(void* h, int k, const double* v) { static_cast<AnySolver*>(h)->scalar_set(k, v); }
void lbmo_scalar_get(void* h, int k, double* v) { static_cast<AnySolver*>(h)->scalar_get(k, v); }

void lbmo_wall_rims(int d, const int* dims, const int* is_wall, const double* u, uint8_t* solid,
                    double* wall_u) {
  bool w[6];
  double uu[6][3];
  for (int f = 0; f < 6; ++f) {
    w[f] = is_wall[f] != 0;
    for (int a = 0; a < 3; ++a) uu[f][a] = u[3 * f + a];
  }
  build_wall_rims(d, dims, w, uu, solid, wall_u);
}

// Stirred tank (cylinder + optional 4 baffles + one radial impeller, SI
// inputs). Returns the marker count; when it exceeds max_markers only the
// count is returned. kind: 0 Rushton, 1 pitched blade.
long lbmo_build_tank2(const int* dims, double dx, double vessel_d, double liquid_h, double baffle_w, double baffle_t,
                      int kind, double imp_d, double clearance, int blades, double omega_z, double spacing,
                      uint8_t* solid, uint8_t* baffle, double* wall_velocity, double* marker_pos, double* marker_w,
                      long max_markers, double* center, double* omega, char* err, int errlen);

long lbmo_build_tank(const int* dims, double dx, double vessel_d, double liquid_h,
                     double baffle_w, double baffle_t, int kind, double imp_d, double clearance,
                     int blades, double omega_z, uint8_t* solid, uint8_t* baffle,
                     double* wall_velocity, double* marker_pos, double* marker_w, long max_markers,
                     double* center, double* omega, char* err, int errlen) {
  return lbmo_build_tank2(dims, dx, vessel_d, liquid_h, baffle_w, baffle_t, kind, imp_d, clearance, blades, omega_z,
                          0.7, solid, baffle, wall_velocity, marker_pos, marker_w, max_markers, center, omega, err,
                          errlen);
}

// Kind 2: the device library's flat-blade turbine at `spacing` cells.
long lbmo_build_tank2(const int* dims, double dx, double vessel_d, double liquid_h, double baffle_w, double baffle_t,
                      int kind, double imp_d, double clearance, int blades, double omega_z, double spacing,
                      uint8_t* solid, uint8_t* baffle, double* wall_velocity, double* marker_pos, double* marker_w,
                      long max_markers, double* center, double* omega, char* err, int errlen) {
  try {
    TankGeometry g;
    for (int a = 0; a < 3; ++a) g.dims[a] = dims[a];
    g.dx_m = dx;
    size_t n = size_t(dims[0]) * dims[1] * dims[2];
    g.solid.assign(n, 0);
    g.baffle_mask.assign(n, 0);
    g.wall_velocity.assign(3 * n, 0.0);
    apply_cylindrical_tank_mask(dims, dx, vessel_d, liquid_h, g.solid.data());
    if (baffle_w > 0.0)
      apply_baffle_mask(dims, dx, vessel_d, liquid_h, baffle_w, baffle_t, g.solid.data(),
                        g.baffle_mask.data());
    if (kind == 2)
      build_flat_blade_turbine(dims, dx, imp_d, clearance, blades, spacing, omega_z, g);
    else
      build_radial_impeller(dims, dx, vessel_d, liquid_h, kind, imp_d, clearance, blades, omega_z, g);
    stamp_impeller_wall_velocity(g);
    long m = long(g.marker_weight.size());
    if (solid) std::memcpy(solid, g.solid.data(), n);
    if (baffle) std::memcpy(baffle, g.baffle_mask.data(), n);
    if (wall_velocity) std::memcpy(wall_velocity, g.wall_velocity.data(), 3 * n * sizeof(double));
    if (m <= max_markers) {
      if (marker_pos) std::memcpy(marker_pos, g.marker_pos.data(), 3 * m * sizeof(double));
      if (marker_w) std::memcpy(marker_w, g.marker_weight.data(), m * sizeof(double));
    }
    for (int a = 0; a < 3; ++a) {
      if (center) center[a] = g.center[a];
      if (omega) omega[a] = g.omega[a];
    }
    return m;
  } catch (const std::exception& e) {
    set_err(err, errlen, e.what());
    return -1;
  }
}

int lbmo_set_store16(void* h, int mode) { return static_cast<AnySolver*>(h)->set_store16(mode) ? 0 : -1; }

// 16-bit codecs over n values: mode 1 the reference's host binary16 codec
// (encode then decode), mode 2 bfloat16 nearest-even, mode 3 binary16
// nearest-even (the device store).
void lbmo_codec16(int mode, const float* in, float* out, long n) {
  for (long i = 0; i < n; ++i)
    out[i] = mode == 1 ? f16_bits_to_f32(f32_to_f16_bits(in[i])) : (mode == 2 ? round_bf16_rne(in[i]) : round_f16_rne(in[i]));
}
void lbmo_f16_bits(const float* in, uint16_t* out, long n) {
  for (long i = 0; i < n; ++i) out[i] = f32_to_f16_bits(in[i]);
}

// Runner power QOIs from a per-step lattice torque series: out = power_qois
// of the mean SI torque (runner_mean_torque); returns records used or -1.
long lbmo_runner_power(const double* torque_lu, long executed, long run_steps, long probe_every, double rho, double dx,
                       double dt, double omega, double d, double volume, double* out) {
  long used = 0;
  const double t = runner_mean_torque(torque_lu, executed, run_steps, probe_every, rho, dx, dt, &used);
  if (!std::isfinite(t)) return -1;
  try {
    PowerQoi p = power_qois(t, omega, rho, d, volume);
    out[0] = p.torque_n_m;
    out[1] = p.power_w;
    out[2] = p.rotational_speed_hz;
    out[3] = p.np;
    out[4] = p.p_over_v_w_m3;
  } catch (...) {
    return -1;
  }
  return used;
}

int lbmo_unit_report(const double* in7, const int* grid, double d_scalar, double* out13, unsigned* bits2) {
  return unit_report(in7[0], in7[1], in7[2], in7[3], in7[4], in7[5], in7[6], grid, d_scalar, out13, &bits2[0],
                     &bits2[1])
             ? 0
             : -1;
}

void lbmo_top_hat_pulse(const int* dims, const uint8_t* solid, double dx, const double* center, double radius,
                        double conc, double* values) {
  top_hat_pulse(dims, solid, dx, center, radius, conc, values);
}

int lbmo_power_qois(double torque, double omega, double rho, double d, double volume, double* out) {
  try {
    PowerQoi p = power_qois(torque, omega, rho, d, volume);
    out[0] = p.torque_n_m;
    out[1] = p.power_w;
    out[2] = p.rotational_speed_hz;
    out[3] = p.np;
    out[4] = p.p_over_v_w_m3;
    return 0;
  } catch (...) {
    return -1;
  }
}

double lbmo_scalar_cv(const double* v, const uint8_t* include, long n) { return scalar_cv(v, include, size_t(n)); }

int lbmo_mixing_time(const double* t, const double* cv, long n, double* out) {
  return mixing_time_from_cv(t, cv, size_t(n), out) ? 0 : -1;
}

// Runner loop (crates/lbm-cli/src/runner.rs:1079-1129): per step clear the
// force field, apply the impeller IBM with the given config, step, record
// torque_lu = -diag.torque[2] and the fluid force; every probe_every steps
// (and the last) record the scalar CV of scalar `k` (if k >= 0) over fluid
// cells. Returns the executed step count (short when the f64 mass becomes
// non-finite at a multiple of 1000 steps).
long lbmo_run_tank(void* h, const double* pos, const double* w, long nm, const double* center,
                   const double* omega, int max_it, double tol, int radius, double relax, long steps,
                   long probe_every, int k, double* torque_lu, double* fluid_force, double* cv_out,
                   double* ibm_iters) {
  AnySolver* s = static_cast<AnySolver*>(h);
  Body b = make_body(pos, w, nm, center, omega);
  IbmConfig c{max_it, tol, radius, relax};
  size_t n = s->cells();
  std::vector<double> conc(k >= 0 ? n : 0);
  std::vector<uint8_t> include(n);
  for (size_t i = 0; i < n; ++i) include[i] = s->solid()[i] ? 0 : 1;
  long executed = 0;
  for (long step = 1; step <= steps; ++step) {
    s->clear_force();
    IbmDiag d = s->ibm(b, c);
    s->step(1);
    executed = step;
    if (torque_lu) torque_lu[step - 1] = -d.torque[2];
    if (fluid_force)
      for (int a = 0; a < 3; ++a) fluid_force[3 * (step - 1) + a] = d.fluid_force[a];
    if (ibm_iters) ibm_iters[step - 1] = d.iterations;
    if (k >= 0 && cv_out && (step % probe_every == 0 || step == steps)) {
      s->scalar_get(k, conc.data());
      cv_out[step - 1] = scalar_cv(conc.data(), include.data(), n);
    }
    if (step % 1000 == 0) {
      double m = s->reduce(RED_FLUID_CELLS, 0) + s->reduce(RED_MASS_DEV, 0);
      if (!std::isfinite(m)) break;
    }
  }
  return executed;
}

// Solver::set_omega_field (NULL clears), gather_velocity_gradient (n x 9,
// row-major g[i][j] = du_i/dx_j) and WaleLes::update (tau_eff_max NaN for
// no bound; diag: 5 values).
void lbmo_set_omega_field(void* h, const double* v) { static_cast<AnySolver*>(h)->set_omega_field(v); }
void lbmo_state_get(void* h, double* f, double* ftmp, double* mom, int* has_ff, double* ff, uint64_t* time) {
  static_cast<AnySolver*>(h)->state_get(f, ftmp, mom, has_ff, ff, time);
}
void lbmo_state_set(void* h, const double* f, const double* ftmp, const double* mom, int has_ff, const double* ff,
                    uint64_t time) {
  static_cast<AnySolver*>(h)->state_set(f, ftmp, mom, has_ff, ff, time);
}
int lbmo_scalar_count(void* h) { return static_cast<AnySolver*>(h)->scalar_count(); }
void lbmo_scalar_raw_get(void* h, int k, int* q, double* d, double* hh, double* htmp, double* conc) {
  static_cast<AnySolver*>(h)->scalar_raw_get(k, q, d, hh, htmp, conc);
}
void lbmo_scalar_raw_set(void* h, int k, double d, const double* hh, const double* htmp, const double* conc) {
  static_cast<AnySolver*>(h)->scalar_raw_set(k, d, hh, htmp, conc);
}
void lbmo_gather_velocity_gradient(void* h, double* g9) { static_cast<AnySolver*>(h)->velocity_gradient(g9); }
void lbmo_wale_update(void* h, double tau_eff_max, double* nu_t, double* diag) {
  static_cast<AnySolver*>(h)->wale(std::isfinite(tau_eff_max), tau_eff_max, nu_t, diag);
}

// Native strain rate and shear rate of every cell (solver.rs:5464-5599).
void lbmo_gather_strain_rate(void* h, double* s6, double* gamma) {
  static_cast<AnySolver*>(h)->strain_rate(s6, gamma);
}

// stress.rs compute_stress_field over SI velocity fields; any output NULL.
void lbmo_compute_stress_field(const int* dims, const double* ux, const double* uy, const double* uz,
                               const uint8_t* solid, double dx, const double* mu, double* s6, double* gamma,
                               double* vstress, double* s2, double* vm) {
  const auto st = compute_stress_field(dims, ux, uy, uz, solid, dx, mu);
  for (size_t i = 0; i < st.size(); ++i) {
    if (s6)
      for (int k = 0; k < 6; ++k) s6[6 * i + k] = st[i].s[k];
    if (gamma) gamma[i] = st[i].gamma_dot;
    if (vstress) vstress[i] = st[i].viscous_stress_pa;
    if (s2) s2[i] = st[i].second_invariant_s2;
    if (vm) vm[i] = st[i].von_mises_proxy_pa;
  }
}

// stress.rs percentile_summary; 1 with out filled, 0 when no finite value.
int lbmo_percentile_summary(const double* v, long n, int has_threshold, double threshold, double* out) {
  return percentile_summary(v, size_t(n), has_threshold != 0, threshold, out) ? 1 : 0;
}

// stress.rs wall_shear_proxy; returns the count, fills up to capacity
// entries (cell, tau_w, y+, |u_par|, normal x3).
long lbmo_wall_shear_proxy(const int* dims, const double* ux, const double* uy, const double* uz,
                           const uint8_t* solid, const double* wall_u, double dx, double rho, double mu,
                           long capacity, int64_t* cell, double* tau, double* yplus, double* upar, double* normal) {
  const auto w = wall_shear_proxy(dims, ux, uy, uz, solid, wall_u, dx, rho, mu);
  for (size_t i = 0; i < w.size() && long(i) < capacity; ++i) {
    cell[i] = int64_t(w[i].cell_index);
    tau[i] = w[i].tau_w_pa;
    yplus[i] = w[i].y_plus;
    upar[i] = w[i].u_parallel_m_s;
    for (int k = 0; k < 3; ++k) normal[3 * i + k] = w[i].normal[k];
  }
  return long(w.size());
}

// oxygen.rs / reaction.rs over f64 arrays (c updated in place). ledger in /
// out: {cumulative, last step, source integral, active cells} for the
// transfer, {cumulative, last step} for the uptake; diag out: {clipped
// cells, clipped fraction, min before clip}. Returns 0 or the error code.
int lbmo_interfacial_flux(double* c, const double* c_star, const double* area, const double* vol, long n, double dt,
                          double kl, double* ledger, double* diag) {
  OxygenLedger l;
  l.cumulative_mol = ledger[0];
  OxygenDiag d;
  const int e = apply_interfacial_flux_sources(c, c_star, area, vol, size_t(n), dt, kl, l, d);
  if (e) return e;
  ledger[0] = l.cumulative_mol;
  ledger[1] = l.last_step_mol;
  ledger[2] = l.source_integral_mol_s;
  ledger[3] = double(l.active_interface_cells);
  diag[0] = double(d.clipped_cells);
  diag[1] = d.clipped_fraction;
  diag[2] = d.min_before_clip;
  return 0;
}

int lbmo_oxygen_uptake(double* c, const double* vol, long n, double dt, int kind, const double* params,
                       const double* density, double* ledger, double* diag) {
  OurModel m;
  m.kind = kind;
  m.our = params[0];
  m.our_max = params[1];
  m.ks = params[2];
  m.c_ref = params[3];
  m.specific_our = params[4];
  OurLedger l;
  l.cumulative_kmol_consumed = ledger[0];
  OxygenDiag d;
  const int e = apply_oxygen_reaction_source(c, vol, size_t(n), dt, m, density, l, d);
  if (e) return e;
  ledger[0] = l.cumulative_kmol_consumed;
  ledger[1] = l.last_step_kmol_consumed;
  diag[0] = double(d.clipped_cells);
  diag[1] = d.clipped_fraction;
  diag[2] = d.min_before_clip;
  return 0;
}

double lbmo_henry_equilibrium(double h, double p) { return henry_equilibrium(h, p); }
double lbmo_interfacial_area_density(double phi, const double* g, double w) {
  return interfacial_area_density(phi, g, w);
}

}  // extern "C"

extern "C" {

// CollisionKind::omegas (params.rs:205-217): out = {omega_p, omega_m}.
void lbmo_omegas(int kind, double magic, double nu, double* out) { omegas(kind, magic, nu, &out[0], &out[1]); }

// Lattice tables: C (q x 3 int8), W (q), OPP (q). Returns Q or -1.
int lbmo_lattice(int q, int8_t* c, double* w, int* opp) {
  auto emit = [&](auto lat) {
    using L = decltype(lat);
    const auto& tb = tables<L>();
    for (int k = 0; k < L::Q; ++k) {
      for (int a = 0; a < 3; ++a) c[3 * k + a] = L::C[k][a];
      w[k] = L::W[k];
      opp[k] = tb.opp[k];
    }
    return L::Q;
  };
  if (q == 7) return emit(D3Q7{});
  if (q == 19) return emit(D3Q19{});
  if (q == 27) return emit(D3Q27{});
  return -1;
}

}  // extern "C"

namespace {
template <class L, class T>
void collide_cells_impl(int kind, double op, double om, double os, long n, double* f,
                        const double* rho, const double* u, const double* ff) {
  StepParams sp;
  sp.collision = kind;
  sp.omega_p = op;
  sp.omega_m = om;
  sp.omega_shear_cfg = os;
  KParams<T> k = make_kparams<L, T>(sp);
  std::vector<T> ft(size_t(L::Q) * n);
  for (size_t i = 0; i < ft.size(); ++i) ft[i] = T(f[i]);
  for (long c = 0; c < n; ++c) {
    T r = T(rho[c]);
    T uu[3] = {T(u[3 * c]), T(u[3 * c + 1]), T(u[3 * c + 2])};
    T fv[3] = {T(0), T(0), T(0)};
    if (ff)
      for (int a = 0; a < 3; ++a) fv[a] = k.force[a] + T(ff[3 * c + a]);
    if (kind == CENTRAL_MOMENT)
      collide_cm_cell<L, T>(&ft[c], size_t(n), r, uu, fv, k);
    else
      collide_trt_cell<L, T>(&ft[c], size_t(n), r, uu, fv, k.omega_p, k.cp, ff != nullptr, k);
  }
  for (size_t i = 0; i < ft.size(); ++i) f[i] = double(ft[i]);
}
}  // namespace

extern "C" {
// Collide `n` independent cells in place (kernels.rs:129-160, 406-533):
// f is q-major (q x n) in the f64 view of precision `real_bits`; ff is an
// optional n x 3 per-cell force field.
int lbmo_collide_cells(int q, int real_bits, int kind, double op, double om, double os, long n,
                       double* f, const double* rho, const double* u, const double* ff) {
  if (q == 19 && real_bits == 64) collide_cells_impl<D3Q19, double>(kind, op, om, os, n, f, rho, u, ff);
  else if (q == 19 && real_bits == 32) collide_cells_impl<D3Q19, float>(kind, op, om, os, n, f, rho, u, ff);
  else if (q == 27 && real_bits == 64) collide_cells_impl<D3Q27, double>(kind, op, om, os, n, f, rho, u, ff);
  else if (q == 27 && real_bits == 32) collide_cells_impl<D3Q27, float>(kind, op, om, os, n, f, rho, u, ff);
  else return -1;
  return 0;
}

// Deviation equilibrium for n cells (kernels.rs:103-121) in precision real_bits.
int lbmo_equilibrium_cells(int q, int real_bits, long n, const double* rho, const double* u, double* feq) {
  auto run = [&](auto lat, auto real) {
    using L = decltype(lat);
    using T = decltype(real);
    StepParams sp;
    KParams<T> k = make_kparams<L, T>(sp);
    for (long c = 0; c < n; ++c) {
      T uu[3] = {T(u[3 * c]), T(u[3 * c + 1]), T(u[3 * c + 2])};
      T out[Q_MAX];
      equilibrium<L, T>(k, T(rho[c]), uu, out);
      for (int qq = 0; qq < L::Q; ++qq) feq[size_t(qq) * n + c] = double(out[qq]);
    }
  };
  if (q == 19 && real_bits == 64) run(D3Q19{}, double{});
  else if (q == 19 && real_bits == 32) run(D3Q19{}, float{});
  else if (q == 27 && real_bits == 64) run(D3Q27{}, double{});
  else if (q == 27 && real_bits == 32) run(D3Q27{}, float{});
  else return -1;
  return 0;
}
}  // extern "C"
