// Host-side runner QOIs and set-up helpers of the stirred-tank path (C++):
// power QOIs from the device torque series, the unit report, the scalar
// top-hat pulse and the backend capability query.
//
// The formulas are the reference's:
//   power_qois                     crates/lbm-core/src/qoi.rs:477-505
//   torque_record_from_ibm         crates/lbm-cli/src/runner.rs:1396-1425
//   write_power_qois (averaging)   crates/lbm-cli/src/runner.rs:1514-1543
//   bioprocess_unit_report         crates/lbm-scenario/src/units.rs:116-325
//   scalar_initial_condition       crates/lbm-cli/src/runner.rs:1317-1377
//   Backend capability hooks       crates/lbm-core/src/backend.rs:162-199, 343
#include <cmath>
#include <cstdint>
#include <cstring>
#include <limits>
#include <stdexcept>
#include <string>

#include "../../include/lbmb.h"

namespace lbmb {
extern thread_local std::string g_last_error;
}

namespace {

constexpr double kTau = 6.283185307179586476925286766559;

struct QoiError : std::runtime_error {
  int code;
  QoiError(int c, const std::string& m) : std::runtime_error(m), code(c) {}
};

template <class F>
int guard(F&& fn) {
  try {
    fn();
    lbmb::g_last_error.clear();
    return LBMB_OK;
  } catch (const QoiError& e) {
    lbmb::g_last_error = e.what();
    return e.code;
  } catch (const std::exception& e) {
    lbmb::g_last_error = e.what();
    return LBMB_ERR_INVALID;
  }
}

bool pos_finite(double v) { return std::isfinite(v) && v > 0.0; }

// f64::powi: binary exponentiation, the low bits first (x^3 = x * x^2,
// x^5 = x * x^4), the products the reference's integer powers round.
double powi(double x, int k) {
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

void power(double torque_n_m, double omega_rad_s, double rho, double d, double volume, lbmb_power_result* out) {
  if (!(std::isfinite(omega_rad_s) && std::isfinite(rho) && std::isfinite(d) && std::isfinite(volume) && rho > 0.0 &&
        d > 0.0 && volume > 0.0))
    throw QoiError(LBMB_ERR_INVALID, "power QOI inputs must be finite and positive where dimensional");
  const double n_hz = omega_rad_s / kTau;
  if (!(n_hz > 0.0)) throw QoiError(LBMB_ERR_INVALID, "rotational speed must be positive for Np/Nq");
  const double p = omega_rad_s * torque_n_m;
  const double denom = rho * powi(n_hz, 3) * powi(d, 5);
  out->torque_n_m = torque_n_m;
  out->power_w = p;
  out->rotational_speed_hz = n_hz;
  out->np = p / denom;
  out->p_over_v_w_m3 = p / volume;
}

}  // namespace

extern "C" {

int lbmb_power_qois(double torque_n_m, double omega_rad_s, double rho_kg_m3, double impeller_diameter_m,
                    double working_volume_m3, lbmb_power_result* out) {
  return guard([&] {
    if (!out) throw QoiError(LBMB_ERR_INVALID, "null output");
    power(torque_n_m, omega_rad_s, rho_kg_m3, impeller_diameter_m, working_volume_m3, out);
  });
}

int lbmb_power_from_torque_series(const double* torque_lu, int64_t executed, int64_t run_steps, int64_t probe_every,
                                  double rho_kg_m3, double dx_m, double dt_s, double omega_rad_s,
                                  double impeller_diameter_m, double working_volume_m3, lbmb_power_result* out,
                                  int64_t* records_used) {
  return guard([&] {
    if (!out || (!torque_lu && executed > 0)) throw QoiError(LBMB_ERR_INVALID, "null argument");
    if (executed < 0 || run_steps < 0 || executed > run_steps)
      throw QoiError(LBMB_ERR_INVALID, "executed steps must lie in [0, run_steps]");
    if (probe_every <= 0) probe_every = 1;
    // torque_record_from_ibm: N m = lattice torque x rho dx^5 / dt^2
    const double torque_scale = rho_kg_m3 * powi(dx_m, 5) / powi(dt_s, 2);
    // the runner records steps with step % probe_every == 0 or the last step
    // of the run; the power QOIs average the records with step >= steps / 2,
    // or every record when none is that late
    const int64_t start = run_steps / 2;
    double sum_window = 0.0, sum_all = 0.0;
    int64_t n_window = 0, n_all = 0;
    for (int64_t step = 1; step <= executed; ++step) {
      if (!(step % probe_every == 0 || step == run_steps)) continue;
      const double t = torque_lu[step - 1] * torque_scale;
      sum_all += t;
      ++n_all;
      if (step >= start) {
        sum_window += t;
        ++n_window;
      }
    }
    if (n_all == 0) throw QoiError(LBMB_ERR_STATE, "no torque records: the power QOIs need at least one");
    const double torque = n_window ? sum_window / double(n_window) : sum_all / double(n_all);
    if (records_used) *records_used = n_window ? n_window : n_all;
    power(torque, omega_rad_s, rho_kg_m3, impeller_diameter_m, working_volume_m3, out);
  });
}

int lbmb_unit_report(const lbmb_unit_input* in, lbmb_unit_mapping* out) {
  return guard([&] {
    if (!in || !out) throw QoiError(LBMB_ERR_INVALID, "null argument");
    auto need = [](const char* name, double v) {
      if (!pos_finite(v)) throw QoiError(LBMB_ERR_INVALID, std::string(name) + " must be finite and positive");
    };
    need("reactor.vessel_diameter_m", in->vessel_diameter_m);
    need("reactor.liquid_height_m", in->liquid_height_m);
    need("impeller.diameter_m", in->impeller_diameter_m);
    need("impeller.rotational_speed_rpm", in->rotational_speed_rpm);
    need("fluids.liquid_density_kg_m3", in->liquid_density_kg_m3);
    need("fluids.liquid_viscosity_pa_s", in->liquid_viscosity_pa_s);
    need("run.dt_s", in->dt_s);
    if (in->grid[0] <= 0 || in->grid[1] <= 0 || in->grid[2] <= 0)
      throw QoiError(LBMB_ERR_INVALID, "run grid dimensions must be positive");
    std::memset(out, 0, sizeof(*out));
    const double n_hz = in->rotational_speed_rpm / 60.0;
    const double u_ref = n_hz * in->impeller_diameter_m;
    const double nu = in->liquid_viscosity_pa_s / in->liquid_density_kg_m3;
    const double dx = in->vessel_diameter_m / double(in->grid[0]);
    out->dx_m = dx;
    out->dt_s = in->dt_s;
    out->u_ref_lu = u_ref * in->dt_s / dx;
    out->nu_lu = nu * in->dt_s / (dx * dx);
    out->tau_lu = 3.0 * out->nu_lu + 0.5;
    out->cs2_lu = 1.0 / 3.0;
    out->mach_lattice = out->u_ref_lu / std::sqrt(out->cs2_lu);
    out->reynolds = in->liquid_density_kg_m3 * n_hz * powi(in->impeller_diameter_m, 2) / in->liquid_viscosity_pa_s;
    out->froude = powi(n_hz, 2) * in->impeller_diameter_m / 9.80665;
    const bool has_d = in->scalar_diffusivity_m2_s > 0.0;
    const double qnan = std::numeric_limits<double>::quiet_NaN();
    out->schmidt = has_d ? nu / in->scalar_diffusivity_m2_s : qnan;
    out->peclet = has_d ? u_ref * in->vessel_diameter_m / in->scalar_diffusivity_m2_s : qnan;
    out->scalar_diffusivity_lu = has_d ? in->scalar_diffusivity_m2_s * in->dt_s / (dx * dx) : qnan;
    out->grid_reynolds = out->u_ref_lu / out->nu_lu;
    uint32_t warn = 0, rej = 0;
    if (out->mach_lattice > 0.30)
      rej |= LBMB_UNIT_MA_LATTICE_TOO_HIGH;
    else if (out->mach_lattice > 0.10)
      warn |= LBMB_UNIT_MA_LATTICE_HIGH;
    if (out->tau_lu <= 0.5)
      rej |= LBMB_UNIT_TAU_NON_POSITIVE_VISCOSITY;
    else if (out->tau_lu <= 0.55)
      warn |= LBMB_UNIT_TAU_NEAR_HALF;
    if (out->grid_reynolds > 15.0) warn |= LBMB_UNIT_GRID_REYNOLDS_HIGH;
    if (has_d && out->nu_lu / out->scalar_diffusivity_lu > 25.0) warn |= LBMB_UNIT_SCALAR_DIFFUSION_UNSTABLE;
    out->warnings = warn;
    out->rejections = rej;
    if (rej) throw QoiError(LBMB_ERR_UNSUPPORTED, "bioprocess unit feasibility rejected the scenario");
  });
}

int lbmb_scalar_top_hat_pulse(const int32_t dims[3], const uint8_t* solid, double dx_m, const double center_m[3],
                              double radius_m, double concentration, double* values) {
  return guard([&] {
    if (!dims || !center_m || !values) throw QoiError(LBMB_ERR_INVALID, "null argument");
    if (dims[0] <= 0 || dims[1] <= 0 || dims[2] <= 0) throw QoiError(LBMB_ERR_INVALID, "grid dimensions must be positive");
    const size_t nxy = size_t(dims[0]) * size_t(dims[1]);
    for (int z = 0; z < dims[2]; ++z)
      for (int y = 0; y < dims[1]; ++y)
        for (int x = 0; x < dims[0]; ++x) {
          const size_t i = size_t(z) * nxy + size_t(y) * size_t(dims[0]) + size_t(x);
          values[i] = 0.0;
          if (solid && solid[i]) continue;
          const double p0 = (double(x) + 0.5) * dx_m, p1 = (double(y) + 0.5) * dx_m, p2 = (double(z) + 0.5) * dx_m;
          const double r =
              std::sqrt(powi(p0 - center_m[0], 2) + powi(p1 - center_m[1], 2) + powi(p2 - center_m[2], 2));
          if (r <= radius_m) values[i] = concentration;
        }
  });
}

int lbmb_scalar_diffusivity_lu(double diffusivity_m2_s, double dt_s, double dx_m, double* d_lu) {
  return guard([&] {
    if (!d_lu) throw QoiError(LBMB_ERR_INVALID, "null output");
    *d_lu = diffusivity_m2_s * dt_s / powi(dx_m, 2);
  });
}

}  // extern "C"
