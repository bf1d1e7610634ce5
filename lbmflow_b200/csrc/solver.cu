// C ABI behind include/lbmb.h: validation (GlobalSpec::validate), engine
// construction and the exception-to-status translation.
//
// Reference boundary: trait Backend<L, T> (crates/lbm-core/src/backend.rs:
// 126-363) driven by Solver<L, T, B, H> (crates/lbm-core/src/solver.rs:
// 1503-1541).
#include "engine.cuh"

namespace lbmb {

thread_local std::string g_last_error;

// ---------------------------------------------------------------------------
// Validation (GlobalSpec::validate, solver.rs:470-600) and construction.
// ---------------------------------------------------------------------------
static void validate(const lbmb_config& c, const uint8_t* solid, const double* wu) {
  if (c.lattice != 19 && c.lattice != 27) invalid("lattice must be 19 (D3Q19) or 27 (D3Q27)");
  if (c.storage < 0 || c.storage > 3) invalid("unknown storage precision");
  if (c.collision < 0 || c.collision > 2) invalid("unknown collision kind");
  if (!std::isfinite(c.nu)) invalid("non-finite parameter: nu");
  if (!(c.nu > 0.0)) invalid("viscosity must be positive");
  if (c.collision == LBMB_TRT && !(std::isfinite(c.magic) && c.magic > 0.0)) invalid("invalid TRT magic parameter");
  if (c.collision == LBMB_CENTRAL_MOMENT &&
      !(std::isfinite(c.omega_shear) && c.omega_shear > 0.0 && c.omega_shear <= 2.0))
    invalid("invalid central-moment shear rate (must be in (0, 2])");
  if (c.collision == LBMB_CENTRAL_MOMENT && c.lattice != 27)
    throw Error(LBMB_ERR_UNSUPPORTED, "central-moment collision is implemented for D3Q27");
  for (int a = 0; a < 3; ++a)
    if (!std::isfinite(c.force[a])) invalid("non-finite parameter: force");
  if (!(std::isfinite(c.smagorinsky_cs) && c.smagorinsky_cs >= 0.0))
    invalid("Smagorinsky constant must be finite and >= 0");
  if (c.free_slip_top && c.periodic[2]) invalid("a free-slip top needs a non-periodic z axis");
  for (int a = 0; a < 3; ++a)
    if (c.dims[a] < 3) invalid("domain too small: every axis needs >= 3 cells");
  const int64_t n = int64_t(c.dims[0]) * c.dims[1] * c.dims[2];
  if (n > (int64_t(1) << 31) - 1) invalid("grid too large for 32-bit force slots");
  auto is_solid = [&](int x, int y, int z) {
    return solid && solid[(int64_t(z) * c.dims[1] + y) * c.dims[0] + x] != 0;
  };
  for (int a = 0; a < 3; ++a) {
    if (c.periodic[a]) continue;
    const int t1 = a == 0 ? 1 : 0, t2 = a == 2 ? 1 : 2;
    for (int side = 0; side < 2; ++side)
      for (int j = 0; j < c.dims[t2]; ++j)
        for (int i = 0; i < c.dims[t1]; ++i) {
          int p[3];
          p[a] = side ? c.dims[a] - 1 : 0;
          p[t1] = i;
          p[t2] = j;
          if (!is_solid(p[0], p[1], p[2]))
            invalid("uncovered face " + std::to_string(2 * a + side) +
                    ": non-periodic faces must be full solid rims");
        }
  }
  if (wu)
    for (int64_t i = 0; i < n; ++i) {
      double sq = 0.0;
      for (int k = 0; k < 3; ++k) {
        if (!std::isfinite(wu[3 * i + k])) invalid("non-finite parameter: velocity");
        sq += wu[3 * i + k] * wu[3 * i + k];
      }
      if (!(std::sqrt(sq) <= 0.3)) invalid("wall velocity exceeds the low-Mach limit 0.3");
    }
}

static EngineBase* make_engine(const lbmb_config& c, const uint8_t* solid, const double* wu) {
  validate(c, solid, wu);
  if (c.lattice == 19) {
    switch (c.storage) {
      case LBMB_STORE_F32: return make_engine_q19_f32(c, solid, wu);
      case LBMB_STORE_F16: return make_engine_q19_f16(c, solid, wu);
      case LBMB_STORE_BF16: return make_engine_q19_bf16(c, solid, wu);
      default: return make_engine_q19_f64(c, solid, wu);
    }
  }
  switch (c.storage) {
    case LBMB_STORE_F32: return make_engine_q27_f32(c, solid, wu);
    case LBMB_STORE_F16: return make_engine_q27_f16(c, solid, wu);
    case LBMB_STORE_BF16: return make_engine_q27_bf16(c, solid, wu);
    default: return make_engine_q27_f64(c, solid, wu);
  }
}

}  // namespace lbmb

struct lbmb_solver {
  std::unique_ptr<lbmb::EngineBase> e;
  int device = 0;
};

struct lbmb_batch {
  std::unique_ptr<lbmb::BatchBase> b;
};

using lbmb::Error;

template <class F>
static int guarded(F&& fn) {
  try {
    fn();
    lbmb::g_last_error.clear();
    return LBMB_OK;
  } catch (const Error& e) {
    lbmb::g_last_error = e.what();
    return e.code;
  } catch (const lbmb::ckpt::Failure& e) {
    lbmb::g_last_error = e.what();
    return LBMB_ERR_CHECKPOINT;
  } catch (const std::bad_alloc&) {
    lbmb::g_last_error = "host allocation failed";
    return LBMB_ERR_NOMEM;
  } catch (const std::exception& e) {
    lbmb::g_last_error = e.what();
    return LBMB_ERR_INVALID;
  }
}

#define NEED(h)                                                          \
  do {                                                                   \
    if (!(h) || !(h)->e) throw Error(LBMB_ERR_INVALID, "null solver");   \
    CK(cudaSetDevice((h)->device));                                      \
  } while (0)

extern "C" {

const char* lbmb_last_error(void) { return lbmb::g_last_error.c_str(); }
const char* lbmb_version(void) { return "lbmflow_b200 0.1 (sm_100a)"; }

int lbmb_create(const lbmb_config* cfg, const uint8_t* solid, const double* wall_u, lbmb_solver** out) {
  return guarded([&] {
    if (!cfg || !out) throw Error(LBMB_ERR_INVALID, "null argument");
    int ndev = 0;
    CK(cudaGetDeviceCount(&ndev));
    if (cfg->device < 0 || cfg->device >= ndev) throw Error(LBMB_ERR_INVALID, "no such CUDA device");
    auto h = std::make_unique<lbmb_solver>();
    h->device = cfg->device;
    h->e.reset(lbmb::make_engine(*cfg, solid, wall_u));
    *out = h.release();
  });
}

int lbmb_destroy(lbmb_solver* h) {
  return guarded([&] {
    if (!h) return;
    cudaSetDevice(h->device);
    delete h;
  });
}

int lbmb_shape(const lbmb_solver* h, int64_t* ncells, int32_t* q) {
  return guarded([&] {
    if (!h || !h->e) throw Error(LBMB_ERR_INVALID, "null solver");
    if (ncells) *ncells = h->e->cells();
    if (q) *q = h->e->q();
  });
}

int lbmb_init_fields(lbmb_solver* h, const double* rho, const double* u) {
  return guarded([&] {
    NEED(h);
    if (!rho || !u) throw Error(LBMB_ERR_INVALID, "null field");
    const int64_t n = h->e->cells();
    for (int64_t c = 0; c < n; ++c) {
      if (!(rho[c] > 0.0 && std::isfinite(rho[c]))) throw Error(LBMB_ERR_INVALID, "init density must be > 0 and finite");
      double sq = 0.0;
      for (int a = 0; a < 3; ++a) {
        if (!std::isfinite(u[3 * c + a])) throw Error(LBMB_ERR_INVALID, "init velocity must be finite");
        sq += u[3 * c + a] * u[3 * c + a];
      }
      if (!(std::sqrt(sq) <= 0.3)) throw Error(LBMB_ERR_INVALID, "init speed exceeds the low-Mach limit 0.3");
    }
    h->e->init_fields(rho, u);
  });
}

int lbmb_stage_in(lbmb_solver* h, const double* f) {
  return guarded([&] {
    NEED(h);
    if (!f) throw Error(LBMB_ERR_INVALID, "null populations");
    h->e->stage_in(f);
  });
}

int lbmb_stage_out(lbmb_solver* h, double* f) {
  return guarded([&] {
    NEED(h);
    if (!f) throw Error(LBMB_ERR_INVALID, "null populations");
    h->e->stage_out(f);
  });
}

int lbmb_step(lbmb_solver* h, int64_t steps) {
  return guarded([&] {
    NEED(h);
    if (steps < 0) throw Error(LBMB_ERR_INVALID, "negative step count");
    h->e->step(steps);
  });
}

int lbmb_run_guarded(lbmb_solver* h, int64_t steps, int64_t check_every, int64_t* completed) {
  int rc = guarded([&] {
    NEED(h);
    if (steps < 0) throw Error(LBMB_ERR_INVALID, "negative step count");
    const int64_t every = std::max<int64_t>(check_every, 1);
    int64_t done = 0;
    while (done < steps) {
      const int64_t chunk = std::min(every, steps - done);
      h->e->step(chunk);
      done += chunk;
      if (completed) *completed = done;
      double r[5];
      h->e->reduce_all(r);
      if (!std::isfinite(r[0] + r[1])) throw Error(LBMB_ERR_DIVERGED, "non-finite mass after step " + std::to_string(done));
    }
  });
  return rc;
}

int lbmb_read_moments(lbmb_solver* h, double* rho, double* ux, double* uy, double* uz) {
  return guarded([&] {
    NEED(h);
    h->e->read_moments(rho, ux, uy, uz);
  });
}

int lbmb_reduce(lbmb_solver* h, int32_t kind, int32_t axis, double* out) {
  return guarded([&] {
    NEED(h);
    if (!out) throw Error(LBMB_ERR_INVALID, "null output");
    if (kind < 0 || kind > 2 || (kind == 2 && (axis < 0 || axis > 2))) throw Error(LBMB_ERR_INVALID, "bad reduction");
    double r[5];
    h->e->reduce_all(r);
    *out = kind == 0 ? r[0] : (kind == 1 ? r[1] : r[2 + axis]);
  });
}

int lbmb_total_mass(lbmb_solver* h, double* out) {
  return guarded([&] {
    NEED(h);
    if (!out) throw Error(LBMB_ERR_INVALID, "null output");
    double r[5];
    h->e->reduce_all(r);
    *out = r[0] + r[1];
  });
}

int lbmb_clear_body_force_field(lbmb_solver* h) {
  return guarded([&] {
    NEED(h);
    h->e->clear_force_field();
  });
}

int lbmb_get_force_field(lbmb_solver* h, double* out) {
  return guarded([&] {
    NEED(h);
    if (!out) throw Error(LBMB_ERR_INVALID, "null output");
    h->e->get_force_field(out);
  });
}

int lbmb_scalar_interfacial_flux(lbmb_solver* h, int32_t k, const double* c_star, double c_star_uniform,
                                 const double* area_density, const double* cell_volume, double cell_volume_uniform,
                                 double dt_s, double kl_m_s, lbmb_oxygen_ledger* ledger, lbmb_oxygen_diag* diag) {
  return guarded([&] {
    NEED(h);
    if (!area_density) lbmb::invalid("area_density must hold one value per cell");
    if (!(std::isfinite(dt_s) && dt_s >= 0.0)) lbmb::invalid("oxygen source time step must be finite and non-negative");
    if (!(std::isfinite(kl_m_s) && kl_m_s > 0.0)) lbmb::invalid("kL must be finite and positive");
    lbmb::OxygenSourceArgs a{};
    a.mode = 0;
    a.dt = dt_s;
    a.kl = kl_m_s;
    a.cstar_u = c_star_uniform;
    a.vol_u = cell_volume_uniform;
    a.cstar = c_star;
    a.area = area_density;
    a.vol = cell_volume;
    double sum = 0.0;
    int64_t active = 0;
    h->e->scalar_oxygen(k, a, &sum, diag, &active);
    if (ledger) {
      ledger->source_integral_mol_s = sum;
      ledger->last_step_mol = sum * dt_s;
      ledger->cumulative_mol += ledger->last_step_mol;
      ledger->active_interface_cells = active;
    }
  });
}

int lbmb_scalar_oxygen_uptake(lbmb_solver* h, int32_t k, const lbmb_our_model* model, const double* cell_density,
                              const double* cell_volume, double cell_volume_uniform, double dt_s,
                              lbmb_our_ledger* ledger, lbmb_oxygen_diag* diag) {
  return guarded([&] {
    NEED(h);
    if (!model) lbmb::invalid("null uptake model");
    if (!(std::isfinite(dt_s) && dt_s >= 0.0)) lbmb::invalid("reaction time step must be finite and non-negative");
    auto nonneg = [](double v) { return std::isfinite(v) && v >= 0.0; };
    lbmb::OxygenSourceArgs a{};
    a.mode = 1;
    a.dt = dt_s;
    a.vol_u = cell_volume_uniform;
    a.vol = cell_volume;
    a.our_kind = model->kind;
    if (model->kind == LBMB_OUR_CONSTANT) {
      if (!nonneg(model->our_kmol_m3_s)) lbmb::invalid("our_kmol_m3_s must be finite and non-negative");
      a.our = model->our_kmol_m3_s;
    } else if (model->kind == LBMB_OUR_MONOD) {
      if (!nonneg(model->our_max)) lbmb::invalid("our_max must be finite and non-negative");
      if (!(std::isfinite(model->ks) && model->ks > 0.0 && std::isfinite(model->c_ref) && model->c_ref > 0.0))
        lbmb::invalid("Monod parameters must be finite and positive where dimensional");
      a.our_max = model->our_max;
      a.ks = model->ks;
      a.c_ref = model->c_ref;
    } else if (model->kind == LBMB_OUR_CELL_DENSITY) {
      if (!nonneg(model->specific_our)) lbmb::invalid("specific_our must be finite and non-negative");
      if (!cell_density) lbmb::invalid("cell-density-scaled OUR requires a cell density field");
      a.specific_our = model->specific_our;
      a.density = cell_density;
    } else {
      lbmb::invalid("unknown uptake model kind");
    }
    double sum = 0.0;
    h->e->scalar_oxygen(k, a, &sum, diag, nullptr);
    if (ledger) {
      ledger->last_step_kmol_consumed = sum;
      ledger->cumulative_kmol_consumed += sum;
    }
  });
}

int lbmb_set_omega_field(lbmb_solver* h, const double* omega) {
  return guarded([&] {
    NEED(h);
    h->e->set_omega_field(omega);
  });
}

int lbmb_gather_velocity_gradient(lbmb_solver* h, double* g9) {
  return guarded([&] {
    NEED(h);
    if (!g9) lbmb::invalid("null output");
    h->e->velocity_gradient(g9);
  });
}

int lbmb_wale_update(lbmb_solver* h, double tau_eff_max, double* nu_t, lbmb_wale_diag* diag) {
  return guarded([&] {
    NEED(h);
    h->e->wale_update(tau_eff_max, nu_t, diag);
  });
}

int lbmb_gather_strain_rate(lbmb_solver* h, double* s6, double* gamma) {
  return guarded([&] {
    NEED(h);
    h->e->strain_rate(s6, gamma);
  });
}

int lbmb_stress_field(lbmb_solver* h, double dx_m, double dt_s, double mu_pa_s, double* s6, double* gamma,
                      double* viscous) {
  return guarded([&] {
    NEED(h);
    h->e->stress_field(dx_m, dt_s, mu_pa_s, s6, gamma, viscous);
  });
}

int lbmb_stress_summary(lbmb_solver* h, double dx_m, double dt_s, double mu_pa_s, double gamma_threshold,
                        double tau_threshold, lbmb_percentiles* gamma, lbmb_percentiles* viscous,
                        double* device_ms) {
  return guarded([&] {
    NEED(h);
    h->e->stress_summary(dx_m, dt_s, mu_pa_s, gamma_threshold, tau_threshold, gamma, viscous, device_ms);
  });
}

int lbmb_wall_shear_proxy(lbmb_solver* h, double dx_m, double dt_s, double rho_kg_m3, double mu_pa_s,
                          lbmb_wall_shear* out, int64_t capacity, int64_t* count) {
  return guarded([&] {
    NEED(h);
    if (!count) throw Error(LBMB_ERR_INVALID, "null count");
    h->e->wall_shear(dx_m, dt_s, rho_kg_m3, mu_pa_s, out, capacity, count);
  });
}

int lbmb_ibm_set_body(lbmb_solver* h, int32_t body, const double* pos, const double* weight, int64_t n,
                      const double center[3], const double omega[3]) {
  return guarded([&] {
    NEED(h);
    if (!pos || !weight || !center || !omega) throw Error(LBMB_ERR_INVALID, "null argument");
    h->e->ibm_set_body(body, pos, weight, n, center, omega);
  });
}

int lbmb_apply_rotating_ibm(lbmb_solver* h, int32_t body, const lbmb_ibm_config* cfg, lbmb_ibm_diag* diag) {
  return guarded([&] {
    NEED(h);
    if (!cfg) throw Error(LBMB_ERR_INVALID, "null IBM config");
    h->e->ibm_apply(body, *cfg, diag);
  });
}

int lbmb_runner_step(lbmb_solver* h, int32_t body, const double* pos, const double* weight, int64_t n,
                     const double center[3], const double omega[3], const lbmb_ibm_config* cfg,
                     lbmb_ibm_diag* diag) {
  return guarded([&] {
    NEED(h);
    if (!pos || !weight || !center || !omega || !cfg) throw Error(LBMB_ERR_INVALID, "null runner step argument");
    h->e->runner_step(body, pos, weight, n, center, omega, *cfg, diag);
  });
}

int lbmb_enable_scalar(lbmb_solver* h, int32_t q, double diffusivity, int32_t* index) {
  return guarded([&] {
    NEED(h);
    const int k = h->e->enable_scalar(q, diffusivity);
    if (index) *index = k;
  });
}

int lbmb_set_scalar_concentration(lbmb_solver* h, int32_t k, const double* c) {
  return guarded([&] {
    NEED(h);
    if (!c) throw Error(LBMB_ERR_INVALID, "null concentration");
    h->e->set_scalar(k, c);
  });
}

int lbmb_gather_scalar_concentration(lbmb_solver* h, int32_t k, double* c) {
  return guarded([&] {
    NEED(h);
    if (!c) throw Error(LBMB_ERR_INVALID, "null concentration");
    h->e->get_scalar(k, c);
  });
}

int lbmb_scalar_cv(lbmb_solver* h, int32_t k, double* cv) {
  return guarded([&] {
    NEED(h);
    if (!cv) throw Error(LBMB_ERR_INVALID, "null output");
    const int64_t n = h->e->cells();
    std::vector<double> c(static_cast<size_t>(n));
    h->e->get_scalar(k, c.data());
    const auto& solid = h->e->solid();
    // qoi::scalar_cv (qoi.rs:507-532): population std / |mean| over fluid cells.
    int64_t cnt = 0;
    double sum = 0.0;
    for (int64_t i = 0; i < n; ++i)
      if (!solid[i]) {
        ++cnt;
        sum += c[i];
      }
    if (cnt == 0) {
      *cv = std::nan("");
      return;
    }
    const double mean = sum / double(cnt);
    if (mean == 0.0) {
      *cv = std::nan("");
      return;
    }
    double var = 0.0;
    for (int64_t i = 0; i < n; ++i)
      if (!solid[i]) {
        const double d = c[i] - mean;
        var += d * d;
      }
    *cv = std::sqrt(var / double(cnt)) / std::fabs(mean);
  });
}

int lbmb_run_impeller(lbmb_solver* h, int32_t body, const lbmb_ibm_config* cfg, int64_t steps, int32_t scalar,
                      int64_t probe_every, double* torque_lu, double* fluid_force, double* cv,
                      int32_t* ibm_iterations) {
  return guarded([&] {
    NEED(h);
    if (!cfg) throw Error(LBMB_ERR_INVALID, "null IBM config");
    if (steps < 0) throw Error(LBMB_ERR_INVALID, "negative step count");
    h->e->run_impeller(body, *cfg, steps, scalar, probe_every, torque_lu, fluid_force, cv, ibm_iterations);
  });
}

int lbmb_run_impeller_status(lbmb_solver* h, int64_t* executed, int32_t* diverged) {
  return guarded([&] {
    NEED(h);
    h->e->run_status(executed, diverged);
  });
}

int lbmb_last_timing(lbmb_solver* h, double* total_ms, double* hydro_ms, int64_t* hydro_launches) {
  return guarded([&] {
    if (!h || !h->e) throw Error(LBMB_ERR_INVALID, "null solver");
    h->e->timing(total_ms, hydro_ms, hydro_launches);
  });
}

int lbmb_set_sweep_kernel(lbmb_solver* h, int32_t kind) {
  return guarded([&] {
    NEED(h);
    if (kind < LBMB_SWEEP_DIRECT || kind > LBMB_SWEEP_WINDOW) lbmb::invalid("unknown sweep kernel kind");
    h->e->set_sweep_kernel(kind);
  });
}

int lbmb_set_sweep_variant(lbmb_solver* h, int32_t even_blocks_per_sm, int32_t odd_blocks_per_sm) {
  return guarded([&] {
    NEED(h);
    h->e->set_sweep_variant(even_blocks_per_sm, odd_blocks_per_sm);
  });
}

int lbmb_autotune_sweep(lbmb_solver* h, int32_t steps_per_trial, lbmb_autotune_result* out,
                        int32_t* trial_desc, double* trial_ms, int32_t capacity) {
  return guarded([&] {
    NEED(h);
    h->e->autotune_sweep(steps_per_trial, out, trial_desc, trial_ms, capacity);
  });
}

int lbmb_get_sweep_kernel(lbmb_solver* h, int32_t* kind) {
  return guarded([&] {
    NEED(h);
    if (!kind) lbmb::invalid("null output");
    *kind = h->e->sweep_kernel();
  });
}

int lbmb_batch_create(lbmb_solver* const* solvers, const int32_t* bodies, int32_t ncases,
                      const lbmb_ibm_config* cfg, lbmb_batch** out) {
  return guarded([&] {
    if (!solvers || !cfg || !out) lbmb::invalid("null argument");
    if (ncases <= 0) lbmb::invalid("batch needs at least one solver");
    std::vector<lbmb::EngineBase*> all;
    for (int32_t k = 0; k < ncases; ++k) {
      if (!solvers[k] || !solvers[k]->e) lbmb::invalid("null solver in batch");
      all.push_back(solvers[k]->e.get());
    }
    auto* h = new lbmb_batch();
    try {
      h->b.reset(all.front()->make_batch(all, bodies, *cfg));
    } catch (...) {
      delete h;
      throw;
    }
    *out = h;
  });
}

int lbmb_batch_autotune(lbmb_batch* b, int32_t steps_per_trial, int32_t* even_blocks_per_sm,
                        int32_t* odd_blocks_per_sm, double* best_ms_per_step) {
  return guarded([&] {
    if (!b || !b->b) lbmb::invalid("null batch");
    b->b->autotune(steps_per_trial, even_blocks_per_sm, odd_blocks_per_sm, best_ms_per_step);
  });
}

int lbmb_batch_run(lbmb_batch* b, int64_t steps, double* torque_lu, double* device_ms) {
  return guarded([&] {
    if (!b || !b->b) lbmb::invalid("null batch");
    b->b->run(steps, torque_lu, device_ms);
  });
}

int lbmb_batch_destroy(lbmb_batch* b) {
  return guarded([&] { delete b; });
}

int lbmb_adjoint_torque(lbmb_solver* h, const lbmb_ibm_config* cfg, const lbmb_adjoint_config* ac,
                        lbmb_adjoint_result* out, double* dJ_dpos, double* torque) {
  return guarded([&] {
    NEED(h);
    if (!cfg || !ac) lbmb::invalid("null argument");
    h->e->adjoint_torque(*cfg, *ac, out, dJ_dpos, torque);
  });
}

int lbmb_set_wait_limit(lbmb_solver* h, int64_t cycles) {
  return guarded([&] {
    NEED(h);
    h->e->set_wait_limit((long long)cycles);
  });
}

int lbmb_capabilities(lbmb_solver* h, lbmb_backend_caps* out) {
  return guarded([&] {
    if (!out) lbmb::invalid("null output");
    if (h && !h->e) lbmb::invalid("null solver");
    std::memset(out, 0, sizeof(*out));
    // backend.rs:162-199: periodic single-part axes wrap inside the sweep;
    // localized sources, open faces, the two-pass split and gravity are not
    // on this path; hydro and scalar distributions are stepped, phase-field
    // distributions are not
    out->handles_single_part_periodic_halo = 1;
    out->supports_localized_features = 0;
    out->supports_d3q27_open_faces = 0;
    out->supports_two_pass = 0;
    out->supports_gravity_body_force = 0;
    out->distribution_hydro = LBMB_SUPPORTED;
    out->distribution_phase = LBMB_UNSUPPORTED_NOT_IMPLEMENTED;
    out->distribution_scalar = LBMB_SUPPORTED;
    out->run_chunk_size = INT64_MAX;  // backend.rs:343-345: any span per call
    out->lattices = 1u | 2u | 4u;
    out->storages = (1u << LBMB_STORE_F32) | (1u << LBMB_STORE_F16) | (1u << LBMB_STORE_BF16) | (1u << LBMB_STORE_F64);
    out->collisions = (1u << LBMB_BGK) | (1u << LBMB_TRT) | (1u << LBMB_CENTRAL_MOMENT);
    out->checkpoint = 1;
    if (h) {
      h->e->allows(&out->adjoint, &out->batch);
    } else {
      out->adjoint = 1;
      out->batch = 1;
    }
  });
}

int lbmb_sync(lbmb_solver* h) {
  return guarded([&] {
    NEED(h);
    h->e->sync();
  });
}

// ---- checkpoint/restart ------------------------------------------------------

int lbmb_get_time(const lbmb_solver* h, uint64_t* step) {
  return guarded([&] {
    if (!h || !h->e || !step) throw Error(LBMB_ERR_INVALID, "null argument");
    *step = h->e->time;
  });
}

int lbmb_set_scalar_name(lbmb_solver* h, int32_t k, const char* name) {
  return guarded([&] {
    NEED(h);
    if (!name) throw Error(LBMB_ERR_INVALID, "null argument");
    h->e->set_scalar_name(k, std::string(name));
  });
}

int lbmb_set_qoi_checkpoint_state(lbmb_solver* h, const char* json, int64_t len) {
  return guarded([&] {
    NEED(h);
    if (!json) {
      h->e->has_qoi = false;
      h->e->qoi_json.clear();
      return;
    }
    if (len < 0) throw Error(LBMB_ERR_INVALID, "negative length");
    std::string t(json, size_t(len));
    if (!lbmb::ckpt::json_object(t)) throw Error(LBMB_ERR_INVALID, "QOI checkpoint state must be a JSON object");
    h->e->has_qoi = true;
    h->e->qoi_json = std::move(t);
  });
}

int lbmb_get_qoi_checkpoint_state(lbmb_solver* h, char* buf, int64_t cap, int64_t* len) {
  return guarded([&] {
    NEED(h);
    if (!len) throw Error(LBMB_ERR_INVALID, "null argument");
    if (!h->e->has_qoi) {
      *len = -1;
      return;
    }
    *len = int64_t(h->e->qoi_json.size());
    if (buf && cap > 0) std::memcpy(buf, h->e->qoi_json.data(), size_t(std::min<int64_t>(cap, *len)));
  });
}

int lbmb_checkpoint_save(lbmb_solver* h, const char* dir) {
  return guarded([&] {
    NEED(h);
    if (!dir) throw Error(LBMB_ERR_INVALID, "null argument");
    h->e->checkpoint_save(dir);
  });
}

int lbmb_checkpoint_restore(lbmb_solver* h, const char* dir) {
  return guarded([&] {
    NEED(h);
    if (!dir) throw Error(LBMB_ERR_INVALID, "null argument");
    h->e->checkpoint_restore(dir);
  });
}

}  // extern "C"
