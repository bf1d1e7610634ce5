// Host-side set-up geometry for the stirred-tank path (C++).
//
// Voxel flags and reference impeller markers follow
// crates/lbm-core/src/geometry.rs and must be bit-identical to it; the
// flat-blade turbine generator (kind LBMB_IMPELLER_FLAT_BLADE) has no
// reference counterpart: it samples the analytic disc + blade surfaces at a
// uniform marker spacing.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <stdexcept>
#include <string>
#include <vector>

#include "../../include/lbmb.h"

namespace lbmb {
extern thread_local std::string g_last_error;
}

namespace {

constexpr double kTau = 6.283185307179586476925286766559;
constexpr double kPi = 3.14159265358979323846264338327950288;
// geometry.rs:10-16
constexpr double RUSHTON_BLADE_THICKNESS_FRACTION = 0.04;
constexpr double RUSHTON_DISC_DIAMETER_FRACTION = 0.65;
constexpr double PITCHED_BLADE_ANGLE_DEG = 45.0;
constexpr double PITCHED_BLADE_THICKNESS_FRACTION = 0.035;

struct GeoError : std::runtime_error {
  int code;
  GeoError(int c, const std::string& m) : std::runtime_error(m), code(c) {}
};

inline size_t cidx(const int32_t d[3], int x, int y, int z) { return (size_t(z) * d[1] + y) * d[0] + x; }

struct Markers {
  std::vector<double> pos, w;
  std::vector<double> si;  // SI positions (m) used for the wall-velocity stamp
};

// build_radial_impeller (geometry.rs:815-906): SI inputs, lattice-unit marker
// positions, weight dx^2.
void radial_impeller(const lbmb_tank_spec& s, bool pitched, double omega_z, Markers& out) {
  const double dx = s.dx_m;
  const double blade_angle_deg = pitched ? PITCHED_BLADE_ANGLE_DEG : 0.0;
  const double thickness_fraction = pitched ? PITCHED_BLADE_THICKNESS_FRACTION : RUSHTON_BLADE_THICKNESS_FRACTION;
  const double cx = 0.5 * s.dims[0] * dx, cy = 0.5 * s.dims[1] * dx;
  const double radius = 0.5 * s.impeller_diameter_m;
  const double center[3] = {cx, cy, s.clearance_m};
  const double radial_inner = pitched ? 0.35 * radius : RUSHTON_DISC_DIAMETER_FRACTION * radius;
  const double dr = std::max(dx, radius / 20.0);
  const double dz = dx, tangential_step = dx;
  const double thickness = std::max(thickness_fraction * s.impeller_diameter_m, dx);
  for (int b = 0; b < s.blade_count; ++b) {
    const double th = kTau * double(b) / double(s.blade_count);
    const double er[2] = {std::cos(th), std::sin(th)};
    const double et[2] = {-std::sin(th), std::cos(th)};
    const double pitch = blade_angle_deg * (kPi / 180.0);
    const double z_span =
        blade_angle_deg == 0.0 ? thickness : thickness + (radius - radial_inner) * std::sin(pitch) * 0.18;
    const size_t nr = size_t(std::max(std::ceil((radius - radial_inner) / dr), 1.0));
    const size_t nt = size_t(std::max(std::ceil(thickness / tangential_step), 1.0));
    const size_t nz = size_t(std::max(std::ceil(z_span / dz), 1.0));
    for (size_t ir = 0; ir <= nr; ++ir) {
      const double rr = radial_inner + (radius - radial_inner) * double(ir) / double(nr);
      for (size_t it = 0; it <= nt; ++it) {
        const double off_t = -0.5 * thickness + thickness * double(it) / double(nt);
        for (size_t iz = 0; iz <= nz; ++iz) {
          const double off_z = -0.5 * z_span + z_span * double(iz) / double(nz);
          const double pz = off_z + (rr - radial_inner) * std::sin(pitch) * 0.18;
          const double p[3] = {center[0] + rr * er[0] + off_t * et[0], center[1] + rr * er[1] + off_t * et[1],
                               center[2] + pz};
          const double rel = std::sqrt(std::pow(p[0] - cx, 2) + std::pow(p[1] - cy, 2));
          if (rel >= 0.5 * s.vessel_diameter_m || p[2] <= 0.0 || p[2] >= s.liquid_height_m) continue;
          out.pos.push_back(p[0] / dx);
          out.pos.push_back(p[1] / dx);
          out.pos.push_back(p[2] / dx);
          out.w.push_back(dx * dx);
          for (int a = 0; a < 3; ++a) out.si.push_back(p[a]);
        }
      }
    }
  }
  (void)omega_z;
}

// Flat-blade (disc) turbine sampled on its analytic surfaces at a uniform
// spacing h (cells): a disc of diameter 0.75 D and `blade_count` flat
// blades of radial length D/4 and height D/5 at the rim, each a plate of
// thickness t = max(0.04 D, 1 cell) represented by markers on both faces.
// Weights are the face area per marker (lattice units).
void flat_blade_turbine(const lbmb_tank_spec& s, Markers& out) {
  const double dx = s.dx_m;
  const double h = s.marker_spacing_cells;
  const double D = s.impeller_diameter_m / dx, R = 0.5 * D;
  const double cx = 0.5 * s.dims[0], cy = 0.5 * s.dims[1], cz = s.clearance_m / dx;
  const double t = std::max(0.04 * D, 1.0);
  const double L = 0.25 * D, H = 0.2 * D, rin = R - L;
  const double rd = 0.375 * D;
  auto push = [&](double x, double y, double z, double w) {
    out.pos.push_back(x);
    out.pos.push_back(y);
    out.pos.push_back(z);
    out.w.push_back(w);
    out.si.push_back(x * dx);
    out.si.push_back(y * dx);
    out.si.push_back(z * dx);
  };
  // disc faces at z = cz -/+ t/2: concentric rings
  const int K = int(std::ceil(rd / h));
  std::vector<double> ring_r;
  std::vector<int> ring_n;
  int disc_count = 0;
  for (int k = 0; k <= K; ++k) {
    const double r = rd * double(k) / double(K);
    const int m = k == 0 ? 1 : std::max(1, int(std::lround(kTau * r / h)));
    ring_r.push_back(r);
    ring_n.push_back(m);
    disc_count += m;
  }
  const double disc_w = kPi * rd * rd / double(disc_count);
  for (int side = 0; side < 2; ++side) {
    const double z = cz + (side ? 0.5 : -0.5) * t;
    for (size_t k = 0; k < ring_r.size(); ++k)
      for (int j = 0; j < ring_n[k]; ++j) {
        const double th = kTau * (double(j) + 0.5 * double(k & 1)) / double(ring_n[k]);
        push(cx + ring_r[k] * std::cos(th), cy + ring_r[k] * std::sin(th), z, disc_w);
      }
  }
  // blade faces at tangential offset -/+ t/2
  const int nr = std::max(1, int(std::ceil(L / h)));
  const int nzb = std::max(1, int(std::ceil(H / h)));
  const double blade_w = L * H / double((nr + 1) * (nzb + 1));
  for (int b = 0; b < s.blade_count; ++b) {
    const double th = kTau * double(b) / double(s.blade_count);
    const double er[2] = {std::cos(th), std::sin(th)}, et[2] = {-std::sin(th), std::cos(th)};
    for (int side = 0; side < 2; ++side) {
      const double off = (side ? 0.5 : -0.5) * t;
      for (int i = 0; i <= nr; ++i) {
        const double r = rin + L * double(i) / double(nr);
        for (int k = 0; k <= nzb; ++k) {
          const double z = cz - 0.5 * H + H * double(k) / double(nzb);
          push(cx + r * er[0] + off * et[0], cy + r * er[1] + off * et[1], z, blade_w);
        }
      }
    }
  }
}

void validate_tank(const lbmb_tank_spec& s) {
  auto bad = [](const std::string& m) { throw GeoError(LBMB_ERR_INVALID, m); };
  for (int a = 0; a < 3; ++a)
    if (s.dims[a] < 3) bad("stirred-tank grid dimensions must preserve a 1-cell solid rim");
  if (!(std::isfinite(s.dx_m) && s.dx_m > 0.0)) bad("grid spacing must be finite and positive");
  if (!(std::isfinite(s.vessel_diameter_m) && s.vessel_diameter_m > 0.0)) bad("vessel diameter must be finite and positive");
  if (!(std::isfinite(s.liquid_height_m) && s.liquid_height_m > 0.0)) bad("liquid height must be finite and positive");
  const double min_cells = s.min_cells > 0.0 ? s.min_cells : 32.0;
  const double cells = std::min(s.vessel_diameter_m, s.impeller_diameter_m) / s.dx_m;
  if (cells < min_cells) bad("stirred-tank geometry is under-resolved");
  if (!(s.impeller_diameter_m > 0.0) || !(s.omega_rad_s > 0.0) || s.blade_count <= 0)
    bad("impeller diameter, speed and blade count must be positive");
  if (!(s.clearance_m > 0.0 && s.clearance_m + 0.5 * s.impeller_diameter_m < s.liquid_height_m))
    bad("impeller must be above the tank bottom and below the liquid surface");
  if (s.impeller_diameter_m >= s.vessel_diameter_m) bad("impeller diameter must fit inside the vessel");
  if (s.baffle_count != 0 && s.baffle_count != 4)
    throw GeoError(LBMB_ERR_UNSUPPORTED, "custom baffle placement is not implemented; use count = 4");
  if (s.baffle_count == 4) {
    if (!(s.baffle_width_m > 0.0) || !(s.baffle_thickness_m > 0.0)) bad("baffle width and thickness must be positive");
    if (s.baffle_width_m + s.baffle_thickness_m >= 0.5 * s.vessel_diameter_m) bad("baffles must fit inside the tank radius");
  }
  if (s.impeller_kind < 0 || s.impeller_kind > 2) throw GeoError(LBMB_ERR_UNSUPPORTED, "unknown impeller kind");
  if (s.impeller_kind == LBMB_IMPELLER_FLAT_BLADE && !(s.marker_spacing_cells > 0.0))
    bad("flat-blade marker spacing must be positive");
}

template <class F>
int guard(F&& fn) {
  try {
    fn();
    lbmb::g_last_error.clear();
    return LBMB_OK;
  } catch (const GeoError& e) {
    lbmb::g_last_error = e.what();
    return e.code;
  } catch (const std::exception& e) {
    lbmb::g_last_error = e.what();
    return LBMB_ERR_INVALID;
  }
}

}  // namespace

extern "C" {

int lbmb_build_wall_rims(const int32_t dims[3], const int32_t is_wall[6], const double u[18], uint8_t* solid,
                         double* wall_u) {
  return guard([&] {
    if (!dims || !is_wall || !u || !solid || !wall_u) throw GeoError(LBMB_ERR_INVALID, "null argument");
    const size_t n = size_t(dims[0]) * dims[1] * dims[2];
    std::vector<double> best(n, -1.0);
    std::memset(solid, 0, n);
    std::fill(wall_u, wall_u + 3 * n, 0.0);
    const int order[6] = {2, 3, 0, 1, 4, 5};  // YNeg, YPos, XNeg, XPos, ZNeg, ZPos (solver.rs:1366-1373)
    for (int face : order) {
      const int a = face / 2;
      if (!is_wall[face]) continue;
      const double* uf = u + 3 * face;
      const double speed = uf[0] * uf[0] + uf[1] * uf[1] + uf[2] * uf[2];
      const int fixed = (face % 2 == 0) ? 0 : dims[a] - 1;
      const int t1 = a == 0 ? 1 : 0, t2 = a == 2 ? 1 : 2;
      for (int c2 = 0; c2 < dims[t2]; ++c2)
        for (int c1 = 0; c1 < dims[t1]; ++c1) {
          int p[3];
          p[a] = fixed;
          p[t1] = c1;
          p[t2] = c2;
          const size_t i = cidx(dims, p[0], p[1], p[2]);
          solid[i] = 1;
          if (speed > best[i]) {
            best[i] = speed;
            for (int k = 0; k < 3; ++k) wall_u[3 * i + k] = uf[k];
          }
        }
    }
  });
}

int lbmb_build_stirred_tank(const lbmb_tank_spec* spec, uint8_t* solid, uint8_t* baffle_mask, double* wall_velocity,
                            double* marker_pos, double* marker_weight, int64_t capacity, int64_t* n_markers,
                            double center[3], double omega[3]) {
  return guard([&] {
    if (!spec) throw GeoError(LBMB_ERR_INVALID, "null tank spec");
    const lbmb_tank_spec& s = *spec;
    validate_tank(s);
    const double dx = s.dx_m;
    const size_t n = size_t(s.dims[0]) * s.dims[1] * s.dims[2];
    std::vector<uint8_t> so(n, 0), bm(n, 0);
    const double cx = 0.5 * s.dims[0] * dx, cy = 0.5 * s.dims[1] * dx;
    const double radius = 0.5 * s.vessel_diameter_m;
    // apply_cylindrical_tank_mask (geometry.rs:657-679)
    for (int z = 0; z < s.dims[2]; ++z) {
      const double zm = (double(z) + 0.5) * dx;
      for (int y = 0; y < s.dims[1]; ++y)
        for (int x = 0; x < s.dims[0]; ++x) {
          const double px = (double(x) + 0.5) * dx, py = (double(y) + 0.5) * dx;
          const double r = std::sqrt((px - cx) * (px - cx) + (py - cy) * (py - cy));
          const bool rim = x == 0 || y == 0 || z == 0 || x + 1 == s.dims[0] || y + 1 == s.dims[1] || z + 1 == s.dims[2];
          if (rim || r >= radius || zm >= s.liquid_height_m) so[cidx(s.dims, x, y, z)] = 1;
        }
    }
    // apply_baffle_mask (geometry.rs:681-723)
    if (s.baffle_count == 4) {
      const double inner = radius - s.baffle_width_m;
      for (int z = 1; z < s.dims[2] - 1; ++z) {
        const double zm = (double(z) + 0.5) * dx;
        if (zm >= s.liquid_height_m) continue;
        for (int y = 1; y < s.dims[1] - 1; ++y)
          for (int x = 1; x < s.dims[0] - 1; ++x) {
            const double rx = (double(x) + 0.5) * dx - cx, ry = (double(y) + 0.5) * dx - cy;
            const double r = std::sqrt(rx * rx + ry * ry);
            if (r >= radius || r < inner) continue;
            if (std::fabs(ry) <= 0.5 * s.baffle_thickness_m || std::fabs(rx) <= 0.5 * s.baffle_thickness_m) {
              so[cidx(s.dims, x, y, z)] = 1;
              bm[cidx(s.dims, x, y, z)] = 1;
            }
          }
      }
    }
    Markers mk;
    if (s.impeller_kind == LBMB_IMPELLER_FLAT_BLADE)
      flat_blade_turbine(s, mk);
    else
      radial_impeller(s, s.impeller_kind == LBMB_IMPELLER_PITCHED, s.omega_rad_s, mk);
    if (mk.w.empty()) throw GeoError(LBMB_ERR_INVALID, "impeller marker generation produced no markers");
    const int64_t m = int64_t(mk.w.size());
    const double cen[3] = {cx / dx, cy / dx, s.clearance_m / dx};
    // stamp_impeller_wall_velocity (geometry.rs:908-920): target velocity in
    // SI at the nearest cell of each marker.
    std::vector<double> wv(3 * n, 0.0);
    for (int64_t k = 0; k < m; ++k) {
      size_t ii[3];
      for (int a = 0; a < 3; ++a) {
        double r = std::round(mk.pos[3 * k + a]);
        r = std::min(std::max(r, 0.0), double(s.dims[a] - 1));
        ii[a] = size_t(r);
      }
      const double* p = &mk.si[3 * k];
      const double rv[3] = {p[0] - cx, p[1] - cy, p[2] - s.clearance_m};
      const double uu[3] = {0.0 * rv[2] - s.omega_rad_s * rv[1], s.omega_rad_s * rv[0] - 0.0 * rv[2],
                            0.0 * rv[1] - 0.0 * rv[0]};
      const size_t i = cidx(s.dims, int(ii[0]), int(ii[1]), int(ii[2]));
      for (int a = 0; a < 3; ++a) wv[3 * i + a] = uu[a];
    }
    if (solid) std::memcpy(solid, so.data(), n);
    if (baffle_mask) std::memcpy(baffle_mask, bm.data(), n);
    if (wall_velocity) std::memcpy(wall_velocity, wv.data(), 3 * n * sizeof(double));
    if (n_markers) *n_markers = m;
    if (marker_pos || marker_weight) {
      if (capacity < m) throw GeoError(LBMB_ERR_INVALID, "marker capacity too small");
      if (marker_pos) std::memcpy(marker_pos, mk.pos.data(), size_t(3 * m) * sizeof(double));
      if (marker_weight) std::memcpy(marker_weight, mk.w.data(), size_t(m) * sizeof(double));
    }
    if (center)
      for (int a = 0; a < 3; ++a) center[a] = cen[a];
    if (omega) {
      omega[0] = 0.0;
      omega[1] = 0.0;
      omega[2] = s.omega_rad_s;
    }
  });
}

}  // extern "C"
