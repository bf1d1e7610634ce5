"""Host-side runner QOIs, unit report, scalar pulse, capability query and
16-bit storage codecs (CPU only).

The library's C entry points are compared with the oracle's restatement of
the reference (bit for bit: the same f64 operations in the same order), and
both are pinned by the reference's own known answers where it has them:
crates/lbm-scenario/tests/bioprocess_units.rs (Re = 25 for the base
scenario, Mach / tau / grid-Re thresholds), crates/lbm-core/src/qoi.rs
tests (power QOIs).
"""
import math

import numpy as np
import pytest

import lbmflow_b200 as lb

TAU = 2.0 * math.pi


# --- power QOIs ---------------------------------------------------------------

def test_power_qois_library_equals_oracle_and_kat(oracle):
    # qoi.rs tests: power_formula_and_sign_convention_are_explicit
    a = lb.power_qois(2.0, TAU * 3.0, 1000.0, 0.5, 2.0)
    b = oracle.power_qois(2.0, TAU * 3.0, 1000.0, 0.5, 2.0)
    for k in ("torque_n_m", "power_w", "rotational_speed_hz", "np", "p_over_v_w_m3"):
        assert a[k] == b[k], k
    assert abs(a["power_w"] - TAU * 6.0) < 1e-12
    assert abs(a["p_over_v_w_m3"] - a["power_w"] / 2.0) < 1e-12
    assert lb.power_qois(-2.0, TAU, 1000.0, 0.5, 1.0)["power_w"] < 0.0
    # zero_torque_gives_zero_power_and_np
    z = lb.power_qois(0.0, TAU, 1000.0, 0.1, 0.01)
    assert z["power_w"] == 0.0 and z["np"] == 0.0
    for bad in ((3.0, TAU, 0.0, 0.1, 0.5), (3.0, TAU, 1000.0, -0.1, 0.5), (3.0, 0.0, 1000.0, 0.1, 0.5),
                (3.0, TAU, 1000.0, 0.1, float("nan"))):
        with pytest.raises(lb.SpecError):
            lb.power_qois(*bad)


@pytest.mark.parametrize("steps,probe,executed", [(200, 1, 200), (200, 7, 200), (1000, 3, 1000), (5, 10, 5),
                                                  (3000, 1, 1000)])
def test_runner_power_from_series_equals_oracle(oracle, steps, probe, executed):
    rng = np.random.default_rng(steps + probe)
    torque = rng.normal(2e-4, 3e-5, size=executed)
    args = (1000.0, 0.2 / 128, 1e-3, TAU * 150.0 / 60.0, 0.2 / 3, 0.2 ** 2 * math.pi / 4 * 0.25)
    a = lb.power_from_torque_series(torque, steps, probe, *args)
    b = oracle.runner_power(torque, steps, probe, *args)
    for k in ("torque_n_m", "power_w", "np", "p_over_v_w_m3", "records_used"):
        assert a[k] == b[k], k
    # the window: records with step >= steps / 2 (all records when none)
    rec = [s for s in range(1, executed + 1) if s % probe == 0 or s == steps]
    win = [s for s in rec if s >= steps // 2] or rec
    assert a["records_used"] == len(win)
    scale = 1000.0 * (0.2 / 128) ** 5 / 1e-3 ** 2
    expect = np.mean([torque[s - 1] * scale for s in win])
    assert abs(a["torque_n_m"] - expect) <= 1e-12 * abs(expect)


# --- unit report (crates/lbm-scenario/tests/bioprocess_units.rs) -------------

BASE = dict(vessel_diameter_m=0.2, liquid_height_m=0.2, impeller_diameter_m=0.05, rotational_speed_rpm=60.0,
            liquid_density_kg_m3=1000.0, liquid_viscosity_pa_s=0.1, dt_s=0.0008, grid=(100, 100, 100))


def _both(oracle, **kw):
    p = dict(BASE, **kw)
    a = lb.unit_report(**p, checked=False)
    b = oracle.unit_report(p["vessel_diameter_m"], p["liquid_height_m"], p["impeller_diameter_m"],
                           p["rotational_speed_rpm"], p["liquid_density_kg_m3"], p["liquid_viscosity_pa_s"],
                           p["dt_s"], p["grid"], p.get("scalar_diffusivity_m2_s") or 0.0)
    for k in oracle.UNIT_KEYS:
        av, bv = a[k], b[k]
        assert (av == bv) or (math.isnan(av) and math.isnan(bv)), k
    names = {v: k for k, v in lb.UNIT_ISSUES.items()}
    assert sum(names[w] for w in a["warnings"]) == b["warnings"]
    assert sum(names[r] for r in a["rejections"]) == b["rejections"]
    return a


def test_unit_report_reynolds_kat(oracle):
    r = _both(oracle)
    assert abs(r["reynolds"] - 25.0) <= 1e-12 * 25.0  # dimensionless_groups_reynolds_matches_analytical_impeller
    assert r["dx_m"] == 0.2 / 100 and r["cs2_lu"] == 1.0 / 3.0
    assert r["tau_lu"] == 3.0 * r["nu_lu"] + 0.5
    assert math.isnan(r["schmidt"]) and math.isnan(r["peclet"])


def test_unit_report_mach_warn_and_reject(oracle):
    # mach_lattice_warn_at_0_11_reject_at_0_31
    w = _both(oracle, dt_s=0.0025403411844343537)
    assert w["mach_lattice"] > 0.10 and "MA_LATTICE_HIGH" in w["warnings"]
    r = _both(oracle, dt_s=0.007159143792496811)
    assert r["mach_lattice"] > 0.30 and "MA_LATTICE_TOO_HIGH" in r["rejections"]
    with pytest.raises(lb.UnsupportedError):
        lb.unit_report(**dict(BASE, dt_s=0.007159143792496811))


def test_unit_report_tau_and_grid_reynolds(oracle):
    # tau_near_half_warn_and_below_half_rejects
    t = _both(oracle, dt_s=0.0002)
    assert t["tau_lu"] <= 0.55 and "TAU_NEAR_HALF" in t["warnings"]
    with pytest.raises(lb.SpecError):
        lb.unit_report(**dict(BASE, liquid_viscosity_pa_s=0.0))
    # grid_reynolds_warning_fires_at_configured_threshold
    g = _both(oracle, liquid_viscosity_pa_s=0.001)
    assert g["u_ref_lu"] / g["nu_lu"] > 15.0 and "GRID_REYNOLDS_HIGH" in g["warnings"]


def test_unit_report_scalar_groups(oracle):
    r = _both(oracle, scalar_diffusivity_m2_s=1e-9)
    nu = 0.1 / 1000.0
    assert r["schmidt"] == nu / 1e-9
    assert r["scalar_diffusivity_lu"] == 1e-9 * 0.0008 / (0.002 * 0.002)
    assert "SCALAR_DIFFUSION_UNSTABLE" in r["warnings"]
    assert lb.scalar_diffusivity_lu(1e-9, 0.0008, 0.002) == r["scalar_diffusivity_lu"]


# --- scalar pulse, capabilities -------------------------------------------------

def test_top_hat_pulse_equals_oracle(oracle):
    g = oracle.build_tank((32, 32, 40), 1.0 / 32, 1.0, 1.25, 1.0 / 3, 1.0 / 3, 6, 1.0)
    center = [0.5, 0.5, 1.1]
    a = lb.scalar_top_hat_pulse((32, 32, 40), g["solid"], 1.0 / 32, center, 0.15, 2.5)
    b = oracle.top_hat_pulse((32, 32, 40), g["solid"], 1.0 / 32, center, 0.15, 2.5)
    assert np.array_equal(a, b)
    assert a.max() == 2.5 and (a[g["solid"] != 0] == 0).all()
    assert int((a > 0).sum()) > 100


def test_capabilities_without_handle():
    c = lb.capabilities()
    assert c["handles_single_part_periodic_halo"] == 1
    assert c["supports_two_pass"] == 0 and c["supports_d3q27_open_faces"] == 0
    assert c["supports_localized_features"] == 0 and c["supports_gravity_body_force"] == 0
    assert c["distribution_hydro"] == 0 and c["distribution_scalar"] == 0 and c["distribution_phase"] == 1
    assert c["run_chunk_size"] == 2 ** 63 - 1
    assert c["lattices"] == 7 and c["storages"] == 15 and c["collisions"] == 7


# --- flat-blade turbine: library generator == oracle restatement ---------------

@pytest.mark.parametrize("n,spacing,baffles", [(48, 0.7, True), (64, 0.5, False), (128, 0.7, True)])
def test_flat_blade_tank_bit_exact(oracle, n, spacing, baffles):
    dims = (n, n, int(round(1.25 * n)))
    dx = 1.0 / n
    kw = dict(baffle_w=0.1 if baffles else 0.0, baffle_t=(2.6 / n) if baffles else 0.0)
    spec = lb.TankSpec(dims=dims, dx_m=dx, vessel_diameter_m=1.0, liquid_height_m=1.25, impeller_diameter_m=1.0 / 3,
                       clearance_m=1.0 / 3, omega_rad_s=1.0, impeller="flat_blade",
                       baffle_count=4 if baffles else 0, baffle_width_m=kw["baffle_w"],
                       baffle_thickness_m=kw["baffle_t"], marker_spacing_cells=spacing, min_cells=12.0)
    a = lb.build_stirred_tank(spec)
    b = oracle.build_tank(dims, dx, 1.0, 1.25, 1.0 / 3, 1.0 / 3, 6, 1.0, kind=2, spacing=spacing, **kw)
    for k in ("solid", "baffle", "wall_velocity", "marker_pos", "marker_w", "center", "omega"):
        assert np.array_equal(np.asarray(a[k]), np.asarray(b[k])), k


# --- 16-bit storage codecs -------------------------------------------------------

def test_reference_f16_codec_known_values(oracle):
    # f32_to_f16_bits (crates/lbm-core/src/gpu/backend.rs:160-186): nearest
    # with ties away from zero, flush below 2^-25, saturate to infinity
    vals = np.array([1.0, -2.0, 65504.0, 65520.0, 2.0 ** -24, 2.0 ** -25, 2.0 ** -26, 1.0 + 2.0 ** -11,
                     1.0 + 3 * 2.0 ** -11, float("nan"), float("inf")], dtype=np.float32)
    bits = oracle.f16_bits(vals)
    assert list(bits) == [0x3C00, 0xC000, 0x7BFF, 0x7C00, 0x0001, 0x0001, 0x0000, 0x3C01, 0x3C02, 0x7C00, 0x7C00]


def test_f16_codecs_agree_off_ties(oracle):
    rng = np.random.default_rng(5)
    v = (rng.normal(0, 1e-2, 200000) * rng.choice([1, 1e-3, 30.0], 200000)).astype(np.float32)
    ref = oracle.codec16("ref_f16", v)
    rne = oracle.codec16("f16", v)
    np16 = v.astype(np.float16).astype(np.float32)
    assert np.array_equal(rne, np16)  # nearest-even equals numpy's binary16
    # the reference codec differs from nearest-even only at exact ties
    diff = ref != rne
    bits = v.view(np.uint32)
    tie = (bits & 0x1FFF) == 0x1000
    normal = np.abs(v) >= 2.0 ** -14
    assert not (diff & normal & ~tie).any()


def test_bf16_rounding_is_nearest_even(oracle):
    import torch
    rng = np.random.default_rng(6)
    v = rng.normal(0, 1e-2, 100000).astype(np.float32)
    v[:4] = np.array([1.0 + 2.0 ** -8, 1.0 + 3 * 2.0 ** -8, -(1.0 + 2.0 ** -8), 3.0], dtype=np.float32)
    t = torch.from_numpy(v).to(torch.bfloat16).to(torch.float32).numpy()
    assert np.array_equal(oracle.codec16("bf16", v), t)
