"""Oxygen transfer and uptake sources of the oracle, pinned to the reference's
own unit tests (crates/lbm-core/src/oxygen.rs and reaction.rs test modules)."""
import numpy as np
import pytest

from oracle import oracle as o


def test_uniform_oxygen_remains_uniform_without_sources():
    c, ledger, diag = o.interfacial_flux(np.full(8, 0.25), 1.0, np.zeros(8), 1.0e-9, 1.0, 1.0e-4)
    assert np.array_equal(c, np.full(8, 0.25))
    assert diag["clipped_cells"] == 0 and ledger["last_step_mol"] == 0.0


def test_henry_boundary_concentration_uses_scenario_inputs():
    assert abs(o.henry_equilibrium(1.3e-5, 21000.0) - 0.273) < 1e-12
    assert np.isnan(o.henry_equilibrium(0.0, 21000.0))


def test_negative_concentration_clip_reports_diagnostic():
    # clipping through the uptake with a zero rate leaves only the clip
    c, _, diag = o.oxygen_uptake(np.array([1.0, 0.0, 0.0, 0.0]), 1.0, 1.0, our=0.0)
    assert diag["clipped_cells"] == 0
    c, _, diag = o.interfacial_flux(np.array([1.0, -0.2, 0.0, -1.0]), 0.0, np.zeros(4), 1.0, 1.0, 1.0)
    assert np.array_equal(c, [1.0, 0.0, 0.0, 0.0])
    assert diag["clipped_cells"] == 2 and diag["clipped_fraction"] == 0.5 and diag["min_before_clip"] == -1.0


def test_interfacial_flux_is_zero_when_area_or_driving_force_is_zero():
    c, ledger, _ = o.interfacial_flux(np.array([0.1, 0.5]), np.array([1.0, 0.5]), np.array([0.0, 20.0]), 1.0, 1.0,
                                      2.0e-5)
    assert np.array_equal(c, [0.1, 0.5]) and ledger["source_integral_mol_s"] == 0.0
    assert ledger["active_interface_cells"] == 1


def test_closed_system_ledger_matches_integral_source():
    _, ledger, _ = o.interfacial_flux(np.zeros(2), 1.0, np.array([10.0, 20.0]), np.array([2.0, 3.0]), 0.5, 0.01)
    assert abs(ledger["last_step_mol"] - (0.01 * 10.0 * 2.0 + 0.01 * 20.0 * 3.0) * 0.5) < 1e-12
    _, l2, _ = o.interfacial_flux(np.zeros(2), 1.0, np.array([10.0, 20.0]), np.array([2.0, 3.0]), 0.5, 0.01,
                                  cumulative=ledger["cumulative_mol"])
    assert abs(l2["cumulative_mol"] - 2 * ledger["last_step_mol"]) < 1e-12


def test_interfacial_area_density():
    # 6 |grad phi| phi (1 - phi) 4 / width
    a = o.interfacial_area_density(0.5, [0.0, 2.0, 0.0], 0.1)
    assert abs(a - 6.0 * 2.0 * 0.25 * 40.0) < 1e-12
    assert np.isnan(o.interfacial_area_density(1.5, [0.0, 0.0, 0.0], 0.1))


def test_constant_our_gives_linear_depletion_closed_uniform_field():
    c, ledger, _ = o.oxygen_uptake(np.ones(4), 1.0, 2.0, our=0.1)
    assert np.all(np.abs(c - 0.8) < 1e-12) and abs(ledger["last_step_kmol_consumed"] - 0.8) < 1e-12


def test_zero_our_has_no_effect():
    c, ledger, _ = o.oxygen_uptake(np.array([0.3, 0.4]), 1.0, 1.0, our=0.0)
    assert np.array_equal(c, [0.3, 0.4]) and ledger["last_step_kmol_consumed"] == 0.0


def test_negative_concentration_guard_fires():
    c, _, diag = o.oxygen_uptake(np.array([0.1]), 1.0, 2.0, our=0.2)
    assert np.array_equal(c, [0.0]) and diag["clipped_cells"] == 1


def test_source_ledger_matches_consumption_integral():
    _, ledger, _ = o.oxygen_uptake(np.ones(2), np.array([2.0, 3.0]), 0.5, our=0.2)
    assert abs(ledger["last_step_kmol_consumed"] - 0.5) < 1e-12


def test_monod_and_cell_density_rates_and_errors():
    c, _, _ = o.oxygen_uptake(np.array([0.2]), 1.0, 1.0, kind="monod", our_max=0.1, ks=0.5, c_ref=0.4)
    cs = 0.2 / 0.4
    assert abs(c[0] - (0.2 - 0.1 * cs / (0.5 + cs))) < 1e-15
    c, _, _ = o.oxygen_uptake(np.array([0.2, 0.3]), 1.0, 0.5, kind="cell_density_scaled", specific_our=0.01,
                              density=np.array([2.0, 4.0]))
    assert np.allclose(c, [0.2 - 0.01, 0.3 - 0.02], atol=1e-15)
    with pytest.raises(ValueError):
        o.oxygen_uptake(np.array([-0.1]), 1.0, 1.0, our=0.1)  # C_L must be >= 0 before OUR
    with pytest.raises(ValueError):
        o.oxygen_uptake(np.array([0.1]), 1.0, 1.0, kind="cell_density_scaled", specific_our=0.1)
    with pytest.raises(ValueError):
        o.interfacial_flux(np.array([0.1]), 1.0, np.array([-1.0]), 1.0, 1.0, 1e-4)
    with pytest.raises(ValueError):
        o.interfacial_flux(np.array([0.1]), 1.0, np.array([1.0]), 0.0, 1.0, 1e-4)
