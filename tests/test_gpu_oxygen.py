"""Oxygen transfer and uptake sources on a device scalar against the oracle.

The device entry points run the reference's composition gather_scalar_
concentration -> apply_interfacial_flux_sources / apply_oxygen_reaction_source
-> set_scalar_concentration. The oracle runs the same composition with its
restatement of oxygen.rs / reaction.rs on the same solver state, so the
concentration after a few ADE steps and the ledgers agree to 1e-12 (f64) /
1e-6 relative (f32); clip counts exactly.
"""
import numpy as np
import pytest

import lbmflow_b200 as lb
from cases import cavity

pytestmark = pytest.mark.gpu


def pair(prec):
    from oracle import oracle as o
    dims, solid, wall_u, nu = cavity(10, u_lid=0.05, re=40.0)
    n = 1000
    g = lb.Solver(dims, storage=prec, nu=nu, solid=solid, wall_u=wall_u)
    c = o.OracleSolver(dims, q=19, real_bits=64 if prec == "f64" else 32, nu=nu, solid=solid, wall_u=wall_u)
    kg = g.enable_scalar_distribution(2e-2, q=7)
    kc = c.scalar_enable(2e-2, q=7)
    rng = np.random.default_rng(3)
    c0 = np.where(solid == 0, rng.uniform(0.0, 0.3, n), 0.0)
    g.set_scalar_concentration(kg, c0)
    c.scalar_set(kc, c0)
    g.run(5)
    c.step(5)
    # liquid-surface band: interface cells in the top fluid layer
    z = np.arange(n) // 100
    area = np.where((solid == 0) & (z == 8), 50.0, 0.0)
    return g, c, kg, kc, solid, area


def check(g, c, kg, kc, prec):
    cg = g.gather_scalar_concentration(kg)
    cc = c.scalar_get(kc)
    tol = 1e-12 if prec == "f64" else 1e-6
    assert np.abs(cg - cc).max() <= tol * max(np.abs(cc).max(), 1e-30)


@pytest.mark.parametrize("prec", ["f64", "f32"])
def test_interfacial_flux_matches_oracle_composition(prec):
    from oracle import oracle as o
    g, c, kg, kc, solid, area = pair(prec)
    vol = 1e-6
    cum_g = cum_c = 0.0
    for _ in range(2):  # two calls in a row, ledger accumulates
        led_g, dg = g.apply_interfacial_flux_sources(kg, area, 0.27, vol, 0.5, 2e-2, cumulative_mol=cum_g)
        new, led_c, dc = o.interfacial_flux(c.scalar_get(kc), 0.27, area, vol, 0.5, 2e-2, cumulative=cum_c)
        c.scalar_set(kc, new)
        cum_g, cum_c = led_g["cumulative_mol"], led_c["cumulative_mol"]
        assert led_g["active_interface_cells"] == led_c["active_interface_cells"] == int((area > 0).sum())
        rel = 1e-12 if prec == "f64" else 1e-6
        assert abs(led_g["source_integral_mol_s"] - led_c["source_integral_mol_s"]) <= rel * abs(
            led_c["source_integral_mol_s"])
        assert abs(cum_g - cum_c) <= rel * abs(cum_c)
        assert dg["clipped_cells"] == dc["clipped_cells"]
        check(g, c, kg, kc, prec)
        g.run(3)
        c.step(3)
    check(g, c, kg, kc, prec)


@pytest.mark.parametrize("prec", ["f64", "f32"])
@pytest.mark.parametrize("kind,kw", [("constant", {"our": 0.02}),
                                     ("monod", {"our_max": 0.05, "ks": 0.5, "c_ref": 0.2}),
                                     ("cell_density_scaled", {"specific_our": 0.01})])
def test_oxygen_uptake_matches_oracle_composition(prec, kind, kw):
    from oracle import oracle as o
    g, c, kg, kc, solid, _ = pair(prec)
    dens = np.linspace(0.0, 3.0, g.n) if kind == "cell_density_scaled" else None
    led_g, dg = g.apply_oxygen_reaction_source(kg, 1e-6, 2.0, kind=kind, cell_density=dens, **kw)
    new, led_c, dc = o.oxygen_uptake(c.scalar_get(kc), 1e-6, 2.0, kind=kind, density=dens, **kw)
    c.scalar_set(kc, new)
    rel = 1e-12 if prec == "f64" else 1e-6
    assert abs(led_g["last_step_kmol_consumed"] - led_c["last_step_kmol_consumed"]) <= rel * abs(
        led_c["last_step_kmol_consumed"])
    assert dg["clipped_cells"] == dc["clipped_cells"]
    if kind == "constant":
        assert dg["clipped_cells"] > 0  # 0.04 removed from values in [0, 0.3): the clip fires
    check(g, c, kg, kc, prec)
    g.run(3)
    c.step(3)
    check(g, c, kg, kc, prec)


def test_sources_reject_invalid_inputs_and_keep_the_scalar():
    g, c, kg, kc, solid, area = pair("f64")
    before = g.gather_scalar_concentration(kg)
    bad = area.copy()
    bad[5] = -1.0
    with pytest.raises(lb.SpecError):
        g.apply_interfacial_flux_sources(kg, bad, 0.27, 1e-6, 0.5, 2e-2)
    with pytest.raises(lb.SpecError):
        g.apply_interfacial_flux_sources(kg, area, 0.27, 0.0, 0.5, 2e-2)
    with pytest.raises(lb.SpecError):
        g.apply_oxygen_reaction_source(kg, 1e-6, 1.0, kind="cell_density_scaled", specific_our=0.1)
    with pytest.raises(lb.SpecError):
        g.apply_oxygen_reaction_source(kg, 1e-6, -1.0, our=0.1)
    assert np.array_equal(g.gather_scalar_concentration(kg), before)
