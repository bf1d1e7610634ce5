"""Shear-rate and stress QOIs on the device against the oracle.

* Native strain rate (Solver::gather_strain_rate / gather_shear_rate): the
  device and the oracle run the same case (lid cavity, uniformly forced
  channel, IBM tank runner with its force field) and are compared cell by
  cell: 1e-9 of the largest |S| in f64, 2e-3 in f32 (the strain rate is a
  difference f - feq of nearly equal numbers, so f32 keeps fewer digits).
* Velocity-gradient stress, percentile summary and wall-shear proxy (the
  bioprocess runner's stress QOI): the oracle restatement of stress.rs gets
  the device's own cached velocity (read_moments) and wall velocity, so both
  sides see the same inputs; the f64 finite differences agree to 1e-12.
"""
import numpy as np
import pytest

import lbmflow_b200 as lb
from cases import cavity
from lbmflow_b200 import sweep

pytestmark = pytest.mark.gpu

DX, DT, MU, RHO = 1.0 / 32.0, 2.0e-3, 1.0e-3, 1000.0


def oracle_solver(dims, prec, **kw):
    from oracle import oracle as o
    return o.OracleSolver(dims, q=kw.pop("q", 19), real_bits=64 if prec == "f64" else 32, **kw)


def compare_strain(g, c, prec):
    s_g, gam_g = g.strain_rate()
    s_c, gam_c = c.strain_rate()
    scale = np.abs(s_c).max()
    tol = 1e-9 if prec == "f64" else 2e-3
    assert scale > 0
    assert np.abs(s_g - s_c).max() <= tol * scale, np.abs(s_g - s_c).max() / scale
    assert np.abs(gam_g - gam_c).max() <= tol * np.abs(gam_c).max()


@pytest.mark.parametrize("prec", ["f64", "f32"])
@pytest.mark.parametrize("q,coll", [(19, "trt"), (27, "cm")])
def test_strain_rate_cavity_matches_oracle(prec, q, coll):
    dims, solid, wall_u, nu = cavity(12, u_lid=0.06, re=40.0)
    os_ = 1.0 / (3.0 * nu + 0.5)
    g = lb.Solver(dims, lattice=q, collision=coll, storage=prec, nu=nu, omega_shear=os_, solid=solid, wall_u=wall_u)
    c = oracle_solver(dims, prec, q=q, collision=coll, nu=nu, omega_shear=os_, solid=solid, wall_u=wall_u)
    g.run(37)
    c.step(37)
    compare_strain(g, c, prec)
    s, gam = g.strain_rate()
    assert np.all(s[solid.astype(bool)] == 0.0) and np.all(gam[solid.astype(bool)] == 0.0)


@pytest.mark.parametrize("prec", ["f64", "f32"])
def test_strain_rate_forced_channel_matches_oracle(prec):
    from oracle import oracle as o
    dims = (6, 10, 6)
    solid, wall_u = o.wall_rims(dims, [False, False, True, True, False, False], np.zeros(18))
    kw = dict(nu=0.1, periodic=(True, False, True), force=(1e-5, 0.0, 2e-6), solid=solid, wall_u=wall_u)
    g = lb.Solver(dims, lattice=19, storage=prec, **kw)
    c = oracle_solver(dims, prec, **kw)
    g.run(60)
    c.step(60)
    compare_strain(g, c, prec)


@pytest.mark.parametrize("prec", ["f64", "f32"])
def test_strain_rate_tank_runner_with_ibm_field_matches_oracle(prec):
    c_ = sweep.TankCase(24, 0.04, 300.0)
    geo = sweep.tank_geometry(24)
    body = lb.RotatingBody(geo["center"], [0.0, 0.0, c_.omega], geo["marker_pos"], geo["marker_w"])
    g = lb.Solver(c_.dims, lattice=19, storage=prec, nu=c_.nu, solid=geo["solid"])
    c = oracle_solver(c_.dims, prec, q=19, nu=c_.nu, solid=geo["solid"])
    g.run_impeller(body, 30)
    c.run_tank(body.positions, body.weights, body.center, body.omega, 30)
    compare_strain(g, c, prec)


def cavity_state(prec="f64", n=14, steps=80):
    dims, solid, wall_u, nu = cavity(n, u_lid=0.06, re=60.0)
    g = lb.Solver(dims, storage=prec, nu=nu, solid=solid, wall_u=wall_u)
    g.run(steps)
    return g, dims, solid, wall_u


@pytest.mark.parametrize("prec", ["f64", "f32"])
def test_stress_field_matches_oracle_on_device_velocity(prec):
    from oracle import oracle as o
    g, dims, solid, _ = cavity_state(prec)
    _, ux, uy, uz = g.read_moments()
    vs = DX / DT
    ref = o.compute_stress_field(dims, ux * vs, uy * vs, uz * vs, solid, DX, MU)
    out = g.stress_field(DX, DT, MU)
    fl = solid == 0
    scale = np.abs(ref["gamma_dot"]).max()
    assert scale > 0
    assert np.abs(out["gamma_dot"] - ref["gamma_dot"])[fl].max() <= 1e-12 * scale
    assert np.abs(out["viscous_stress"] - ref["viscous_stress"])[fl].max() <= 1e-12 * MU * scale
    assert np.abs(out["s"] - ref["s"])[fl].max() <= 1e-12 * scale
    assert np.all(out["gamma_dot"][~fl] == 0.0)


@pytest.mark.parametrize("prec", ["f64", "f32"])
def test_stress_summary_matches_oracle_percentiles(prec):
    from oracle import oracle as o
    g, dims, solid, _ = cavity_state(prec, n=20, steps=120)
    _, ux, uy, uz = g.read_moments()
    vs = DX / DT
    ref = o.compute_stress_field(dims, ux * vs, uy * vs, uz * vs, solid, DX, MU)
    fl = solid == 0
    want_g = o.percentile_summary(ref["gamma_dot"][fl], 0.0)
    want_t = o.percentile_summary(ref["viscous_stress"][fl], 0.0)
    for _ in range(2):  # a second call sees the same state
        got_g, got_t, ms = g.stress_summary(DX, DT, MU, 0.0, 0.0)
        assert ms > 0 and got_g["count"] == int(fl.sum())
        for k in ("p50", "p90", "p95", "p99", "max"):
            assert abs(got_g[k] - want_g[k]) <= 1e-12 * want_g["max"], k
            assert abs(got_t[k] - want_t[k]) <= 1e-12 * want_t["max"], k
        assert got_g["fraction_above_threshold"] == want_g["fraction_above_threshold"]
        assert got_t["fraction_above_threshold"] == want_t["fraction_above_threshold"]
    # a threshold inside the distribution, and none
    t = want_g["p90"]
    got_g, _, _ = g.stress_summary(DX, DT, MU, t, None)
    assert got_g["fraction_above_threshold"] == o.percentile_summary(ref["gamma_dot"][fl], t)[
        "fraction_above_threshold"]
    _, got_t, _ = g.stress_summary(DX, DT, MU, None, None)
    assert got_t["fraction_above_threshold"] is None


def test_wall_shear_proxy_matches_oracle():
    from oracle import oracle as o
    g, dims, solid, wall_u = cavity_state("f64")
    _, ux, uy, uz = g.read_moments()
    vs = DX / DT
    ref = o.wall_shear_proxy(dims, ux * vs, uy * vs, uz * vs, solid, wall_u.reshape(-1, 3) * vs, DX, RHO, MU)
    got = g.wall_shear_proxy(DX, DT, RHO, MU)
    assert np.array_equal(got["cell_index"], ref["cell_index"])
    scale = ref["tau_w"].max()
    assert scale > 0
    assert np.abs(got["tau_w"] - ref["tau_w"]).max() <= 1e-12 * scale
    assert np.abs(got["u_parallel"] - ref["u_parallel"]).max() <= 1e-12 * ref["u_parallel"].max()
    assert np.abs(got["y_plus"] - ref["y_plus"]).max() <= 1e-12 * ref["y_plus"].max()
    assert np.abs(got["normal"] - ref["normal"]).max() <= 1e-14


def test_stress_rejects_bad_units():
    g, _, _, _ = cavity_state("f32", n=8, steps=2)
    with pytest.raises(lb.SpecError):
        g.stress_summary(0.0, DT, MU)
    with pytest.raises(lb.SpecError):
        g.stress_field(DX, DT, -1.0)
    with pytest.raises(lb.SpecError):
        g.wall_shear_proxy(DX, DT, 0.0, MU)
