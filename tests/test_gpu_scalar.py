"""GPU parity of the passive-scalar ADE (solver.rs:2113-2205) on D3Q7 and on
the hydro lattice, and of the device-side mixing index (qoi.rs:507-532)."""
import numpy as np
import pytest

import lbmflow_b200 as lb
from cases import cavity, tgv_fields

pytestmark = pytest.mark.gpu


def test_uniform_scalar_stays_uniform():
    # crates/lbm-core/src/solver.rs:5922-5946
    g = lb.Solver((6, 5, 4), lattice=19, storage="f64", nu=0.08, periodic=(True, True, True))
    k = g.enable_scalar_distribution(0.02)
    g.set_scalar_concentration(k, np.full(g.n, 2.0))
    g.run(8)
    assert np.abs(g.gather_scalar_concentration(k) - 2.0).max() < 1e-12


@pytest.mark.parametrize("sq", [19, 7])
def test_closed_domain_scalar_mass_conserved(sq):
    # crates/lbm-core/src/solver.rs:5948-5990
    dims = (10, 10, 10)
    solid, wu = lb.build_wall_rims(dims, [True] * 6, np.zeros(18))
    g = lb.Solver(dims, lattice=19, storage="f64", nu=0.08, solid=solid, wall_u=wu)
    k = g.enable_scalar_distribution(0.02, q=sq)
    c0 = np.zeros((10, 10, 10))
    c0[4:6, 4:6, 4:6] = 1.0
    g.set_scalar_concentration(k, c0.ravel())
    g.run(20)
    c1 = g.gather_scalar_concentration(k)
    assert abs(c1.sum() - c0.sum()) < 1e-10
    assert c1[(5 * 10 + 5) * 10 + 5] < 1.0


@pytest.mark.parametrize("sq", [19, 7])
def test_scalar_advects_with_flow(sq):
    # crates/lbm-core/src/solver.rs:5992-6035
    dims = (24, 8, 6)
    g = lb.Solver(dims, lattice=19, storage="f64", nu=0.08, periodic=(True, True, True))
    g.init_with(np.ones(g.n), np.tile([0.04, 0.0, 0.0], g.n))
    k = g.enable_scalar_distribution(0.01, q=sq)
    c0 = np.zeros(dims[::-1])
    c0[:, :, 4:7] = 1.0
    c0 = c0.ravel()
    g.set_scalar_concentration(k, c0)
    x = np.tile(np.arange(dims[0]), dims[1] * dims[2])
    before = (x * c0).sum() / c0.sum()
    g.run(10)
    c1 = g.gather_scalar_concentration(k)
    assert (x * c1).sum() / c1.sum() > before


@pytest.mark.parametrize("q,sq,prec", [(19, 19, "f64"), (19, 7, "f64"), (27, 27, "f64"), (27, 7, "f64"),
                                       (19, 7, "f32")])
def test_scalar_in_cavity_matches_oracle(q, sq, prec):
    from oracle import oracle as o
    dims, solid, wall_u, nu = cavity(14, re=20.0)
    bits = 64 if prec == "f64" else 32
    g = lb.Solver(dims, lattice=q, storage=prec, nu=nu, solid=solid, wall_u=wall_u)
    c = o.OracleSolver(dims, q=q, real_bits=bits, nu=nu, solid=solid, wall_u=wall_u)
    c64 = o.OracleSolver(dims, q=q, real_bits=64, nu=nu, solid=solid, wall_u=wall_u)
    g.run(20)
    c.step(20)
    c64.step(20)
    rng = np.random.default_rng(11)
    conc = np.where(solid == 0, rng.uniform(0.0, 1.0, g.n), 0.0)
    kg = g.enable_scalar_distribution(0.01, q=sq)
    g.set_scalar_concentration(kg, conc)
    for s in (c, c64):
        ks = s.scalar_enable(0.01, q=sq)
        s.scalar_set(ks, conc)
    g.run(25)
    c.step(25)
    c64.step(25)
    fl = solid == 0
    cg, cc, ce = g.gather_scalar_concentration(kg)[fl], c.scalar_get(0)[fl], c64.scalar_get(0)[fl]
    if prec == "f64":
        assert np.abs(cg - cc).max() < 1e-11
    else:
        assert np.abs(cg - ce).max() <= 3.0 * np.abs(cc - ce).max() + 1e-9
    cv_ref = o.scalar_cv(cc, np.ones(cc.size))
    cv_tol = 1e-9 if prec == "f64" else 1e-6  # f32 concentrations carry ~1e-7 relative rounding
    assert abs(g.scalar_cv(kg) - cv_ref) < cv_tol * max(cv_ref, 1.0)


def test_runner_cv_probes_on_device():
    from oracle import oracle as o
    n = 24
    spec = lb.TankSpec(dims=(n, n, n), dx_m=1.0 / n, vessel_diameter_m=1.0, liquid_height_m=1.0,
                       impeller_diameter_m=0.5, clearance_m=0.4, omega_rad_s=1.0, min_cells=12.0)
    geo = lb.build_stirred_tank(spec)
    body = lb.RotatingBody(geo["center"], [0.0, 0.0, 0.05 / 6.0], geo["marker_pos"], geo["marker_w"])
    solid = geo["solid"]
    g = lb.Solver((n, n, n), lattice=19, storage="f64", nu=0.02, solid=solid)
    c = o.OracleSolver((n, n, n), q=19, real_bits=64, nu=0.02, solid=solid)
    z = np.repeat(np.arange(n), n * n)
    conc = np.where((solid == 0) & (z > n - 6), 1.0, 0.0)
    kg = g.enable_scalar_distribution(1e-3, q=19)
    g.set_scalar_concentration(kg, conc)
    kc = c.scalar_enable(1e-3, q=19)
    c.scalar_set(kc, conc)
    rg = g.run_impeller(body, 12, scalar=kg, probe_every=4)
    rc = c.run_tank(body.positions, body.weights, body.center, body.omega, 12, probe_every=4, scalar=kc)
    probed = ~np.isnan(rc["cv"])
    assert np.array_equal(probed, ~np.isnan(rg["cv"]))
    assert np.abs(rg["cv"][probed] - rc["cv"][probed]).max() < 1e-9
    assert np.abs(rg["torque_lu"] - rc["torque_lu"]).max() <= 1e-9 * np.abs(rc["torque_lu"]).max()
