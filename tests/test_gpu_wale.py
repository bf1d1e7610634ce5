"""Per-cell relaxation field, velocity gradient and WALE LES on the device
against the oracle (which is pinned to the reference's wale_les.rs tests).

* A uniform field equal to the configured rate gives the field-off result to
  5 f64 ulps (the reference's own band: the two paths differ only in where
  c+ = 1 - omega+/2 is evaluated).
* A seeded non-uniform field: every sweep kernel that takes it follows the
  oracle (1e-11 f64, 1e-5 f32 relative).
* Velocity gradient and WALE nu_t / diagnostics on the device velocity equal
  the oracle's (1e-12 of the maximum in f64; clip counts exact), and after
  the update both advance with the installed field alike.
"""
import numpy as np
import pytest

import lbmflow_b200 as lb
from cases import TOL, cavity

pytestmark = pytest.mark.gpu

FIELD_KINDS = ["direct", "bulk", "window"]


def oracle(dims, prec, **kw):
    from oracle import oracle as o
    return o.OracleSolver(dims, q=kw.pop("q", 19), real_bits=64 if prec == "f64" else 32, **kw)


def periodic_state(n=12, nu=0.02, u0=0.04):
    k1, k2 = 2 * np.pi / n, 4 * np.pi / n
    z, y, x = np.meshgrid(np.arange(n), np.arange(n), np.arange(n), indexing="ij")
    u = np.stack([u0 * np.sin(k1 * x) * np.cos(k1 * y) * np.cos(k1 * z),
                  -u0 * np.cos(k1 * x) * np.sin(k1 * y) * np.cos(k1 * z) + 0.5 * u0 * np.sin(k2 * y) * np.cos(k2 * z),
                  -0.5 * u0 * np.cos(k2 * y) * np.sin(k2 * z)], -1).reshape(-1, 3)
    return (n, n, n), np.ones(n ** 3), u, nu


@pytest.mark.parametrize("kind", ["direct", "window"])
def test_uniform_field_equals_field_off(kind):
    dims, rho, u, nu = periodic_state()
    st = "f64" if kind == "direct" else "f32"
    off = lb.Solver(dims, storage=st, nu=nu, periodic=(True, True, True))
    on = lb.Solver(dims, storage=st, nu=nu, periodic=(True, True, True))
    for g in (off, on):
        g.set_sweep_kernel(kind)
        g.init_with(rho, u)
    on.set_omega_field(np.full(on.n, 1.0 / (3.0 * nu + 0.5)))
    assert on.sweep_kernel == kind
    off.run(7)
    on.run(7)
    eps = np.finfo(np.float64 if st == "f64" else np.float32).eps
    a, b = off.stage_out(), on.stage_out()
    assert np.abs(a - b).max() <= 5 * eps * max(np.abs(a).max(), 1.0)


@pytest.mark.parametrize("kind", FIELD_KINDS)
@pytest.mark.parametrize("q,coll", [(19, "trt"), (27, "cm")])
def test_nonuniform_field_matches_oracle(kind, q, coll):
    dims, solid, wall_u, nu = cavity(14, u_lid=0.06, re=40.0)
    prec = "f64" if kind in ("direct", "bulk") else "f32"
    os_ = 1.0 / (3.0 * nu + 0.5)
    g = lb.Solver(dims, lattice=q, collision=coll, storage=prec, nu=nu, omega_shear=os_, solid=solid, wall_u=wall_u)
    c = oracle(dims, prec, q=q, collision=coll, nu=nu, omega_shear=os_, solid=solid, wall_u=wall_u)
    g.set_sweep_kernel(kind)
    om = np.random.default_rng(11).uniform(1.2, 1.9, g.n)
    g.set_omega_field(om)
    c.set_omega_field(om)
    g.run(23)
    c.step(23)
    fl = solid == 0
    ug, uc = g.read_moments()[1][fl], c.moments()[1][fl]
    assert np.abs(ug - uc).max() <= TOL[prec] * np.abs(uc).max()


@pytest.mark.parametrize("prec", ["f64", "f32"])
def test_velocity_gradient_matches_oracle(prec):
    dims, solid, wall_u, nu = cavity(12, u_lid=0.06, re=40.0)
    g = lb.Solver(dims, storage=prec, nu=nu, solid=solid, wall_u=wall_u)
    c = oracle(dims, prec, nu=nu, solid=solid, wall_u=wall_u)
    g.run(31)
    c.step(31)
    gg, gc = g.velocity_gradient(), c.velocity_gradient()
    tol = 1e-9 if prec == "f64" else 2e-3
    assert np.abs(gg - gc).max() <= tol * np.abs(gc).max()
    assert np.all(gg[solid.astype(bool)] == 0.0)


@pytest.mark.parametrize("prec", ["f64", "f32"])
@pytest.mark.parametrize("bound", [None, "quarter"])
def test_wale_update_matches_oracle_and_steps_alike(prec, bound):
    dims, rho, u, nu = periodic_state()
    g = lb.Solver(dims, storage=prec, nu=nu, periodic=(True, True, True))
    c = oracle(dims, prec, nu=nu, periodic=(True, True, True))
    g.init_with(rho, u)
    c.init_with(rho, u)
    g.run(3)
    c.step(3)
    tau_max = None
    if bound:
        raw, _ = c.wale_update()
        tau_max = 0.5 + 3.0 * (nu + np.sort(raw)[raw.size // 4])
    nu_g, dg = g.wale_update(tau_max)
    nu_c, dc = c.wale_update(tau_max)
    tol = 1e-12 if prec == "f64" else 1e-3
    assert np.abs(nu_g - nu_c).max() <= tol * nu_c.max()
    if prec == "f64":
        assert dg["clipped_cells"] == dc["clipped_cells"]
    assert abs(dg["max_nu_t_before_clipping"] - dc["max_nu_t_before_clipping"]) <= tol * dc["max_nu_t_before_clipping"]
    if bound:
        assert dg["clipped_cells"] > 0 and dg["nu_t_max"] is not None
    g.run(11)
    c.step(11)
    ug, uc = g.read_moments()[1], c.moments()[1]
    assert np.abs(ug - uc).max() <= TOL[prec] * np.abs(uc).max()


def test_field_refusals_and_removal():
    dims, solid, wall_u, nu = cavity(12, re=40.0)
    g = lb.Solver(dims, storage="f32", nu=nu, solid=solid, wall_u=wall_u)
    g.set_sweep_kernel("pair")
    g.set_omega_field(np.full(g.n, 1.5))
    assert g.sweep_kernel == "window"
    for kind in ("tile", "pair", "lean", "async"):
        with pytest.raises(lb.UnsupportedError):
            g.set_sweep_kernel(kind)
    assert {t[0] for t in g.autotune_sweep(4)["trials"]} <= {"direct", "bulk", "window"}
    g.set_omega_field(None)
    g.set_sweep_kernel("pair")
    s = lb.Solver(dims, storage="f32", nu=nu, solid=solid, wall_u=wall_u, smagorinsky_cs=0.1)
    with pytest.raises(lb.UnsupportedError):
        s.set_omega_field(np.full(s.n, 1.5))
    with pytest.raises(lb.UnsupportedError):
        s.wale_update()
    with pytest.raises(lb.SpecError):
        g.wale_update(0.4)
