"""Discrete adjoint of the runner loop against central finite differences.

J = mean torque over the second half of the run (fixed three IBM sweeps, no
early exit). The finite differences use the f64 forward through the public
runner (`run_impeller`), with the relative step 1e-4 on nu and Omega and a
step of 1e-6 cells along random marker-position directions (the linear IBM
kernel has kinks at integer positions; a small step keeps every marker on
one side of them). Markers that sit exactly on an integer coordinate are on
a kink, where J has no derivative, so the generated markers are moved by a
seeded jitter of at most 0.1 cell first. Tolerance: 1e-5 relative for the
f64 adjoint; the f32 adjoint agrees with the f64 gradient to 1e-3.
"""
import numpy as np
import pytest

import lbmflow_b200 as lb
from lbmflow_b200 import sweep

pytestmark = pytest.mark.gpu

STEPS, WIN, K = 48, 24, 16
CFG = lb.DirectForcingConfig(max_iterations=3, slip_tolerance=0.0)


def tank(T=20, u_tip=0.04, re=200.0):
    c = sweep.TankCase(T, u_tip, re)
    geo = dict(sweep.tank_geometry(T))
    rng = np.random.default_rng(7)
    geo["marker_pos"] = geo["marker_pos"] + rng.uniform(-0.1, 0.1, size=geo["marker_pos"].shape)
    return c, geo


def J_of(c, geo, storage, nu=None, omega=None, pos=None):
    g = lb.Solver(c.dims, lattice=19, collision="trt", storage=storage, nu=c.nu if nu is None else nu,
                  solid=geo["solid"])
    body = lb.RotatingBody(geo["center"], [0.0, 0.0, c.omega if omega is None else omega],
                           geo["marker_pos"] if pos is None else pos, geo["marker_w"])
    t = g.run_impeller(body, STEPS, CFG)["torque_lu"]
    g.close()
    return float(np.mean(t[WIN:]))


def adjoint(c, geo, storage):
    g = lb.Solver(c.dims, lattice=19, collision="trt", storage=storage, nu=c.nu, solid=geo["solid"])
    body = lb.RotatingBody(geo["center"], [0.0, 0.0, c.omega], geo["marker_pos"], geo["marker_w"])
    r = g.adjoint_torque(body, STEPS, WIN, K, CFG)
    g.close()
    return r


@pytest.fixture(scope="module")
def case():
    c, geo = tank()
    return c, geo, adjoint(c, geo, "f64")


def test_adjoint_forward_equals_runner(case):
    c, geo, r = case
    assert abs(r["J"] - J_of(c, geo, "f64")) <= 1e-14 * abs(r["J"])
    assert r["adjoint_ms"] > 0 and r["forward_ms"] > 0


def test_adjoint_dnu_matches_finite_difference(case):
    c, geo, r = case
    h = 1e-4 * c.nu
    fd = (J_of(c, geo, "f64", nu=c.nu + h) - J_of(c, geo, "f64", nu=c.nu - h)) / (2 * h)
    assert abs(r["dJ_dnu"] - fd) <= 1e-5 * abs(fd), (r["dJ_dnu"], fd)


def test_adjoint_domega_matches_finite_difference(case):
    c, geo, r = case
    h = 1e-4 * c.omega
    fd = (J_of(c, geo, "f64", omega=c.omega + h) - J_of(c, geo, "f64", omega=c.omega - h)) / (2 * h)
    assert abs(r["dJ_domega_z"] - fd) <= 1e-5 * abs(fd), (r["dJ_domega_z"], fd)


@pytest.mark.parametrize("seed", [1, 2, 3])
def test_adjoint_dpos_matches_finite_difference(case, seed):
    c, geo, r = case
    rng = np.random.default_rng(seed)
    d = rng.normal(size=geo["marker_pos"].shape)
    d /= np.linalg.norm(d)
    h = 1e-6
    p0 = geo["marker_pos"]
    fd = (J_of(c, geo, "f64", pos=p0 + h * d) - J_of(c, geo, "f64", pos=p0 - h * d)) / (2 * h)
    ad = float(np.sum(r["dJ_dpos"] * d))
    assert abs(ad - fd) <= 1e-5 * max(abs(fd), 1e-12) + 1e-9, (ad, fd)


def test_adjoint_f32_tracks_f64(case):
    c, geo, r64 = case
    r32 = adjoint(c, geo, "f32")
    assert abs(r32["dJ_dnu"] - r64["dJ_dnu"]) <= 1e-3 * abs(r64["dJ_dnu"])
    assert abs(r32["dJ_domega_z"] - r64["dJ_domega_z"]) <= 1e-3 * abs(r64["dJ_domega_z"])
    g32, g64 = r32["dJ_dpos"], r64["dJ_dpos"]
    assert np.linalg.norm(g32 - g64) <= 1e-3 * np.linalg.norm(g64)


def test_adjoint_rejects_unsupported():
    c, geo = tank()
    g = lb.Solver(c.dims, lattice=27, collision="cm", storage="f32", nu=c.nu, solid=geo["solid"])
    body = lb.RotatingBody(geo["center"], [0.0, 0.0, c.omega], geo["marker_pos"], geo["marker_w"])
    with pytest.raises(lb.UnsupportedError):
        g.adjoint_torque(body, 8, 4, 4, CFG)
    g = lb.Solver(c.dims, lattice=19, storage="f32", nu=c.nu, solid=geo["solid"], smagorinsky_cs=0.1)
    with pytest.raises(lb.UnsupportedError):
        g.adjoint_torque(body, 8, 4, 4, CFG)
