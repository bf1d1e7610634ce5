"""Free-slip (specular) top wall on the device against the oracle.

The top solid layer reflects populations leaving layer nz - 2 upwards into
the mirrored direction of the in-plane neighbour (bounce-back where that
neighbour is solid). Checked on a force-driven half channel (periodic in x
and y), in a closed box with side walls (partner-solid fallback at the
corners), through every sweep kernel kind, and in the IBM runner loop of a
small stirred tank with a free-slip liquid surface.
"""
import numpy as np
import pytest

import lbmflow_b200 as lb
from cases import Pair
from lbmflow_b200 import sweep

pytestmark = pytest.mark.gpu


def channel(dims=(6, 5, 12)):
    from oracle import oracle as o
    solid, wu = o.wall_rims(dims, [False, False, False, False, True, True], np.zeros(18))
    return solid, wu


@pytest.mark.parametrize("q,coll", [(19, "trt"), (27, "trt"), (27, "cm"), (19, "bgk")])
def test_half_channel_matches_oracle(q, coll):
    dims = (6, 5, 12)
    solid, wu = channel(dims)
    p = Pair(dims, q, "f64", collision=coll, nu=0.1, periodic=(True, True, False), force=(1e-5, 2e-6, 0),
             solid=solid, wall_u=wu, free_slip_top=True)
    p.run(45)
    p.check(solid == 0)
    p.run(2)
    p.check(solid == 0)


@pytest.mark.parametrize("kind", ["direct", "bulk", "async", "pair", "tile", "lean", "window"])
@pytest.mark.parametrize("q,coll", [(19, "trt"), (27, "cm")])
def test_closed_box_each_kernel_matches_oracle(kind, q, coll):
    # walls on every face, free-slip top, a swirl from a seeded state: no
    # uniform force, so every sweep kind that supports the form runs
    from oracle import oracle as o
    dims = (14, 12, 10)
    solid, wu = o.wall_rims(dims, [True] * 6, np.zeros(18))
    if coll == "cm" and kind == "lean":
        pytest.skip("TRT-only kernel")
    p = Pair(dims, q, "f32", collision=coll, nu=0.02, solid=solid, wall_u=wu, free_slip_top=True, sweep=kind)
    z, y, x = np.meshgrid(np.arange(10), np.arange(12), np.arange(14), indexing="ij")
    u = np.stack([0.02 * np.sin(y / 3.0), 0.02 * np.cos(x / 3.0), 0.01 * np.sin(x / 4.0)], -1).reshape(-1, 3)
    u[solid.astype(bool)] = 0.0
    p.init_with(np.ones(p.n), u)
    p.run(33)
    p.check(solid == 0)


def test_free_slip_conserves_mass_and_differs_from_lid():
    from oracle import oracle as o
    dims = (12, 12, 12)
    solid, wu = o.wall_rims(dims, [True] * 6, np.zeros(18))
    a = lb.Solver(dims, storage="f64", nu=0.05, solid=solid, wall_u=wu, free_slip_top=True, force=(1e-5, 0, 0))
    b = lb.Solver(dims, storage="f64", nu=0.05, solid=solid, wall_u=wu, free_slip_top=False, force=(1e-5, 0, 0))
    m0 = a.total_mass_f64()
    a.run(400)
    b.run(400)
    assert abs(a.total_mass_f64() - m0) < 1e-9
    ua = a.read_moments()[1].reshape(12, 12, 12)[:, 6, 6]
    ub = b.read_moments()[1].reshape(12, 12, 12)[:, 6, 6]
    assert ua[10] > 1.5 * ub[10]  # the surface layer slides


@pytest.mark.parametrize("prec", ["f64", "f32"])
def test_tank_runner_with_free_slip_surface(prec):
    from oracle import oracle as o
    c = sweep.TankCase(24, 0.04, 300.0)
    geo = sweep.tank_geometry(24)
    body = lb.RotatingBody(geo["center"], [0.0, 0.0, c.omega], geo["marker_pos"], geo["marker_w"])
    g = lb.Solver(c.dims, lattice=19, collision="trt", storage=prec, nu=c.nu, solid=geo["solid"],
                  free_slip_top=True)
    ref = o.OracleSolver(c.dims, q=19, real_bits=64 if prec == "f64" else 32, collision="trt", nu=c.nu,
                         solid=geo["solid"], free_slip_top=True)
    rg = g.run_impeller(body, 40)
    rc = ref.run_tank(body.positions, body.weights, body.center, body.omega, 40)
    tol = 1e-9 if prec == "f64" else 2e-4
    assert np.abs(rg["torque_lu"] - rc["torque_lu"]).max() <= tol * np.abs(rc["torque_lu"]).max()
    fl = geo["solid"] == 0
    ug, uc = g.read_moments()[1][fl], ref.moments()[1][fl]
    assert np.abs(ug - uc).max() <= (1e-9 if prec == "f64" else 1e-5) * np.abs(uc).max()


def test_adjoint_with_free_slip_matches_finite_difference():
    c = sweep.TankCase(20, 0.04, 200.0)
    geo = sweep.tank_geometry(20)
    cfg = lb.DirectForcingConfig(max_iterations=3, slip_tolerance=0.0)
    body = lb.RotatingBody(geo["center"], [0.0, 0.0, c.omega], geo["marker_pos"], geo["marker_w"])

    def J(nu):
        g = lb.Solver(c.dims, lattice=19, storage="f64", nu=nu, solid=geo["solid"], free_slip_top=True)
        t = g.run_impeller(body, 40, cfg)["torque_lu"]
        return float(np.mean(t[20:]))

    g = lb.Solver(c.dims, lattice=19, storage="f64", nu=c.nu, solid=geo["solid"], free_slip_top=True)
    r = g.adjoint_torque(body, 40, 20, 16, cfg)
    h = 1e-4 * c.nu
    fd = (J(c.nu + h) - J(c.nu - h)) / (2 * h)
    assert abs(r["dJ_dnu"] - fd) <= 1e-5 * abs(fd), (r["dJ_dnu"], fd)


def test_free_slip_needs_solid_z_faces():
    with pytest.raises(lb.SpecError):
        lb.Solver((8, 8, 8), nu=0.1, periodic=(True, True, True), free_slip_top=True)
