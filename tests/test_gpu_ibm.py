"""GPU parity of the direct-forcing IBM and the runner loop.

The IBM runs in f64 on the device over the stencil cells only; on the same
population state its diagnostics and the spread force field must match the
oracle (f64, summation-order noise only). The runner loop (clear force
field -> IBM -> step, per-step torque) is compared step by step.
"""
import math

import numpy as np
import pytest

import lbmflow_b200 as lb
from cases import seeded_state

pytestmark = pytest.mark.gpu

TAU = 2.0 * math.pi


def small_tank(n=32, impeller="rushton", baffles=True):
    spec = lb.TankSpec(dims=(n, n, n), dx_m=1.0 / n, vessel_diameter_m=1.0, liquid_height_m=1.0,
                       impeller_diameter_m=0.5, clearance_m=0.4, omega_rad_s=1.0, impeller=impeller,
                       baffle_count=4 if baffles else 0, baffle_width_m=0.1, baffle_thickness_m=2.5 / n,
                       min_cells=12.0)
    g = lb.build_stirred_tank(spec)
    omega = np.array([0.0, 0.0, 0.05 / (0.25 * n)])
    body = lb.RotatingBody(g["center"], omega, g["marker_pos"], g["marker_w"])
    return (n, n, n), g["solid"], body


def swirl_state(dims, solid, q, seed=3):
    """Smooth rotating flow with small noise, as deviation populations."""
    from oracle import oracle as o
    nx, ny, nz = dims
    z, y, x = np.meshgrid(np.arange(nz), np.arange(ny), np.arange(nx), indexing="ij")
    rx, ry = x - nx / 2 + 0.5, y - ny / 2 + 0.5
    u = np.stack([-0.004 * ry, 0.004 * rx, 0.001 * np.sin(z / 3.0)], -1).reshape(-1, 3) / max(nx, 1) * 4
    rho = np.ones(nx * ny * nz) + 1e-3 * np.cos(x / 2.0).ravel()
    feq = o.equilibrium_cells(q, 64, rho, u)
    return feq + seeded_state(q, feq.shape[1], seed, scale=1e-5)


def assert_diag_close(dg, do, tol):
    assert dg.iterations == do["iterations"]
    for k in ("slip_max", "slip_rms", "slip_max_rel", "slip_rms_rel"):
        assert abs(getattr(dg, k) - do[k]) <= tol * max(abs(do[k]), 1e-30), k
    for k in ("torque", "fluid_force", "marker_force"):
        a, b = getattr(dg, k), do[k]
        assert np.abs(a - b).max() <= tol * max(np.abs(b).max(), 1e-30), k
    assert dg.momentum_error_rel < 1e-9 and do["momentum_error_rel"] < 1e-9


@pytest.mark.parametrize("q", [19, 27])
@pytest.mark.parametrize("radius,iters,tol_slip", [(1, 3, 1e-2), (2, 4, 1e-3), (1, 5, 0.0)])
def test_ibm_apply_matches_oracle(q, radius, iters, tol_slip):
    from oracle import oracle as o
    dims, solid, body = small_tank()
    g = lb.Solver(dims, lattice=q, storage="f64", nu=0.02, solid=solid)
    c = o.OracleSolver(dims, q=q, real_bits=64, nu=0.02, solid=solid)
    f = swirl_state(dims, solid, q)
    g.stage_in(f)
    c.stage_in(f)
    cfg = lb.DirectForcingConfig(iters, tol_slip, radius, 1.0)
    dg = g.apply_rotating_ibm(body, cfg)
    do = c.ibm_apply(body.positions, body.weights, body.center, body.omega, iters, tol_slip, radius, 1.0)
    assert_diag_close(dg, do, 1e-10)
    fg, fc = g.force_field(), c.force_field()
    assert np.abs(fg - fc).max() <= 1e-12 * np.abs(fc).max()
    # a second application accumulates into the field (solver.rs:3256-3279)
    dg2 = g.apply_rotating_ibm(body, cfg)
    do2 = c.ibm_apply(body.positions, body.weights, body.center, body.omega, iters, tol_slip, radius, 1.0)
    assert_diag_close(dg2, do2, 1e-10)
    assert np.abs(g.force_field() - c.force_field()).max() <= 1e-12 * np.abs(c.force_field()).max()


def test_ibm_f32_storage_uses_same_u_now():
    # f32 populations staged identically: the f64 IBM sees the same u_now
    # and rho, so the diagnostics agree to f64 noise and the spread field to
    # one f32 rounding.
    from oracle import oracle as o
    dims, solid, body = small_tank()
    g = lb.Solver(dims, lattice=19, storage="f32", nu=0.02, solid=solid)
    c = o.OracleSolver(dims, q=19, real_bits=32, nu=0.02, solid=solid)
    f = swirl_state(dims, solid, 19).astype(np.float32).astype(np.float64)
    g.stage_in(f)
    c.stage_in(f)
    dg = g.apply_rotating_ibm(body)
    do = c.ibm_apply(body.positions, body.weights, body.center, body.omega)
    assert_diag_close(dg, do, 1e-10)
    fc = c.force_field()
    assert np.abs(g.force_field() - fc).max() <= 2e-7 * np.abs(fc).max()


@pytest.mark.parametrize("q,coll,prec", [(19, "trt", "f64"), (27, "cm", "f64"), (19, "trt", "f32")])
def test_runner_loop_torque_matches_oracle(q, coll, prec):
    from oracle import oracle as o
    dims, solid, body = small_tank(n=28)
    nu = 0.01
    os_ = 1.0 / (3.0 * nu + 0.5)
    bits = 64 if prec == "f64" else 32
    g = lb.Solver(dims, lattice=q, collision=coll, storage=prec, nu=nu, omega_shear=os_, solid=solid)
    c = o.OracleSolver(dims, q=q, real_bits=bits, collision=coll, nu=nu, omega_shear=os_, solid=solid)
    steps = 40  # graph-captured blocks of 16 + remainder
    rg = g.run_impeller(body, steps)
    rc = c.run_tank(body.positions, body.weights, body.center, body.omega, steps)
    tg, tc = rg["torque_lu"], rc["torque_lu"]
    assert np.array_equal(rg["ibm_iterations"], rc["ibm_iterations"].astype(np.int32))
    tol = 1e-9 if prec == "f64" else 2e-4
    assert np.abs(tg - tc).max() <= tol * np.abs(tc).max(), np.abs(tg - tc).max() / np.abs(tc).max()
    assert np.abs(rg["fluid_force"] - rc["fluid_force"]).max() <= tol * np.abs(rc["fluid_force"]).max()
    fl = solid == 0
    ug, uc = g.read_moments()[1][fl], c.moments()[1][fl]
    assert np.abs(ug - uc).max() <= (1e-9 if prec == "f64" else 1e-5) * np.abs(uc).max()


def test_runner_matches_host_driven_loop():
    # The device runner (graphs, device-side early exit) equals the same
    # loop driven call by call through the public API.
    dims, solid, body = small_tank(n=24)
    a = lb.Solver(dims, storage="f64", nu=0.02, solid=solid)
    b = lb.Solver(dims, storage="f64", nu=0.02, solid=solid)
    r = a.run_impeller(body, 20)
    tq = []
    for _ in range(20):
        b.clear_body_force_field()
        d = b.apply_rotating_ibm(body)
        b.run(1)
        tq.append(-d.torque[2])
    assert np.array_equal(r["torque_lu"], np.array(tq))
    assert np.array_equal(a.stage_out(), b.stage_out())


def _slab_cylinder(omega_z):
    # 3D analogue of the reference 2D rotating-cylinder KATs
    # (crates/lbm-core/tests/rotating_ibm.rs:71-140): a circle of 96 markers
    # (r = 8) in a 48 x 48 x 3 periodic box, quiescent fluid.
    g = lb.Solver((48, 48, 3), lattice=19, storage="f64", nu=1.0 / 6.0, periodic=(True, True, True))
    body = lb.RotatingBody.circle_2d([24.0, 24.0], 8.0, omega_z, 96, z=1.0)
    return g, body


def test_ibm_sweeps_reduce_slip_and_conserve_momentum():
    g1, body = _slab_cylinder(0.003)
    single = g1.apply_rotating_ibm(body, lb.DirectForcingConfig(1, 0.0, 2, 1.0))
    g2, body = _slab_cylinder(0.003)
    multi = g2.apply_rotating_ibm(body, lb.DirectForcingConfig(16, 0.0, 2, 1.0))
    assert multi.iterations == 16
    assert multi.slip_max_rel < single.slip_max_rel * 0.5
    assert multi.momentum_error_rel < 1e-3


def test_ibm_torque_flips_with_omega_sign():
    gp, bp = _slab_cylinder(0.003)
    gn, bn = _slab_cylinder(-0.003)
    cfg = lb.DirectForcingConfig(4, 1e-3, 2, 1.0)
    dp, dn = gp.apply_rotating_ibm(bp, cfg), gn.apply_rotating_ibm(bn, cfg)
    assert dp.torque[2] * dn.torque[2] < 0.0
    assert abs(dp.torque[2] + dn.torque[2]) / abs(dp.torque[2]) < 1e-12
    assert abs(dp.slip_max_rel - dn.slip_max_rel) < 1e-15


def test_ibm_rejects_bad_configs():
    g, body = _slab_cylinder(0.003)
    for cfg in (lb.DirectForcingConfig(0), lb.DirectForcingConfig(3, -1.0), lb.DirectForcingConfig(3, 1e-2, 3),
                lb.DirectForcingConfig(3, 1e-2, 1, 1.5)):
        with pytest.raises(lb.SpecError):
            g.apply_rotating_ibm(body, cfg)
    outside = lb.RotatingBody([0, 0, 0], [0, 0, 0.01], [[200.0, 5.0, 1.0]], [1.0])
    with pytest.raises(lb.SpecError):
        g.apply_rotating_ibm(outside)
