"""Every collide-stream kernel kind against the oracle.

The library has several sweep kernels for the same update (direct loads,
bulk copies staged in shared memory, a per-thread cp.async ring, and the
two-cells-per-thread packed-fp32x2 pair kernel). Each one must reproduce
the oracle on walls, moving walls, periodic wraps, the optional subgrid
model and the IBM runner loop; kinds that cannot run a configuration must
refuse it with UnsupportedError instead of silently changing the result.
"""
import numpy as np
import pytest

import lbmflow_b200 as lb
from cases import Pair, cavity, tgv_fields

pytestmark = pytest.mark.gpu

KINDS = ["direct", "bulk", "async", "pair", "tile", "lean", "window"]


def supported(kind, q, coll, prec, nx=14, force=False):
    if kind == "async" and prec in ("f16", "bf16"):
        return False
    if kind == "lean":
        return coll in ("trt", "bgk") and prec in ("f32", "f16", "bf16") and not force
    if kind == "window":
        return prec in ("f32", "f16", "bf16") and not force
    if kind in ("pair", "tile"):
        return prec in ("f32", "f16", "bf16") and nx % 2 == 0 and not force and (coll != "cm" or q == 27)
    return True


@pytest.mark.parametrize("kind", KINDS)
@pytest.mark.parametrize("q,coll", [(19, "trt"), (27, "trt"), (19, "bgk"), (27, "cm")])
@pytest.mark.parametrize("steps", [1, 2, 37])
def test_cavity_each_kernel_matches_oracle(kind, q, coll, steps):
    dims, solid, wall_u, nu = cavity(14, u_lid=0.06, re=40.0)
    if not supported(kind, q, coll, "f32"):
        g = lb.Solver(dims, lattice=q, collision=coll, storage="f32", nu=nu, solid=solid, wall_u=wall_u)
        with pytest.raises(lb.UnsupportedError):
            g.set_sweep_kernel(kind)
        return
    p = Pair(dims, q, "f32", collision=coll, nu=nu, solid=solid, wall_u=wall_u, sweep=kind)
    assert p.g.sweep_kernel == kind
    p.run(steps)
    p.check(solid == 0)


@pytest.mark.parametrize("kind", ["async", "pair", "tile", "lean", "window"])
@pytest.mark.parametrize("q", [19, 27])
def test_smagorinsky_each_kernel_matches_oracle(kind, q):
    dims, solid, wall_u, nu = cavity(14, u_lid=0.08, re=2000.0)
    p = Pair(dims, q, "f32", collision="trt", nu=nu, solid=solid, wall_u=wall_u, smagorinsky_cs=0.17, sweep=kind)
    p.run(45)
    p.check(solid == 0)


@pytest.mark.parametrize("kind", ["async", "pair", "tile", "window"])
def test_smagorinsky_central_moment_each_kernel(kind):
    dims, solid, wall_u, nu = cavity(14, u_lid=0.08, re=2000.0)
    p = Pair(dims, 27, "f32", collision="cm", nu=nu, solid=solid, wall_u=wall_u, smagorinsky_cs=0.17, sweep=kind)
    p.run(45)
    p.check(solid == 0)


@pytest.mark.parametrize("kind", KINDS)
def test_periodic_tgv_each_kernel(kind):
    # every cell is on or next to a periodic face at this size: wrap paths
    dims = (12, 10, 8)
    p = Pair(dims, 19, "f32", nu=0.02, periodic=(True, True, True), sweep=kind)
    rho, u = tgv_fields(dims)
    p.init_with(rho, u)
    p.run(41)
    p.check(np.ones(p.n, bool))


@pytest.mark.parametrize("kind,q,coll", [("pair", 19, "trt"), ("tile", 19, "trt"), ("lean", 19, "trt"),
                                         ("window", 19, "trt"), ("pair", 27, "cm"), ("tile", 27, "cm"),
                                         ("window", 27, "cm"), ("pair", 27, "trt")])
@pytest.mark.parametrize("prec", ["f16", "bf16"])
def test_pair_kernel_low_precision_matches_direct(prec, kind, q, coll):
    # Same storage, two kernels: the 16-bit rounding happens at the same
    # points, so the fields agree to a few storage ulps after 200 steps.
    dims, solid, wall_u, nu = cavity(24, re=50.0)
    a = lb.Solver(dims, lattice=q, collision=coll, storage=prec, nu=nu, solid=solid, wall_u=wall_u)
    b = lb.Solver(dims, lattice=q, collision=coll, storage=prec, nu=nu, solid=solid, wall_u=wall_u)
    a.set_sweep_kernel("direct")
    b.set_sweep_kernel(kind)
    a.run(200)
    b.run(200)
    ua, ub = a.read_moments()[1], b.read_moments()[1]
    fl = solid == 0
    eps = {"f16": 2.0 ** -10, "bf16": 2.0 ** -7}[prec]
    assert np.abs(ua - ub)[fl].max() <= 40 * eps * 0.06, np.abs(ua - ub)[fl].max()
    ref = lb.Solver(dims, lattice=q, collision=coll, storage="f32", nu=nu, solid=solid, wall_u=wall_u)
    ref.run(200)
    ur = ref.read_moments()[1].reshape(24, 24, 24)[:, 12, 12]
    l2 = np.linalg.norm(ub.reshape(24, 24, 24)[:, 12, 12] - ur) / np.linalg.norm(ur)
    assert l2 < {"f16": 5e-3, "bf16": 5e-2}[prec], l2


@pytest.mark.parametrize("kind", ["pair", "tile", "lean", "direct", "bulk", "async", "window"])
def test_runner_loop_each_kernel_matches_oracle(kind):
    from oracle import oracle as o
    n = 28
    spec = lb.TankSpec(dims=(n, n, n), dx_m=1.0 / n, vessel_diameter_m=1.0, liquid_height_m=1.0,
                       impeller_diameter_m=0.5, clearance_m=0.4, omega_rad_s=1.0, impeller="rushton",
                       baffle_count=4, baffle_width_m=0.1, baffle_thickness_m=2.5 / n, min_cells=12.0)
    geo = lb.build_stirred_tank(spec)
    body = lb.RotatingBody(geo["center"], [0.0, 0.0, 0.05 / (0.25 * n)], geo["marker_pos"], geo["marker_w"])
    solid = geo["solid"]
    nu = 0.01
    g = lb.Solver((n, n, n), lattice=19, collision="trt", storage="f32", nu=nu, solid=solid)
    g.set_sweep_kernel(kind)
    if kind == "async":
        g.set_sweep_variant(5, 6)  # 96 / 80 registers (3- / 2-tile ring)
    if kind == "window":
        g.set_sweep_variant(4, 2)  # 64 registers (2-tile ring) / 128
    c = o.OracleSolver((n, n, n), q=19, real_bits=32, collision="trt", nu=nu, solid=solid)
    rg = g.run_impeller(body, 40)
    rc = c.run_tank(body.positions, body.weights, body.center, body.omega, 40)
    tg, tc = rg["torque_lu"], rc["torque_lu"]
    assert np.abs(tg - tc).max() <= 2e-4 * np.abs(tc).max()
    fl = solid == 0
    ug, uc = g.read_moments()[1][fl], c.moments()[1][fl]
    assert np.abs(ug - uc).max() <= 1e-5 * np.abs(uc).max()


@pytest.mark.parametrize("budget", [(4, 4), (5, 5), (6, 6), (4, 6)])
@pytest.mark.parametrize("q,coll", [(19, "trt"), (27, "cm")])
def test_async_register_budgets_match_oracle(budget, q, coll):
    dims, solid, wall_u, nu = cavity(14, u_lid=0.06, re=40.0)
    p = Pair(dims, q, "f32", collision=coll, nu=nu, solid=solid, wall_u=wall_u, smagorinsky_cs=0.1, sweep="async")
    p.g.set_sweep_variant(*budget)
    p.run(23)
    p.check(solid == 0)


@pytest.mark.parametrize("kind,q,coll", [("lean", 19, "trt"), ("window", 19, "trt"), ("window", 27, "cm")])
def test_odd_nx_matches_oracle(kind, q, coll):
    dims, solid, wall_u, nu = cavity(13, u_lid=0.06, re=40.0)
    p = Pair(dims, q, "f32", collision=coll, nu=nu, solid=solid, wall_u=wall_u, sweep=kind)
    p.run(21)
    p.check(solid == 0)


@pytest.mark.parametrize("budget", [(2, 2), (3, 3), (4, 4), (2, 4)])
@pytest.mark.parametrize("prec", ["f32", "f16"])
def test_window_register_budgets(budget, prec):
    dims, solid, wall_u, nu = cavity(14, u_lid=0.06, re=40.0)
    a = lb.Solver(dims, lattice=19, storage=prec, nu=nu, solid=solid, wall_u=wall_u)
    b = lb.Solver(dims, lattice=19, storage=prec, nu=nu, solid=solid, wall_u=wall_u)
    a.set_sweep_kernel("lean")
    b.set_sweep_kernel("window")
    b.set_sweep_variant(*budget)
    a.run(31)
    b.run(31)
    ua, ub = a.read_moments()[1], b.read_moments()[1]
    assert np.abs(ua - ub)[solid == 0].max() <= 1e-5 * np.abs(ua).max()


def test_pair_kernel_refuses_what_it_cannot_run():
    dims, solid, wall_u, nu = cavity(13, re=40.0)  # odd nx
    g = lb.Solver(dims, storage="f32", nu=nu, solid=solid, wall_u=wall_u)
    for kind in ("pair", "tile"):
        with pytest.raises(lb.UnsupportedError):
            g.set_sweep_kernel(kind)
    assert g.sweep_kernel not in ("pair", "tile")
    dims, solid, wall_u, nu = cavity(14, re=40.0)
    g = lb.Solver(dims, storage="f32", nu=nu, solid=solid, wall_u=wall_u, force=(1e-6, 0, 0))
    for kind in ("pair", "lean", "window"):
        with pytest.raises(lb.UnsupportedError):
            g.set_sweep_kernel(kind)
    g = lb.Solver(dims, storage="f64", nu=nu, solid=solid, wall_u=wall_u)
    for kind in ("pair", "window"):
        with pytest.raises(lb.UnsupportedError):
            g.set_sweep_kernel(kind)
    g = lb.Solver(dims, lattice=27, collision="cm", storage="f32", nu=nu, solid=solid, wall_u=wall_u)
    with pytest.raises(lb.UnsupportedError):
        g.set_sweep_kernel("lean")
    g = lb.Solver(dims, storage="f16", nu=nu, solid=solid, wall_u=wall_u)
    with pytest.raises(lb.UnsupportedError):
        g.set_sweep_kernel("async")
    with pytest.raises(lb.SpecError):
        g.set_sweep_kernel(9)
    g = lb.Solver(dims, storage="f32", nu=nu, solid=solid, wall_u=wall_u)
    g.set_sweep_kernel("async")
    for bad in ((3, 4), (4, 7)):
        with pytest.raises(lb.SpecError):
            g.set_sweep_variant(*bad)


@pytest.mark.parametrize("prec,q", [("f32", 19), ("f16", 19), ("f32", 27), ("f64", 19)])
def test_autotune_keeps_state_and_picks_fastest(prec, q):
    dims, solid, wall_u, nu = cavity(16, u_lid=0.06, re=40.0)
    g = lb.Solver(dims, lattice=q, storage=prec, nu=nu, solid=solid, wall_u=wall_u)
    g.run(7)  # odd parity on entry
    before = g.stage_out()
    r = g.autotune_sweep(steps_per_trial=6)
    assert np.array_equal(g.stage_out(), before)
    assert r["n_trials"] if "n_trials" in r else len(r["trials"]) >= 1
    assert r["best_ms_per_step"] == min(t[3] for t in r["trials"])
    assert g.sweep_kernel == r["kind"]
    if prec == "f16":
        assert all(t[0] != "async" for t in r["trials"])
    if prec == "f64":
        assert {t[0] for t in r["trials"]} == {"direct", "async", "bulk"}
    # the tuned solver still follows the oracle
    if prec in ("f32",):
        p = Pair(dims, q, "f32", nu=nu, solid=solid, wall_u=wall_u)
        p.g.autotune_sweep(steps_per_trial=4)
        p.run(30)
        p.check(solid == 0)


@pytest.mark.parametrize("budget", [(3, 3), (4, 4), (5, 5), (3, 5)])
@pytest.mark.parametrize("prec", ["f32", "f16", "bf16"])
def test_pair_register_budgets(budget, prec):
    # every register budget of the TRT pair kernel against direct loads in
    # the same storage, on a walled cavity (wall selects) and a periodic box
    # (generic path)
    dims, solid, wall_u, nu = cavity(18, u_lid=0.06, re=40.0)
    a = lb.Solver(dims, lattice=19, storage=prec, nu=nu, solid=solid, wall_u=wall_u)
    b = lb.Solver(dims, lattice=19, storage=prec, nu=nu, solid=solid, wall_u=wall_u)
    a.set_sweep_kernel("direct")
    b.set_sweep_kernel("pair")
    b.set_sweep_variant(*budget)
    a.run(31)
    b.run(31)
    ua, ub = a.read_moments()[1], b.read_moments()[1]
    tol = {"f32": 1e-5, "f16": 40 * 2.0 ** -10, "bf16": 40 * 2.0 ** -7}[prec]
    assert np.abs(ua - ub)[solid == 0].max() <= tol * max(np.abs(ua).max(), 1e-3)


@pytest.mark.parametrize("budget", [(3, 3), (4, 4), (5, 5), (4, 3)])
@pytest.mark.parametrize("q,coll,prec", [(19, "trt", "f32"), (19, "trt", "f16"), (19, "trt", "bf16"),
                                         (27, "cm", "f32"), (27, "cm", "f16")])
def test_pair_staged_matches_direct(budget, q, coll, prec):
    # the cp.async-staged pair kernel reads the same bytes as the direct one
    # (pairs, odd-offset pairs, wall links' own slots, 16-bit words split by
    # element): the populations must agree bit for bit, on a walled cavity
    # whose x extent leaves half-solid pairs at both ends of every row
    dims, solid, wall_u, nu = cavity(19, u_lid=0.06, re=40.0)
    dims = (dims[0] + 1, dims[1], dims[2])  # even nx: 20 cells, walls at x = 0 and 19
    s3 = np.zeros((dims[2], dims[1], dims[0]), np.uint8)
    s3[:, :, :19] = solid.reshape(dims[2], dims[1], 19)
    s3[:, :, 19] = 1
    solid = s3.ravel()
    w3 = np.zeros((dims[2], dims[1], dims[0], 3))
    w3[:, :, :19] = wall_u.reshape(dims[2], dims[1], 19, 3)
    wall_u = w3.reshape(-1, 3)
    runs = []
    for staged in (False, True):
        s = lb.Solver(dims, lattice=q, collision=coll, storage=prec, nu=nu, solid=solid, wall_u=wall_u)
        s.set_sweep_kernel("pair")
        s.set_sweep_variant(*(b + (10 if staged else 0) for b in budget))
        s.run(23)
        runs.append(s.stage_out())
        s.close()
    assert np.array_equal(runs[0], runs[1])
