"""The device runner loop across calls and its divergence abort.

The runner (crates/lbm-cli/src/runner.rs:1079-1129) steps clear force field
-> IBM -> step and, after every 1000th step, stops with status "diverged"
when the f64 total mass is no longer finite (runner.rs:1125-1128). The
device runner keeps its captured graph and series buffers between calls;
split runs must equal one long run bit for bit.
"""
import numpy as np
import pytest

import lbmflow_b200 as lb
from test_gpu_ibm import small_tank

pytestmark = pytest.mark.gpu


def _tank_solver(n=24, storage="f64", coll="trt", q=19):
    dims, solid, body = small_tank(n=n)
    nu = 0.02
    g = lb.Solver(dims, lattice=q, collision=coll, storage=storage, nu=nu, omega_shear=1.0 / (3 * nu + 0.5),
                  solid=solid)
    return g, body, dims, solid


@pytest.mark.parametrize("storage", ["f64", "f32"])
def test_split_runs_equal_one_run(storage):
    a, body, _, _ = _tank_solver(storage=storage)
    b, _, _, _ = _tank_solver(storage=storage)
    ra = a.run_impeller(body, 80)
    parts = [b.run_impeller(body, k) for k in (33, 16, 31)]  # odd starts, graph reuse, remainders
    tb = np.concatenate([p["torque_lu"] for p in parts])
    assert np.array_equal(ra["torque_lu"], tb)
    assert np.array_equal(a.stage_out(), b.stage_out())
    assert all(p["status"] == "completed" for p in parts) and ra["executed"] == 80


def test_runner_graph_follows_sweep_kernel_change():
    a, body, _, _ = _tank_solver(storage="f32")
    b, _, _, _ = _tank_solver(storage="f32")
    a.set_sweep_kernel("direct")
    ra = a.run_impeller(body, 32)
    rb1 = b.run_impeller(body, 16)
    b.set_sweep_kernel("direct")
    rb2 = b.run_impeller(body, 16)
    assert b.sweep_kernel == "direct"
    # the two sweep kernels compute the same update up to fp32 rounding
    tb = np.concatenate([rb1["torque_lu"], rb2["torque_lu"]])
    assert np.abs(ra["torque_lu"] - tb).max() <= 1e-4 * np.abs(ra["torque_lu"]).max()


def test_runner_stops_on_non_finite_mass():
    from oracle import oracle as o
    g, body, dims, solid = _tank_solver(n=24)
    c = o.OracleSolver(dims, q=19, real_bits=64, nu=0.02, solid=solid)
    f = g.stage_out()
    fluid = np.flatnonzero(solid == 0)
    f[3, fluid[len(fluid) // 3]] = np.nan  # a NaN population staged on the host
    g.stage_in(f)
    c.stage_in(f)
    steps = 2500
    rg = g.run_impeller(body, steps)
    rc = c.run_tank(body.positions, body.weights, body.center, body.omega, steps)
    assert rc["executed"] == 1000
    assert rg["status"] == "diverged" and rg["executed"] == 1000
    assert np.isnan(rg["torque_lu"][1000:]).all()
    assert (rg["ibm_iterations"][1000:] == 0).all()
    assert g.time == 1000
    # the error code reaches a C-ABI caller
    import ctypes as C
    tq = np.empty(10)
    rc2 = lb.lib().lbmb_run_impeller(g.h, g._slot_for(body), C.byref(lb.DirectForcingConfig()._c()), 10, -1, 1,
                                     tq.ctypes.data_as(C.POINTER(C.c_double)), None, None, None)
    assert rc2 == lb.OK  # fewer than 1000 steps: no check inside the call
    rc3 = lb.lib().lbmb_run_impeller(g.h, g._slot_for(body), C.byref(lb.DirectForcingConfig()._c()), 1000, -1, 1,
                                     None, None, None, None)
    assert rc3 == lb.ERR_DIVERGED
    ex, dv = C.c_int64(), C.c_int32()
    assert lb.lib().lbmb_run_impeller_status(g.h, C.byref(ex), C.byref(dv)) == lb.OK
    assert ex.value == 1000 and dv.value == 1


def test_runner_timing_excludes_first_capture():
    # The captured graph is kept: a second short call reports the device
    # time of its steps, close to the first call's steady-state rate.
    g, body, _, _ = _tank_solver(n=32, storage="f32")
    g.run_impeller(body, 32)
    t1 = g.last_timing()
    g.run_impeller(body, 32)
    t2 = g.last_timing()
    assert t1[2] == 32 and t2[2] == 32
    assert t2[0] > 0.0


@pytest.mark.parametrize("storage,kind", [("f64", None), ("f32", "pair"), ("f16", "pair"), ("f32", "direct")])
def test_runner_step_equals_the_four_calls(storage, kind):
    # lbmb_runner_step overlaps the direct forcing with the full-grid sweep;
    # it must give what the reference loop's calls give one after another
    # (runner.rs:1080-1085): clear field, upload markers, apply, step
    a, body, _, _ = _tank_solver(storage=storage, coll="cm", q=27)
    b, _, _, _ = _tank_solver(storage=storage, coll="cm", q=27)
    if kind:
        a.set_sweep_kernel(kind)
        b.set_sweep_kernel(kind)
    cfg = lb.DirectForcingConfig()
    for step in range(9):  # odd count: both parities, twice
        a.clear_body_force_field()
        a.set_body(0, body)
        da = a.apply_rotating_ibm(body, cfg)
        a.run(1)
        db = b.runner_step(0, body, cfg)
        assert da.iterations == db.iterations
        assert np.array_equal(da.torque, db.torque) and np.array_equal(da.fluid_force, db.fluid_force)
        assert da.slip_max == db.slip_max
    assert np.array_equal(a.stage_out(), b.stage_out())
    # and the device runner takes over from it without a seam
    ra = a.run_impeller(body, 6)
    rb = b.run_impeller(body, 6)
    assert np.array_equal(ra["torque_lu"], rb["torque_lu"])
