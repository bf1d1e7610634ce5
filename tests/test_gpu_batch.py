"""Batched runner: many tanks of different sizes advanced in lockstep.

Every case of a batch must follow exactly the sequence it follows alone
(same kernels, same IBM reduction order, same early exit), so the batched
torque series and populations are compared bit for bit with each case run
through its own runner loop on the lean sweep kernel.
"""
import numpy as np
import pytest

import lbmflow_b200 as lb
from lbmflow_b200 import sweep

pytestmark = pytest.mark.gpu


def small_cases():
    return [sweep.TankCase(20, 0.04, 300.0, index=0), sweep.TankCase(27, 0.03, 800.0, index=1),
            sweep.TankCase(32, 0.05, 600.0, index=2)]


@pytest.mark.parametrize("storage", ["f32", "f16"])
def test_batch_equals_each_case_alone(storage):
    cases = small_cases()
    steps = 37  # graph blocks of 16 + remainder, odd end parity
    built = [sweep.build_case(c, storage=storage) for c in cases]
    alone = [sweep.build_case(c, storage=storage) for c in cases]
    b = lb.Batch([g for g, _ in built], [body for _, body in built])
    tq, ms = b.run(steps)
    assert ms > 0 and tq.shape == (3, steps)
    for k, (g, body) in enumerate(alone):
        assert g.sweep_kernel == "lean"
        r = g.run_impeller(body, steps)
        assert np.array_equal(tq[k], r["torque_lu"]), k
        assert np.array_equal(built[k][0].stage_out(), g.stage_out()), k
    # a second call continues from the stored parity and force field
    tq2, _ = b.run(5)
    for k, (g, body) in enumerate(alone):
        assert np.array_equal(tq2[k], g.run_impeller(body, 5)["torque_lu"])
    b.close()


def test_batch_autotune_keeps_state():
    cases = small_cases()
    built = [sweep.build_case(c) for c in cases]
    b = lb.Batch([g for g, _ in built], [body for _, body in built])
    b.run(3)
    before = [g.stage_out() for g, _ in built]
    r = b.autotune(4)
    assert r["even_blocks_per_sm"] in (6, 7, 8) and r["odd_blocks_per_sm"] in (6, 7, 8)
    assert r["best_ms_per_step"] > 0
    for (g, _), f in zip(built, before):
        assert np.array_equal(g.stage_out(), f)


def test_batch_matches_oracle_runner():
    from oracle import oracle as o
    c = sweep.TankCase(24, 0.04, 400.0)
    g, body = sweep.build_case(c, les_cs=0.0)
    geo = sweep.tank_geometry(c.T)
    ref = o.OracleSolver(c.dims, q=19, real_bits=32, collision="trt", nu=c.nu, solid=geo["solid"])
    b = lb.Batch([g], [body])
    tq, _ = b.run(30)
    rc = ref.run_tank(body.positions, body.weights, body.center, body.omega, 30)
    assert np.abs(tq[0] - rc["torque_lu"]).max() <= 2e-4 * np.abs(rc["torque_lu"]).max()


def test_sweep_batch_and_sequential_agree():
    cases = sweep.seeded_cases(n=4, t_range=(20, 36))
    a = sweep.run_sweep(cases, 24, mode="batch", autotune=False)
    s = sweep.run_sweep(cases, 24, mode="sequential", autotune=False)
    assert [p["Np"] for p in a["per_case"]] == [p["Np"] for p in s["per_case"]]
    assert a["aggregate"]["Np"]["count"] == 4
    assert a["mlups"] > 0 and s["mlups"] > 0


def test_batch_rejects_mixed_or_unsupported():
    c = small_cases()
    g1, b1 = sweep.build_case(c[0], storage="f32")
    g2, b2 = sweep.build_case(c[1], storage="f16")
    with pytest.raises(lb.SpecError):
        lb.Batch([g1, g2], [b1, b2])
    geo = sweep.tank_geometry(20)
    body = lb.RotatingBody(geo["center"], [0, 0, 0.01], geo["marker_pos"], geo["marker_w"])
    cm = lb.Solver(c[0].dims, lattice=27, collision="cm", storage="f32", nu=0.01, solid=geo["solid"])
    with pytest.raises(lb.UnsupportedError):
        lb.Batch([cm], [body])
    sc = lb.Solver(c[0].dims, lattice=19, storage="f32", nu=0.01, solid=geo["solid"])
    sc.enable_scalar_distribution(1e-3, q=7)
    with pytest.raises(lb.UnsupportedError):
        lb.Batch([sc], [body])
