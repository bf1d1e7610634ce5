"""Checkpoint/restart of the device solver in the reference's v3 format.

* Resume is bit-exact (Solver::save / restore, the reference's
  checkpoint_resume_bit_exact test, solver.rs:6296-6302): run K+M equals run
  K, save, restore into a fresh solver, run M, for every storage precision,
  both lattices, odd and even K (the in-place layout's parity differs between
  the two runs), every sweep kernel, and the stirred-tank runner loop with
  its IBM force field and a D3Q7 scalar.
* The device's checkpoint at step K equals the oracle's checkpoint of the
  same run: identical manifest (hashes, sizes), populations and moments
  within the f64 parity tolerance (1e-11 of the maximum).
* Files cross between the two: an oracle checkpoint restored on the device
  continues like the oracle, and a device checkpoint restored in the oracle
  continues like the device.
* A refused restore leaves the solver untouched.
"""
import json

import numpy as np
import pytest

import lbmflow_b200 as lb
from cases import TOL, cavity
from oracle import checkpoint as ock
from oracle import oracle as o

pytestmark = pytest.mark.gpu


def tank_kw(q, coll, prec, n=14):
    dims, solid, wall_u, nu = cavity(n, u_lid=0.06, re=60.0)
    return dict(dims=dims, lattice=q, collision=coll, storage=prec, nu=nu, solid=solid, wall_u=wall_u,
                force=(0.0, 0.0, 0.0))


def make(kw, sweep=None):
    k = dict(kw)
    dims = k.pop("dims")
    g = lb.Solver(dims, **k)
    if sweep:
        g.set_sweep_kernel(sweep)
    return g


def assert_same_state(a, b):
    assert a.time == b.time
    fa, fb = a.stage_out(), b.stage_out()
    assert np.array_equal(fa, fb), np.abs(fa - fb).max()
    for x, y in zip(a.read_moments(), b.read_moments()):
        assert np.array_equal(x, y)


@pytest.mark.parametrize("prec", ["f64", "f32", "f16", "bf16"])
@pytest.mark.parametrize("q,coll", [(19, "trt"), (27, "cm")])
@pytest.mark.parametrize("k", [6, 7])
def test_resume_is_bit_exact(tmp_path, prec, q, coll, k):
    kw = tank_kw(q, coll, prec)
    cont, part = make(kw), make(kw)
    cont.run(k + 9)
    part.run(k)
    part.save(str(tmp_path))
    m = json.loads((tmp_path / "manifest.json").read_text())
    assert m["step"] == k and m["dtype"] == ("f64" if prec == "f64" else "f32")
    fresh = make(kw)
    fresh.restore(str(tmp_path))
    assert fresh.time == k
    fresh.run(9)
    assert_same_state(cont, fresh)


@pytest.mark.parametrize("q,coll,kind", [(27, "cm", "direct"), (27, "cm", "bulk"), (27, "cm", "async"),
                                         (27, "cm", "pair"), (27, "cm", "tile"), (27, "cm", "window"),
                                         (19, "trt", "lean"), (19, "trt", "window")])
def test_resume_is_bit_exact_for_every_sweep_kernel(tmp_path, q, coll, kind):
    kw = tank_kw(q, coll, "f32", n=16)
    cont, part = make(kw, kind), make(kw, kind)
    assert cont.sweep_kernel == kind
    cont.run(7 + 40)
    part.run(7)
    part.save(str(tmp_path))
    fresh = make(kw, kind)
    fresh.restore(str(tmp_path))
    fresh.run(40)
    assert_same_state(cont, fresh)


def small_tank(n=24):
    spec = lb.TankSpec(dims=(n, n, n), dx_m=1.0 / n, vessel_diameter_m=1.0, liquid_height_m=1.0,
                       impeller_diameter_m=0.5, clearance_m=0.4, omega_rad_s=1.0, impeller="rushton",
                       baffle_count=4, baffle_width_m=0.1, baffle_thickness_m=2.5 / n, min_cells=12.0)
    g = lb.build_stirred_tank(spec)
    body = lb.RotatingBody(g["center"], np.array([0.0, 0.0, 0.05 / (0.25 * n)]), g["marker_pos"], g["marker_w"])
    return (n, n, n), g["solid"], body


@pytest.mark.parametrize("prec", ["f32", "f16"])
def test_runner_resume_is_bit_exact(tmp_path, prec):
    """The stirred-tank runner (runner.rs save_every / restore): torque
    series, populations, force field and the mixing scalar continue bit for
    bit. The body is registered before the restore, as the runner builds
    the solver and its impeller before restoring."""
    dims, solid, body = small_tank()
    kw = dict(lattice=27, collision="cm", storage=prec, nu=0.02, omega_shear=1.0 / 0.56, solid=solid)

    def build():
        g = lb.Solver(dims, **kw)
        g.set_body(0, body)
        return g

    def scalar(g):
        k = g.enable_scalar_distribution(0.01, q=7, name="tracer")
        z = np.arange(g.n) // (dims[0] * dims[1])
        g.set_scalar_concentration(k, np.where((solid == 0) & (z > dims[2] // 2), 1.0, 0.0))
        return k

    cont, part = build(), build()
    kc, kp = scalar(cont), scalar(part)
    a = cont.run_impeller(body, 30, scalar=kc)
    b1 = part.run_impeller(body, 13, scalar=kp)
    part.save(str(tmp_path))
    fresh = build()
    fresh.restore(str(tmp_path))
    b2 = fresh.run_impeller(body, 17, scalar=0)
    torque = np.concatenate([b1["torque_lu"], b2["torque_lu"]])
    assert np.array_equal(a["torque_lu"], torque)
    assert np.array_equal(a["cv"][13:], b2["cv"])
    assert_same_state(cont, fresh)
    assert np.array_equal(cont.force_field(), fresh.force_field())
    assert np.array_equal(cont.gather_scalar_concentration(kc), fresh.gather_scalar_concentration(0))
    m = ock.read(tmp_path, {"dims": dims, "lattice": 27, "collision": "cm", "nu": 0.02, "magic": lb.MAGIC_STD,
                            "omega_shear": 1.0 / 0.56, "periodic": (False,) * 3, "force": (0.0, 0.0, 0.0),
                            "dtype": "f32"}, solid)
    assert m["scalars"][0]["name"] == "tracer" and m["scalars"][0]["q"] == 7 and m["force_field"] is not None


def oracle_spec(kw, dtype):
    om = kw.get("omega_shear") or 1.0 / (3.0 * kw["nu"] + 0.5)
    return {"dims": kw["dims"], "lattice": kw["lattice"], "collision": kw["collision"], "nu": kw["nu"],
            "magic": lb.MAGIC_STD, "omega_shear": om, "periodic": (False,) * 3, "force": kw["force"],
            "dtype": dtype}


def oracle_for(kw, bits):
    return o.OracleSolver(kw["dims"], q=kw["lattice"], real_bits=bits, collision=kw["collision"], nu=kw["nu"],
                          omega_shear=1.0 / (3.0 * kw["nu"] + 0.5), solid=kw["solid"], wall_u=kw["wall_u"],
                          force=kw["force"])


@pytest.mark.parametrize("q,coll", [(19, "trt"), (27, "cm")])
def test_device_checkpoint_equals_oracle_checkpoint(tmp_path, q, coll):
    kw = tank_kw(q, coll, "f64")
    kw["force"] = (2e-6, 0.0, -1e-6)
    g = make(kw)
    c = oracle_for(kw, 64)
    g.run(23)
    c.step(23)
    g.save(str(tmp_path / "g"))
    spec = oracle_spec(kw, "f64")
    ock.save(c, tmp_path / "c", spec, kw["solid"], kw["wall_u"])
    mg = json.loads((tmp_path / "g" / "manifest.json").read_text())
    mc = json.loads((tmp_path / "c" / "manifest.json").read_text())
    for key in mg:
        if key != "ranks":
            assert mg[key] == mc[key], key
    rg, rc = mg["ranks"][0], mc["ranks"][0]
    for key in ("file", "origin", "core", "bytes", "mask_hash"):
        assert rg[key] == rc[key], key
    sg = ock.read(tmp_path / "g", spec, kw["solid"], kw["wall_u"])
    sc = ock.read(tmp_path / "c", spec, kw["solid"], kw["wall_u"])
    fl = kw["solid"] == 0
    assert np.abs(sg["f"][:, fl] - sc["f"][:, fl]).max() <= TOL["f64"] * np.abs(sc["f"]).max()
    assert np.abs(sg["moments"] - sc["moments"]).max() <= 1e-10
    assert not sg["ftmp"].any()


@pytest.mark.parametrize("prec", ["f64", "f32"])
def test_checkpoints_cross_between_oracle_and_device(tmp_path, prec):
    kw = tank_kw(19, "trt", prec)
    bits = 64 if prec == "f64" else 32
    spec = oracle_spec(kw, prec)
    fl = kw["solid"] == 0
    # oracle -> device
    c = oracle_for(kw, bits)
    c.step(15)
    ock.save(c, tmp_path / "c", spec, kw["solid"], kw["wall_u"], stash="solver")
    g = make(kw)
    g.restore(str(tmp_path / "c"))
    assert g.time == 15
    g.run(12)
    c.step(12)
    ug, uc = g.read_moments()[1][fl], c.moments()[1][fl]
    assert np.abs(ug - uc).max() <= 3 * TOL[prec] * np.abs(uc).max()
    # device -> oracle
    g.save(str(tmp_path / "g"))
    c2 = oracle_for(kw, bits)
    ock.restore(c2, tmp_path / "g", spec, kw["solid"], kw["wall_u"])
    g.run(12)
    c2.step(12)
    ug, uc = g.read_moments()[1][fl], c2.moments()[1][fl]
    assert np.abs(ug - uc).max() <= 3 * TOL[prec] * np.abs(uc).max()


def test_sixteen_bit_checkpoint_loads_into_f32(tmp_path):
    """16-bit storage writes dtype "f32" with exactly widened values: an f32
    solver restores the same logical populations."""
    kw16 = tank_kw(19, "trt", "f16")
    g = make(kw16)
    g.run(11)
    g.save(str(tmp_path))
    g32 = make(dict(kw16, storage="f32"))
    g32.restore(str(tmp_path))
    assert np.array_equal(g32.stage_out(), g.stage_out())


def test_refused_restore_leaves_the_solver_untouched(tmp_path):
    kw = tank_kw(19, "trt", "f32")
    a = make(kw)
    a.run(5)
    a.save(str(tmp_path / "a"))
    b = make(dict(kw, nu=kw["nu"] * 1.1))
    b.run(3)
    before = b.stage_out()
    with pytest.raises(lb.CheckpointError) as e:
        b.restore(str(tmp_path / "a"))
    assert e.value.code == "CKPT_SCENARIO_MISMATCH" and "scenario_hash differed" in e.value.message
    assert np.array_equal(b.stage_out(), before) and b.time == 3
    # a solver with more scalars than the checkpoint is refused before installing
    c = make(kw)
    c.enable_scalar_distribution(0.02, q=7)
    c.run(2)
    before = c.stage_out()
    with pytest.raises(lb.CheckpointError) as e:
        c.restore(str(tmp_path / "a"))
    assert e.value.code == "CKPT_SCENARIO_MISMATCH"
    assert np.array_equal(c.stage_out(), before) and c.time == 2
    with pytest.raises(lb.CheckpointError) as e:
        c.restore(str(tmp_path / "missing"))
    assert e.value.code == "CKPT_IO"


def test_qoi_state_and_time_round_trip(tmp_path):
    kw = tank_kw(19, "trt", "f32")
    g = make(kw)
    assert g.time == 0 and g.qoi_checkpoint_state is None
    g.run(4)
    g.qoi_checkpoint_state = '{"accumulators": []}'
    g.save(str(tmp_path))
    assert json.loads((tmp_path / "manifest.json").read_text())["reserved"]["stats"] is True
    h = lb.Solver.load(str(tmp_path), kw["dims"], lattice=19, collision="trt", storage="f32", nu=kw["nu"],
                       solid=kw["solid"], wall_u=kw["wall_u"])
    assert h.time == 4 and h.qoi_checkpoint_state == '{"accumulators": []}'
    with pytest.raises(lb.SpecError):
        h.qoi_checkpoint_state = "[1, 2]"


@pytest.mark.parametrize("prec", ["f64", "f32", "f16"])
def test_device_writer_equals_host_writer(tmp_path, prec):
    """The device-packed checkpoint (padded planes packed on the device,
    pinned copy, overlapped hash) is byte-identical to the host writer of
    the same state gathered through the ABI, which the CPU tests pin to the
    oracle's writer."""
    dims, solid, body = small_tank()
    om = 1.0 / 0.56
    g = lb.Solver(dims, lattice=27, collision="cm", storage=prec, nu=0.02, omega_shear=om, solid=solid)
    g.run_impeller(body, 5)
    g.save(str(tmp_path / "d"))
    spec = {"dims": dims, "lattice": 27, "collision": "cm", "nu": 0.02, "magic": lb.MAGIC_STD, "omega_shear": om,
            "periodic": (False,) * 3, "force": (0.0, 0.0, 0.0), "dtype": "f64" if prec == "f64" else "f32"}
    state = {"step": g.time, "f": g.stage_out(), "moments": np.stack(g.read_moments()),
             "force_field": g.force_field(), "scalars": [], "qoi": None}
    lb.checkpoint_write_host(str(tmp_path / "h"), spec, state, solid=solid)
    for fn in ("manifest.json", ock.RANK_FILE):
        assert (tmp_path / "d" / fn).read_bytes() == (tmp_path / "h" / fn).read_bytes(), fn
