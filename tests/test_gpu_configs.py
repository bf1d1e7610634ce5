"""GPU parity on the benchmark configurations at their stated sizes.

1. The plain-method cavity exactly as stated: 64^3, D3Q19 TRT (magic 3/16),
   Re = 100, lid 0.05 on ZPos moving +x, every other wall half-way
   bounce-back, quiescent start, 1000 steps, nu = U (N - 2) / Re
   (crates/lbm-core/tests/t15_5_cavity3d.rs:148-182). f64 against the f64
   oracle (populations within 1e-11 of the largest, the reference's CPU
   tolerance, crates/lbm-core/tests/backend_simd_equiv.rs:1-20); f32 under
   the rule that the GPU is as close to the f64 oracle as the reference's
   own f32 path is (3x its distance); both centreline profiles (u_x(z) at
   x = y = N/2, u_z(x) at y = z = N/2) likewise.
2. The stirred-tank headline configuration, 128 x 128 x 160, D3Q27 central
   moment, flat-blade turbine (6 blades, D = T/3, clearance T/3, markers at
   0.7 cells), 4 baffles, free-slip surface, Smagorinsky 0.1: a 100-step
   prefix of the runner loop from rest in f64 and f32 against the oracle,
   per-step torque and final rho and u (t14_backend_equiv.rs:1-8 allows
   1e-5 relative on fields and 1e-4 on diagnostics between CPU and GPU).
3. 16-bit shifted storage (binary16, bfloat16) against the oracle's 16-bit
   storage mode (every written population rounded to the format, nearest
   even, in deviation form): after one step from a shared state every
   population is within one unit in the last place of the format, and only
   a few percent differ at all (the fp32 arithmetic of the two differs by
   rounding, which moves a value across a rounding boundary now and then);
   over the cavity and the tank prefix the GPU's 16-bit run is as close to
   the f64 solution as the oracle's 16-bit run is (within 3x, the rule of
   the f32 comparisons). Storing f instead of f - w, or truncating, would
   miss both bounds by orders of magnitude.
"""
import numpy as np
import pytest

import lbmflow_b200 as lb
from cases import cavity

pytestmark = pytest.mark.gpu

N_CAV = 64
CAV_STEPS = 1000


def _centrelines(ux, uz, n):
    """u_x(z) at x = y = n/2 and u_z(x) at y = z = n/2 (cell centres)."""
    c = n // 2
    ux = ux.reshape(n, n, n)
    uz = uz.reshape(n, n, n)
    return ux[:, c, c].copy(), uz[c, c, :].copy()


@pytest.fixture(scope="module")
def cav64():
    from oracle import oracle as o
    dims, solid, wall_u, nu = cavity(N_CAV, u_lid=0.05, re=100.0)
    out = {"dims": dims, "solid": solid, "wall_u": wall_u, "nu": nu}
    for bits in (64, 32):
        c = o.OracleSolver(dims, q=19, real_bits=bits, nu=nu, solid=solid, wall_u=wall_u)
        c.step(CAV_STEPS)
        out[bits] = {"f": c.stage_out(), "m": c.moments()}
    return out


def test_cavity64_config_parameters(cav64):
    assert cav64["dims"] == (64, 64, 64)
    assert abs(cav64["nu"] - 0.031) < 1e-15  # 0.05 * 62 / 100
    assert abs(3.0 * cav64["nu"] + 0.5 - 0.593) < 1e-12


def test_cavity64_f64_matches_oracle(cav64):
    d = cav64
    g = lb.Solver(d["dims"], lattice=19, collision="trt", storage="f64", nu=d["nu"], solid=d["solid"],
                  wall_u=d["wall_u"])
    g.run(CAV_STEPS)
    fl = d["solid"] == 0
    fg, fc = g.stage_out()[:, fl], d[64]["f"][:, fl]
    assert np.abs(fg - fc).max() <= 1e-11 * np.abs(fc).max()
    mg, mc = g.read_moments(), d[64]["m"]
    for k in range(4):
        assert np.abs(mg[k][fl] - mc[k][fl]).max() <= 1e-10 * max(np.abs(mc[k][fl]).max(), 1e-30)
    pg, pc = _centrelines(mg[1], mg[3], N_CAV), _centrelines(mc[1], mc[3], N_CAV)
    for a, b in zip(pg, pc):
        assert np.abs(a - b).max() <= 1e-11 * np.abs(b).max()
    # the lid drives the flow: u_x near the lid is a fair fraction of U
    assert pc[0][N_CAV - 2] > 0.2 * 0.05
    # mass is conserved to round-off over 1000 steps
    assert abs(g.total_mass_f64() - float(fl.sum())) < 1e-9


def test_cavity64_f32_matches_oracle(cav64):
    d = cav64
    g = lb.Solver(d["dims"], lattice=19, collision="trt", storage="f32", nu=d["nu"], solid=d["solid"],
                  wall_u=d["wall_u"])
    g.run(CAV_STEPS)
    fl = d["solid"] == 0
    ex, ref = d[64], d[32]
    e_gpu = np.abs(g.stage_out()[:, fl] - ex["f"][:, fl]).max()
    e_ref = np.abs(ref["f"][:, fl] - ex["f"][:, fl]).max()
    assert e_gpu <= 3.0 * e_ref + 1e-9, (e_gpu, e_ref)
    mg = g.read_moments()
    pg = _centrelines(mg[1], mg[3], N_CAV)
    px = _centrelines(ex["m"][1], ex["m"][3], N_CAV)
    pr = _centrelines(ref["m"][1], ref["m"][3], N_CAV)
    for a, b, r in zip(pg, px, pr):
        assert np.abs(a - b).max() <= 3.0 * np.abs(r - b).max() + 1e-9
        assert np.abs(a - b).max() <= 1e-5 * np.abs(b).max()


ULP16 = {"f16": 10, "bf16": 7}  # explicit mantissa bits


def _ulp(v, prec):
    """Spacing of the 16-bit format at |v| (normal range)."""
    e = np.floor(np.log2(np.maximum(np.abs(v), 2.0 ** -14)))
    return 2.0 ** (e - ULP16[prec])


@pytest.mark.parametrize("prec", ["f16", "bf16"])
@pytest.mark.parametrize("q,coll", [(19, "trt"), (27, "cm")])
def test_16bit_one_step_within_one_ulp(prec, q, coll):
    from oracle import oracle as o
    dims, solid, wall_u, nu = cavity(24, re=50.0)
    g = lb.Solver(dims, lattice=q, collision=coll, storage=prec, nu=nu, solid=solid, wall_u=wall_u)
    c = o.OracleSolver(dims, q=q, real_bits=32, collision=coll, nu=nu, omega_shear=1.0 / (3 * nu + 0.5),
                       solid=solid, wall_u=wall_u, store16=prec)
    g.run(40)  # a developed state, staged into both
    f0 = g.stage_out()
    c.stage_in(f0)
    assert np.array_equal(c.stage_out(), f0)  # values already in the format stage exactly
    g.run(1)
    c.step(1)
    fl = solid == 0
    fg, fc = g.stage_out()[:, fl], c.stage_out()[:, fl]
    assert np.all(np.abs(fg - fc) <= _ulp(fc, prec) * 1.0001)
    assert np.mean(fg != fc) < 0.05  # rounding flips are rare


@pytest.mark.parametrize("prec", ["f16", "bf16"])
def test_16bit_staging_uses_reference_codec(prec):
    # lbmb_stage_in of f16 storage encodes with the reference's host codec
    # (gpu/backend.rs:160-186: ties away from zero); bf16 rounds to nearest
    # even.
    from oracle import oracle as o
    dims, solid, wall_u, nu = cavity(10)
    g = lb.Solver(dims, lattice=19, storage=prec, nu=nu, solid=solid, wall_u=wall_u)
    rng = np.random.default_rng(11)
    f = rng.normal(0, 3e-2, size=(19, g.n)).astype(np.float32)
    # exact ties of both formats
    f[1, :200] = (1.0 + 2.0 ** -11) * 2.0 ** rng.integers(-8, 0, 200)
    f[2, :200] = (1.0 + 2.0 ** -8) * 2.0 ** rng.integers(-8, 0, 200)
    g.stage_in(f.astype(np.float64))
    got = g.stage_out()
    # solid cells return their raw slots, fluid cells their logical ones: at
    # parity 0 both are the staged values
    want = o.codec16("ref_f16" if prec == "f16" else "bf16", f).reshape(19, g.n)
    assert np.array_equal(got, want.astype(np.float64))


@pytest.mark.parametrize("prec", ["f16", "bf16"])
def test_cavity64_16bit_tracks_oracle_16bit(prec, cav64):
    from oracle import oracle as o
    d = cav64
    steps = 300
    g = lb.Solver(d["dims"], lattice=19, storage=prec, nu=d["nu"], solid=d["solid"], wall_u=d["wall_u"])
    c16 = o.OracleSolver(d["dims"], q=19, real_bits=32, nu=d["nu"], solid=d["solid"], wall_u=d["wall_u"],
                         store16=prec)
    c64 = o.OracleSolver(d["dims"], q=19, real_bits=64, nu=d["nu"], solid=d["solid"], wall_u=d["wall_u"])
    g.run(steps)
    c16.step(steps)
    c64.step(steps)
    fl = d["solid"] == 0
    m_g, m_16, m_64 = g.read_moments(), c16.moments(), c64.moments()
    for k in range(4):
        e_gpu = np.linalg.norm(m_g[k][fl] - m_64[k][fl])
        e_ref = np.linalg.norm(m_16[k][fl] - m_64[k][fl])
        assert e_ref > 0.0
        assert e_gpu <= 3.0 * e_ref, (k, e_gpu, e_ref)


# ---- the headline tank, 100-step prefix --------------------------------------

T_TANK = 128
TANK_STEPS = 100


def _tank():
    T = T_TANK
    nz = int(round(1.25 * T))
    dx = 1.0 / T
    spec = lb.TankSpec(dims=(T, T, nz), dx_m=dx, vessel_diameter_m=1.0, liquid_height_m=nz * dx,
                       impeller_diameter_m=1.0 / 3.0, clearance_m=1.0 / 3.0, omega_rad_s=1.0, impeller="flat_blade",
                       marker_spacing_cells=0.7, baffle_count=4, baffle_width_m=0.1, baffle_thickness_m=2.6 * dx)
    geo = lb.build_stirred_tank(spec)
    D = T / 3.0
    omega = 0.05 / (0.5 * D)
    nu = (omega / (2.0 * np.pi)) * D * D / 2000.0
    body = lb.RotatingBody(geo["center"], [0.0, 0.0, omega], geo["marker_pos"], geo["marker_w"])
    return (T, T, nz), geo["solid"], body, nu


TANK_STEPS_16 = 50


def _oracle_tank(dims, solid, body, nu, bits, store16=None, steps=TANK_STEPS):
    from oracle import oracle as o
    c = o.OracleSolver(dims, q=27, real_bits=bits, collision="cm", nu=nu, omega_shear=1.0 / (3.0 * nu + 0.5),
                       solid=solid, smagorinsky_cs=0.1, free_slip_top=True, store16=store16)
    r = c.run_tank(body.positions, body.weights, body.center, body.omega, steps)
    return {"torque": r["torque_lu"], "force": r["fluid_force"], "m": c.moments()}


@pytest.fixture(scope="module")
def tank_ref():
    dims, solid, body, nu = _tank()
    return {"case": (dims, solid, body, nu), 64: _oracle_tank(dims, solid, body, nu, 64),
            32: _oracle_tank(dims, solid, body, nu, 32)}


def _gpu_tank(case, storage, steps=TANK_STEPS):
    dims, solid, body, nu = case
    g = lb.Solver(dims, lattice=27, collision="cm", storage=storage, nu=nu, omega_shear=1.0 / (3.0 * nu + 0.5),
                  solid=solid, smagorinsky_cs=0.1, free_slip_top=True)
    r = g.run_impeller(body, steps)
    return g, r


def test_tank_config_markers(tank_ref):
    dims, solid, body, nu = tank_ref["case"]
    assert dims == (128, 128, 160)
    assert 5000 <= len(body.weights) <= 7000  # "~6k" markers
    D = 128 / 3.0
    omega = body.omega[2]
    assert abs(omega * D / 2.0 - 0.05) < 1e-15  # tip speed 0.05
    assert abs((omega / (2.0 * np.pi)) * D * D / nu - 2000.0) < 1e-9  # impeller Re = 2000


def test_tank_prefix_f64_matches_oracle(tank_ref):
    g, r = _gpu_tank(tank_ref["case"], "f64")
    ref = tank_ref[64]
    tq = ref["torque"]
    assert np.abs(r["torque_lu"] - tq).max() <= 1e-9 * np.abs(tq).max()
    assert np.abs(r["fluid_force"] - ref["force"]).max() <= 1e-9 * np.abs(ref["force"]).max()
    fl = tank_ref["case"][1] == 0
    mg = g.read_moments()
    for k in range(4):
        b = ref["m"][k][fl]
        assert np.abs(mg[k][fl] - b).max() <= 1e-10 * max(np.abs(b).max(), 1e-30), k


def test_tank_prefix_f32_matches_oracle(tank_ref):
    g, r = _gpu_tank(tank_ref["case"], "f32")
    ex, ref = tank_ref[64], tank_ref[32]
    e_gpu = np.abs(r["torque_lu"] - ex["torque"]).max()
    e_ref = np.abs(ref["torque"] - ex["torque"]).max()
    assert e_gpu <= 3.0 * e_ref + 1e-12 * np.abs(ex["torque"]).max(), (e_gpu, e_ref)
    assert e_gpu <= 1e-4 * np.abs(ex["torque"]).max()
    fl = tank_ref["case"][1] == 0
    mg = g.read_moments()
    for k in range(4):
        b = ex["m"][k][fl]
        eg = np.abs(mg[k][fl] - b).max()
        er = np.abs(ref["m"][k][fl] - b).max()
        assert eg <= 3.0 * er + 1e-9, (k, eg, er)


@pytest.mark.parametrize("prec", ["f16", "bf16"])
def test_tank_prefix_16bit_tracks_oracle_16bit(prec, tank_ref):
    # the first 50 steps: both 16-bit runs' torque series against the f64
    # oracle's over the same steps
    dims, solid, body, nu = tank_ref["case"]
    n = TANK_STEPS_16
    g, r = _gpu_tank(tank_ref["case"], prec, steps=n)
    o16 = _oracle_tank(dims, solid, body, nu, 32, store16=prec, steps=n)
    tq64 = tank_ref[64]["torque"][:n]
    e_gpu = np.linalg.norm(r["torque_lu"] - tq64)
    e_ref = np.linalg.norm(o16["torque"] - tq64)
    assert e_ref > 0.0
    assert e_gpu <= 3.0 * e_ref, (e_gpu, e_ref)
