"""CPU-only checks of the C-ABI library: it loads, exports every entry point
include/lbmb.h declares, and its host-side set-up code (wall rims, stirred
tank voxel flags, impeller markers) is bit-identical to the oracle."""
import ctypes as C
import math
import os
import re
import subprocess

import numpy as np
import pytest

import lbmflow_b200 as lb

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
TAU = 2.0 * math.pi


def header_functions():
    text = open(os.path.join(ROOT, "include", "lbmb.h")).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(lbmb_[a-z0-9_]+)\s*\(", text)))


def test_library_exports_every_declared_symbol():
    lib = lb.lib()
    declared = header_functions()
    assert len(declared) >= 20
    out = subprocess.run(["nm", "-D", "--defined-only", lb.LIB_PATH], capture_output=True, text=True).stdout
    exported = set(re.findall(r" T (lbmb_\w+)", out))
    missing = [f for f in declared if f not in exported]
    assert not missing, missing
    for f in declared:
        assert hasattr(lib, f)
    assert set(lb.EXPORTS) == set(declared)


def test_version_and_error_text():
    assert b"sm_100a" in lb.lib().lbmb_version()
    # A null config is rejected through the status code, not a crash.
    h = C.c_void_p()
    rc = lb.lib().lbmb_create(None, None, None, C.byref(h))
    assert rc == lb.ERR_INVALID
    assert b"null" in lb.lib().lbmb_last_error()


def test_wall_rims_bit_exact(oracle):
    dims = (9, 7, 6)
    u = np.zeros((6, 3))
    u[5] = [0.05, 0.0, 0.0]
    u[2] = [0.0, 0.0, 0.02]
    is_wall = [True, True, True, True, True, True]
    s1, w1 = lb.build_wall_rims(dims, is_wall, u.ravel())
    s2, w2 = oracle.wall_rims(dims, is_wall, u.ravel())
    assert np.array_equal(s1, s2)
    assert np.array_equal(w1.view(np.uint64), w2.view(np.uint64))


@pytest.mark.parametrize("n,kind,blades,baffles", [(64, 0, 6, True), (96, 0, 6, False), (64, 1, 4, True),
                                                   (80, 1, 4, False)])
def test_stirred_tank_voxels_and_markers_bit_exact(oracle, n, kind, blades, baffles):
    # Voxel flags, baffle mask, wall-velocity stamp and impeller marker
    # positions/weights must equal the reference generator bit for bit
    # (geometry.rs:207-345, 657-916).
    dx = 1.0 / n
    bw, bt = (0.08, 0.025) if baffles else (0.0, 0.0)
    omega = 120.0 * TAU / 60.0
    spec = lb.TankSpec(dims=(n, n, n), dx_m=dx, vessel_diameter_m=1.0, liquid_height_m=1.0,
                       impeller_diameter_m=0.5, clearance_m=0.35, omega_rad_s=omega, blade_count=blades,
                       impeller=["rushton", "pitched"][kind], baffle_count=4 if baffles else 0,
                       baffle_width_m=bw, baffle_thickness_m=bt)
    g = lb.build_stirred_tank(spec)
    o = oracle.build_tank((n, n, n), dx, 1.0, 1.0, 0.5, 0.35, blades, omega, baffle_w=bw, baffle_t=bt, kind=kind)
    assert np.array_equal(g["solid"], o["solid"])
    assert np.array_equal(g["baffle"], o["baffle"])
    assert np.array_equal(g["wall_velocity"].view(np.uint64), o["wall_velocity"].view(np.uint64))
    assert g["marker_pos"].shape == o["marker_pos"].shape
    assert np.array_equal(g["marker_pos"].view(np.uint64), o["marker_pos"].view(np.uint64))
    assert np.array_equal(g["marker_w"].view(np.uint64), o["marker_w"].view(np.uint64))
    assert np.array_equal(g["center"], o["center"])
    assert np.array_equal(g["omega"], o["omega"])


def test_flat_blade_turbine_marker_set():
    # The flat-blade turbine of the tank configuration: T = 128 cells,
    # D = T/3 at clearance T/3, 0.7-cell spacing -> about 6k markers inside
    # the liquid, weights summing to the sampled surface area.
    T = 128
    dx = 1.0 / T
    spec = lb.TankSpec(dims=(128, 128, 160), dx_m=dx, vessel_diameter_m=1.0, liquid_height_m=160 * dx,
                       impeller_diameter_m=1.0 / 3.0, clearance_m=1.0 / 3.0, omega_rad_s=1.0,
                       impeller="flat_blade", marker_spacing_cells=0.7, baffle_count=4,
                       baffle_width_m=0.1, baffle_thickness_m=2.6 * dx)
    g = lb.build_stirred_tank(spec)
    m = g["marker_pos"]
    assert 5000 < len(m) < 7500
    D = T / 3.0
    r = np.hypot(m[:, 0] - 64.0, m[:, 1] - 64.0)
    assert r.max() <= D / 2 + 1.0
    assert abs(g["marker_w"].sum() - 2 * (math.pi * (0.375 * D) ** 2 + 6 * 0.25 * D * 0.2 * D)) < 1e-6 * len(m)
    # markers must sit in fluid cells of the tank
    idx = (np.floor(m[:, 2]).astype(int) * 128 + np.floor(m[:, 1]).astype(int)) * 128 + np.floor(m[:, 0]).astype(int)
    assert g["solid"][idx].sum() == 0


def test_tank_validation_errors():
    base = dict(dims=(96, 96, 96), dx_m=1 / 96, vessel_diameter_m=1.0, liquid_height_m=1.0,
                impeller_diameter_m=0.4, clearance_m=0.9, omega_rad_s=1.0)
    with pytest.raises(lb.SpecError):  # geometry.rs:1032-1045 impeller outside liquid
        lb.build_stirred_tank(lb.TankSpec(**base))
    with pytest.raises(lb.SpecError):  # geometry.rs:1055-1063 under-resolved
        lb.build_stirred_tank(lb.TankSpec(**{**base, "dims": (48, 48, 48), "dx_m": 1 / 48,
                                              "impeller_diameter_m": 0.2, "clearance_m": 0.35}))
    with pytest.raises(lb.UnsupportedError):
        lb.build_stirred_tank(lb.TankSpec(**{**base, "clearance_m": 0.35, "baffle_count": 3,
                                              "baffle_width_m": 0.08, "baffle_thickness_m": 0.02}))
