"""ctypes view of the CPU oracle (test infrastructure only).

The oracle is the C++ restatement of the reference CPU path in
``lbm_oracle.hpp``. Only ``tests/``, ``__graft_entry__.smoke()`` and
``bench.py``'s CPU-baseline / reference legs may import this module, and only
as the checker or the timed CPU baseline.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_build", "liblbmb_oracle.so")

_dp = C.POINTER(C.c_double)
_ip = C.POINTER(C.c_int)
_u8p = C.POINTER(C.c_uint8)

COLLISION = {"bgk": 0, "trt": 1, "cm": 2, "central_moment": 2}
MAGIC_STD = 3.0 / 16.0


def build() -> str:
    """Compile the oracle shared library with its Makefile (gcc, OpenMP)."""
    subprocess.run(["make", "-s", "-C", HERE], check=True)
    return LIB_PATH


_lib = None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            build()
        L = C.CDLL(LIB_PATH)
        L.lbmo_create.restype = C.c_void_p
        L.lbmo_create.argtypes = [C.c_int, C.c_int, _ip, _ip, C.c_int, C.c_double, C.c_double,
                                  C.c_double, _dp, _u8p, _dp, C.c_char_p, C.c_int]
        L.lbmo_destroy.argtypes = [C.c_void_p]
        L.lbmo_step.argtypes = [C.c_void_p, C.c_int]
        L.lbmo_set_smagorinsky.argtypes = [C.c_void_p, C.c_double]
        L.lbmo_set_free_slip_top.argtypes = [C.c_void_p, C.c_int]
        for name in ("lbmo_stage_in", "lbmo_stage_out", "lbmo_get_force_field"):
            getattr(L, name).argtypes = [C.c_void_p, _dp]
        L.lbmo_init_with.argtypes = [C.c_void_p, _dp, _dp]
        L.lbmo_read_moments.argtypes = [C.c_void_p, _dp, _dp, _dp, _dp]
        L.lbmo_reduce.restype = C.c_double
        L.lbmo_reduce.argtypes = [C.c_void_p, C.c_int, C.c_int]
        L.lbmo_clear_force_field.argtypes = [C.c_void_p]
        L.lbmo_ibm_apply.restype = C.c_int
        L.lbmo_ibm_apply.argtypes = [C.c_void_p, _dp, _dp, C.c_long, _dp, _dp, C.c_int, C.c_double,
                                     C.c_int, C.c_double, _dp, C.c_char_p, C.c_int]
        L.lbmo_ibm_direct_forcing.restype = C.c_int
        L.lbmo_ibm_direct_forcing.argtypes = [_ip, C.c_int, _u8p, _dp, _dp, _dp, _dp, C.c_long, _dp,
                                              _dp, C.c_int, C.c_double, C.c_int, C.c_double, _dp,
                                              _dp, C.c_char_p, C.c_int]
        L.lbmo_marker_stencil.restype = C.c_int
        L.lbmo_marker_stencil.argtypes = [_dp, _ip, C.c_int, C.c_int, _dp]
        L.lbmo_scalar_enable.restype = C.c_int
        L.lbmo_scalar_enable.argtypes = [C.c_void_p, C.c_int, C.c_double]
        L.lbmo_scalar_set.argtypes = [C.c_void_p, C.c_int, _dp]
        L.lbmo_scalar_get.argtypes = [C.c_void_p, C.c_int, _dp]
        L.lbmo_wall_rims.argtypes = [C.c_int, _ip, _ip, _dp, _u8p, _dp]
        L.lbmo_build_tank.restype = C.c_long
        L.lbmo_build_tank.argtypes = [_ip, C.c_double, C.c_double, C.c_double, C.c_double,
                                      C.c_double, C.c_int, C.c_double, C.c_double, C.c_int,
                                      C.c_double, _u8p, _u8p, _dp, _dp, _dp, C.c_long, _dp, _dp,
                                      C.c_char_p, C.c_int]
        L.lbmo_build_tank2.restype = C.c_long
        L.lbmo_build_tank2.argtypes = [_ip, C.c_double, C.c_double, C.c_double, C.c_double, C.c_double, C.c_int,
                                       C.c_double, C.c_double, C.c_int, C.c_double, C.c_double, _u8p, _u8p, _dp,
                                       _dp, _dp, C.c_long, _dp, _dp, C.c_char_p, C.c_int]
        L.lbmo_set_store16.restype = C.c_int
        L.lbmo_set_store16.argtypes = [C.c_void_p, C.c_int]
        _fp = C.POINTER(C.c_float)
        L.lbmo_codec16.argtypes = [C.c_int, _fp, _fp, C.c_long]
        L.lbmo_f16_bits.argtypes = [_fp, C.POINTER(C.c_uint16), C.c_long]
        L.lbmo_runner_power.restype = C.c_long
        L.lbmo_runner_power.argtypes = [_dp, C.c_long, C.c_long, C.c_long] + [C.c_double] * 6 + [_dp]
        L.lbmo_unit_report.restype = C.c_int
        L.lbmo_unit_report.argtypes = [_dp, _ip, C.c_double, _dp, C.POINTER(C.c_uint)]
        L.lbmo_top_hat_pulse.argtypes = [_ip, _u8p, C.c_double, _dp, C.c_double, C.c_double, _dp]
        L.lbmo_power_qois.restype = C.c_int
        L.lbmo_power_qois.argtypes = [C.c_double] * 5 + [_dp]
        L.lbmo_scalar_cv.restype = C.c_double
        L.lbmo_scalar_cv.argtypes = [_dp, _u8p, C.c_long]
        L.lbmo_mixing_time.restype = C.c_int
        L.lbmo_mixing_time.argtypes = [_dp, _dp, C.c_long, _dp]
        L.lbmo_run_tank.restype = C.c_long
        L.lbmo_run_tank.argtypes = [C.c_void_p, _dp, _dp, C.c_long, _dp, _dp, C.c_int, C.c_double,
                                    C.c_int, C.c_double, C.c_long, C.c_long, C.c_int, _dp, _dp,
                                    _dp, _dp]
        L.lbmo_gather_strain_rate.argtypes = [C.c_void_p, _dp, _dp]
        L.lbmo_set_omega_field.argtypes = [C.c_void_p, _dp]
        L.lbmo_gather_velocity_gradient.argtypes = [C.c_void_p, _dp]
        L.lbmo_wale_update.argtypes = [C.c_void_p, C.c_double, _dp, _dp]
        L.lbmo_compute_stress_field.argtypes = [_ip, _dp, _dp, _dp, _u8p, C.c_double, _dp, _dp, _dp, _dp, _dp, _dp]
        L.lbmo_percentile_summary.restype = C.c_int
        L.lbmo_percentile_summary.argtypes = [_dp, C.c_long, C.c_int, C.c_double, _dp]
        L.lbmo_wall_shear_proxy.restype = C.c_long
        L.lbmo_wall_shear_proxy.argtypes = [_ip, _dp, _dp, _dp, _u8p, _dp, C.c_double, C.c_double, C.c_double,
                                            C.c_long, C.POINTER(C.c_int64), _dp, _dp, _dp, _dp]
        L.lbmo_interfacial_flux.restype = C.c_int
        L.lbmo_interfacial_flux.argtypes = [_dp, _dp, _dp, _dp, C.c_long, C.c_double, C.c_double, _dp, _dp]
        L.lbmo_oxygen_uptake.restype = C.c_int
        L.lbmo_oxygen_uptake.argtypes = [_dp, _dp, C.c_long, C.c_double, C.c_int, _dp, _dp, _dp, _dp]
        L.lbmo_henry_equilibrium.restype = C.c_double
        L.lbmo_henry_equilibrium.argtypes = [C.c_double, C.c_double]
        L.lbmo_state_get.argtypes = [C.c_void_p, _dp, _dp, _dp, _ip, _dp, C.POINTER(C.c_uint64)]
        L.lbmo_state_set.argtypes = [C.c_void_p, _dp, _dp, _dp, C.c_int, _dp, C.c_uint64]
        L.lbmo_scalar_count.restype = C.c_int
        L.lbmo_scalar_count.argtypes = [C.c_void_p]
        L.lbmo_scalar_raw_get.argtypes = [C.c_void_p, C.c_int, _ip, _dp, _dp, _dp, _dp]
        L.lbmo_scalar_raw_set.argtypes = [C.c_void_p, C.c_int, C.c_double, _dp, _dp, _dp]
        L.lbmo_interfacial_area_density.restype = C.c_double
        L.lbmo_interfacial_area_density.argtypes = [C.c_double, _dp, C.c_double]
        _lib = L
    return _lib


def _d(a):
    return a.ctypes.data_as(_dp) if a is not None else None


def _as_d(a, n=None):
    a = np.ascontiguousarray(a, dtype=np.float64)
    if n is not None:
        assert a.size == n, (a.size, n)
    return a


DIAG_FIELDS = ("iterations", "slip_max", "slip_rms", "slip_max_rel", "slip_rms_rel", "torque",
               "fluid_force", "marker_force", "momentum_error_rel")


def diag_dict(v) -> dict:
    return {"iterations": int(v[0]), "slip_max": v[1], "slip_rms": v[2], "slip_max_rel": v[3],
            "slip_rms_rel": v[4], "torque": np.array(v[5:8]), "fluid_force": np.array(v[8:11]),
            "marker_force": np.array(v[11:14]), "momentum_error_rel": v[14]}


class OracleSolver:
    """Single-part CpuScalar solver (lattice 19|27, real 32|64)."""

    def __init__(self, dims, q=19, real_bits=64, collision="trt", nu=1.0 / 6.0, magic=MAGIC_STD,
                 omega_shear=0.0, periodic=(False, False, False), force=(0.0, 0.0, 0.0),
                 solid=None, wall_u=None, smagorinsky_cs=0.0, free_slip_top=False, store16=None):
        L = lib()
        self.dims = tuple(int(d) for d in dims)
        self.n = self.dims[0] * self.dims[1] * self.dims[2]
        self.q = q
        self.real_bits = real_bits
        dims_a = (C.c_int * 3)(*self.dims)
        per_a = (C.c_int * 3)(*[int(bool(p)) for p in periodic])
        force_a = np.asarray(force, dtype=np.float64)
        self._solid = None if solid is None else np.ascontiguousarray(solid, dtype=np.uint8).ravel()
        self._wall = None if wall_u is None else _as_d(wall_u).ravel()
        err = C.create_string_buffer(256)
        self.h = L.lbmo_create(q, real_bits, dims_a, per_a, COLLISION[collision], magic,
                               omega_shear, nu, _d(force_a),
                               None if self._solid is None else self._solid.ctypes.data_as(_u8p),
                               _d(self._wall), err, 256)
        if not self.h:
            raise ValueError(err.value.decode())
        if smagorinsky_cs:
            L.lbmo_set_smagorinsky(self.h, float(smagorinsky_cs))
        if free_slip_top:
            L.lbmo_set_free_slip_top(self.h, 1)
        if store16:
            # 16-bit population storage (fp32 arithmetic): "f16" or "bf16"
            if L.lbmo_set_store16(self.h, {"f16": 1, "bf16": 2}[store16]) != 0:
                raise ValueError("16-bit storage needs real_bits=32")

    def __del__(self):
        if getattr(self, "h", None):
            lib().lbmo_destroy(self.h)
            self.h = None

    def step(self, n=1):
        lib().lbmo_step(self.h, n)

    def stage_in(self, f):
        f = _as_d(f, self.q * self.n)
        lib().lbmo_stage_in(self.h, _d(f))

    def stage_out(self):
        f = np.zeros(self.q * self.n)
        lib().lbmo_stage_out(self.h, _d(f))
        return f.reshape(self.q, self.n)

    def init_with(self, rho, u):
        rho = _as_d(rho, self.n)
        u = _as_d(u, 3 * self.n)
        lib().lbmo_init_with(self.h, _d(rho), _d(u))

    def moments(self):
        out = [np.zeros(self.n) for _ in range(4)]
        lib().lbmo_read_moments(self.h, *[_d(a) for a in out])
        return out

    def set_omega_field(self, omega):
        """Solver::set_omega_field (None clears)."""
        lib().lbmo_set_omega_field(self.h, None if omega is None else _d(_as_d(omega, self.n)))

    def velocity_gradient(self):
        """Solver::gather_velocity_gradient: n x 3 x 3, g[i][j] = du_i/dx_j."""
        g = np.zeros(9 * self.n)
        lib().lbmo_gather_velocity_gradient(self.h, _d(g))
        return g.reshape(self.n, 3, 3)

    def wale_update(self, tau_eff_max=None):
        """WaleLes::update (Cw 0.325): nu_t per cell and diagnostics; the
        omega+ field is installed for the next collision."""
        nu_t, diag = np.zeros(self.n), np.zeros(5)
        lib().lbmo_wale_update(self.h, float("nan") if tau_eff_max is None else float(tau_eff_max), _d(nu_t),
                               _d(diag))
        return nu_t, {"clipped_cells": int(diag[0]), "clipped_fraction": diag[1],
                      "max_nu_t_before_clipping": diag[2],
                      "tau_eff_max": None if np.isnan(diag[3]) else diag[3],
                      "nu_t_max": None if np.isnan(diag[4]) else diag[4]}

    def strain_rate(self):
        """Native strain rate (n x 6: xx yy zz xy xz yz) and shear rate
        gamma_dot = sqrt(2 S:S) per cell (solver.rs:5393-5599)."""
        s6, g = np.zeros(6 * self.n), np.zeros(self.n)
        lib().lbmo_gather_strain_rate(self.h, _d(s6), _d(g))
        return s6.reshape(self.n, 6), g

    def reduce(self, kind, axis=0):
        return lib().lbmo_reduce(self.h, kind, axis)

    def total_mass(self):
        return self.reduce(0) + self.reduce(1)

    def clear_force_field(self):
        lib().lbmo_clear_force_field(self.h)

    def force_field(self):
        out = np.zeros(3 * self.n)
        lib().lbmo_get_force_field(self.h, _d(out))
        return out.reshape(self.n, 3)

    def ibm_apply(self, pos, w, center, omega, max_iterations=3, slip_tolerance=1e-2,
                  kernel_radius=1, relaxation=1.0):
        pos = _as_d(pos).ravel()
        w = _as_d(w).ravel()
        center = _as_d(center)
        omega = _as_d(omega)
        diag = np.zeros(15)
        err = C.create_string_buffer(256)
        rc = lib().lbmo_ibm_apply(self.h, _d(pos), _d(w), w.size, _d(center), _d(omega),
                                  max_iterations, slip_tolerance, kernel_radius, relaxation,
                                  _d(diag), err, 256)
        if rc != 0:
            raise ValueError(err.value.decode())
        return diag_dict(diag)

    def scalar_enable(self, diffusivity, q=None):
        k = lib().lbmo_scalar_enable(self.h, self.q if q is None else q, diffusivity)
        if k < 0:
            raise ValueError("scalar enable rejected")
        return k

    def scalar_set(self, k, values):
        v = _as_d(values, self.n)
        lib().lbmo_scalar_set(self.h, k, _d(v))

    def scalar_get(self, k):
        out = np.zeros(self.n)
        lib().lbmo_scalar_get(self.h, k, _d(out))
        return out

    def state(self):
        """Raw state: f and ftmp (Q x n, deviation form), moments (4 x n),
        force field (n x 3 or None), time, and per scalar its lattice,
        diffusivity, h and htmp (q x n) and concentration."""
        f, ft, mo, ff = (np.zeros(self.q * self.n), np.zeros(self.q * self.n), np.zeros(4 * self.n),
                         np.zeros(3 * self.n))
        has, t = C.c_int(), C.c_uint64()
        lib().lbmo_state_get(self.h, _d(f), _d(ft), _d(mo), C.byref(has), _d(ff), C.byref(t))
        scal = []
        for k in range(lib().lbmo_scalar_count(self.h)):
            q, d = C.c_int(), C.c_double()
            lib().lbmo_scalar_raw_get(self.h, k, C.byref(q), C.byref(d), None, None, None)
            h, ht, c = np.zeros(q.value * self.n), np.zeros(q.value * self.n), np.zeros(self.n)
            lib().lbmo_scalar_raw_get(self.h, k, C.byref(q), C.byref(d), _d(h), _d(ht), _d(c))
            scal.append({"q": q.value, "diffusivity": d.value, "h": h.reshape(q.value, self.n),
                         "htmp": ht.reshape(q.value, self.n), "conc": c})
        return {"step": t.value, "f": f.reshape(self.q, self.n), "ftmp": ft.reshape(self.q, self.n),
                "moments": mo.reshape(4, self.n), "force_field": ff.reshape(self.n, 3) if has.value else None,
                "scalars": scal}

    def set_state(self, st):
        """Install a raw state as the reference's load_into does (no moment
        recomputation); scalars k < len(st["scalars"]) must be enabled."""
        ff = st.get("force_field")
        lib().lbmo_state_set(self.h, _d(_as_d(st["f"], self.q * self.n)), _d(_as_d(st["ftmp"], self.q * self.n)),
                             _d(_as_d(st["moments"], 4 * self.n)), int(ff is not None),
                             _d(_as_d(np.zeros(3 * self.n) if ff is None else ff, 3 * self.n)), int(st["step"]))
        for k, x in enumerate(st.get("scalars", [])):
            q = int(x["q"])
            lib().lbmo_scalar_raw_set(self.h, k, float(x["diffusivity"]), _d(_as_d(x["h"], q * self.n)),
                                      _d(_as_d(x["htmp"], q * self.n)), _d(_as_d(x["conc"], self.n)))

    def run_tank(self, pos, w, center, omega, steps, probe_every=1, scalar=-1,
                 max_iterations=3, slip_tolerance=1e-2, kernel_radius=1, relaxation=1.0):
        pos = _as_d(pos).ravel()
        w = _as_d(w).ravel()
        torque = np.full(steps, np.nan)
        ff = np.full(3 * steps, np.nan)
        cv = np.full(steps, np.nan)
        iters = np.zeros(steps)
        done = lib().lbmo_run_tank(self.h, _d(pos), _d(w), w.size, _d(_as_d(center)),
                                   _d(_as_d(omega)), max_iterations, slip_tolerance,
                                   kernel_radius, relaxation, steps, probe_every, scalar,
                                   _d(torque), _d(ff), _d(cv), _d(iters))
        return {"executed": int(done), "torque_lu": torque, "fluid_force": ff.reshape(steps, 3),
                "cv": cv, "ibm_iterations": iters}


def ibm_direct_forcing(dims, d, solid, rho, u_now, pos, w, center, omega, max_iterations=3,
                       slip_tolerance=1e-2, kernel_radius=1, relaxation=1.0):
    n = dims[0] * dims[1] * dims[2]
    solid = np.ascontiguousarray(solid, dtype=np.uint8).ravel()
    rho = _as_d(rho, n)
    u_now = _as_d(u_now, 3 * n)
    pos = _as_d(pos).ravel()
    w = _as_d(w).ravel()
    spread = np.zeros(3 * n)
    diag = np.zeros(15)
    err = C.create_string_buffer(256)
    rc = lib().lbmo_ibm_direct_forcing((C.c_int * 3)(*dims), d, solid.ctypes.data_as(_u8p),
                                       _d(rho), _d(u_now), _d(pos), _d(w), w.size,
                                       _d(_as_d(center)), _d(_as_d(omega)), max_iterations,
                                       slip_tolerance, kernel_radius, relaxation, _d(spread),
                                       _d(diag), err, 256)
    if rc != 0:
        raise ValueError(err.value.decode())
    return spread.reshape(n, 3), diag_dict(diag)


def marker_stencil(p, dims, d=3, radius=1):
    out = np.zeros(4 * 64)
    k = lib().lbmo_marker_stencil(_d(_as_d(p)), (C.c_int * 3)(*dims), d, radius, _d(out))
    return out[: 4 * k].reshape(k, 4)


def wall_rims(dims, is_wall, wall_u, d=3):
    n = dims[0] * dims[1] * dims[2]
    solid = np.zeros(n, dtype=np.uint8)
    wu = np.zeros(3 * n)
    u = _as_d(wall_u, 18)
    lib().lbmo_wall_rims(d, (C.c_int * 3)(*dims), (C.c_int * 6)(*[int(b) for b in is_wall]),
                         _d(u), solid.ctypes.data_as(_u8p), _d(wu))
    return solid, wu.reshape(n, 3)


def build_tank(dims, dx, vessel_d, liquid_h, impeller_d, clearance, blades, omega_z,
               baffle_w=0.0, baffle_t=0.0, kind=0, spacing=0.7):
    """Tank voxels and one impeller's markers. kind 0 Rushton, 1 pitched
    blade (the reference's generators), 2 the device library's flat-blade
    turbine at `spacing` cells."""
    n = dims[0] * dims[1] * dims[2]
    err = C.create_string_buffer(256)
    dims_a = (C.c_int * 3)(*dims)
    m = lib().lbmo_build_tank2(dims_a, dx, vessel_d, liquid_h, baffle_w, baffle_t, kind,
                               impeller_d, clearance, blades, omega_z, spacing, None, None, None, None,
                               None, 0, None, None, err, 256)
    if m < 0:
        raise ValueError(err.value.decode())
    solid = np.zeros(n, dtype=np.uint8)
    baffle = np.zeros(n, dtype=np.uint8)
    wv = np.zeros(3 * n)
    pos = np.zeros(3 * m)
    w = np.zeros(m)
    center = np.zeros(3)
    omega = np.zeros(3)
    lib().lbmo_build_tank2(dims_a, dx, vessel_d, liquid_h, baffle_w, baffle_t, kind, impeller_d,
                           clearance, blades, omega_z, spacing, solid.ctypes.data_as(_u8p),
                           baffle.ctypes.data_as(_u8p), _d(wv), _d(pos), _d(w), m, _d(center),
                           _d(omega), err, 256)
    return {"solid": solid, "baffle": baffle, "wall_velocity": wv.reshape(n, 3),
            "marker_pos": pos.reshape(m, 3), "marker_w": w, "center": center, "omega": omega}


def power_qois(torque, omega, rho, d, volume):
    out = np.zeros(5)
    if lib().lbmo_power_qois(torque, omega, rho, d, volume, _d(out)) != 0:
        raise ValueError("invalid power QOI inputs")
    return dict(zip(("torque_n_m", "power_w", "rotational_speed_hz", "np", "p_over_v_w_m3"), out))


def codec16(mode, values):
    """16-bit storage rounding of float32 values: "ref_f16" the reference's
    host binary16 codec (gpu/backend.rs:160-213, encode then decode),
    "bf16" bfloat16 nearest-even, "f16" binary16 nearest-even."""
    v = np.ascontiguousarray(values, dtype=np.float32).ravel()
    out = np.empty_like(v)
    fp = C.POINTER(C.c_float)
    lib().lbmo_codec16({"ref_f16": 1, "bf16": 2, "f16": 3}[mode], v.ctypes.data_as(fp), out.ctypes.data_as(fp), v.size)
    return out


def f16_bits(values):
    """The reference's f32_to_f16_bits (gpu/backend.rs:160-186)."""
    v = np.ascontiguousarray(values, dtype=np.float32).ravel()
    out = np.empty(v.size, dtype=np.uint16)
    lib().lbmo_f16_bits(v.ctypes.data_as(C.POINTER(C.c_float)), out.ctypes.data_as(C.POINTER(C.c_uint16)), v.size)
    return out


def runner_power(torque_lu, run_steps, probe_every, rho, dx, dt, omega, d, volume, executed=None):
    """write_power_qois over a per-step lattice torque series
    (runner.rs:1396-1425, 1514-1543)."""
    t = _as_d(torque_lu).ravel()
    executed = t.size if executed is None else int(executed)
    out = np.zeros(5)
    used = lib().lbmo_runner_power(_d(t), executed, int(run_steps), int(probe_every), rho, dx, dt, omega, d, volume,
                                   _d(out))
    if used < 0:
        raise ValueError("no torque records or invalid power QOI inputs")
    r = dict(zip(("torque_n_m", "power_w", "rotational_speed_hz", "np", "p_over_v_w_m3"), out))
    r["records_used"] = int(used)
    return r


UNIT_KEYS = ("dx_m", "dt_s", "u_ref_lu", "nu_lu", "tau_lu", "cs2_lu", "reynolds", "froude", "mach_lattice",
             "schmidt", "peclet", "scalar_diffusivity_lu", "grid_reynolds")


def unit_report(vessel_d, liquid_h, imp_d, rpm, rho, mu, dt, grid, d_scalar=0.0):
    """bioprocess_unit_report_unchecked (units.rs:116-325), single phase."""
    out = np.zeros(13)
    bits = (C.c_uint * 2)()
    if lib().lbmo_unit_report(_d(np.array([vessel_d, liquid_h, imp_d, rpm, rho, mu, dt], dtype=np.float64)),
                              (C.c_int * 3)(*grid), float(d_scalar or 0.0), _d(out), bits) != 0:
        raise ValueError("unit report inputs must be finite and positive")
    r = dict(zip(UNIT_KEYS, out))
    r["warnings"], r["rejections"] = int(bits[0]), int(bits[1])
    return r


def top_hat_pulse(dims, solid, dx, center, radius, conc=1.0):
    """scalar_initial_condition, pulse branch (runner.rs:1317-1377)."""
    n = dims[0] * dims[1] * dims[2]
    out = np.zeros(n)
    so = None if solid is None else np.ascontiguousarray(solid, dtype=np.uint8).ravel()
    lib().lbmo_top_hat_pulse((C.c_int * 3)(*dims), None if so is None else so.ctypes.data_as(_u8p), float(dx),
                             _d(_as_d(center)), float(radius), float(conc), _d(out))
    return out


def scalar_cv(values, include):
    v = _as_d(values).ravel()
    inc = np.ascontiguousarray(include, dtype=np.uint8).ravel()
    r = lib().lbmo_scalar_cv(_d(v), inc.ctypes.data_as(_u8p), v.size)
    return None if np.isnan(r) else r


def mixing_time_from_cv(series):
    t = _as_d([s[0] for s in series])
    cv = _as_d([s[1] for s in series])
    out = np.zeros(3)
    if lib().lbmo_mixing_time(_d(t), _d(cv), t.size, _d(out)) != 0:
        return None
    return {"cv0": out[0], "t95": None if np.isnan(out[1]) else out[1],
            "t99": None if np.isnan(out[2]) else out[2]}


def collide_cells(q, real_bits, kind, omega_p, omega_m, omega_shear, f, rho, u, force_field=None):
    """Collide independent cells in place; f is (q, n) float64."""
    L = lib()
    L.lbmo_collide_cells.restype = C.c_int
    L.lbmo_collide_cells.argtypes = [C.c_int, C.c_int, C.c_int, C.c_double, C.c_double,
                                     C.c_double, C.c_long, _dp, _dp, _dp, _dp]
    f = np.ascontiguousarray(f, dtype=np.float64).copy()
    n = f.shape[1]
    ff = None if force_field is None else _as_d(force_field, 3 * n)
    rc = L.lbmo_collide_cells(q, real_bits, COLLISION[kind], omega_p, omega_m, omega_shear, n,
                              _d(f), _d(_as_d(rho, n)), _d(_as_d(u, 3 * n)), _d(ff))
    if rc != 0:
        raise ValueError("unsupported lattice/precision")
    return f


def equilibrium_cells(q, real_bits, rho, u):
    L = lib()
    L.lbmo_equilibrium_cells.restype = C.c_int
    L.lbmo_equilibrium_cells.argtypes = [C.c_int, C.c_int, C.c_long, _dp, _dp, _dp]
    rho = _as_d(rho)
    n = rho.size
    out = np.zeros((q, n))
    L.lbmo_equilibrium_cells(q, real_bits, n, _d(rho), _d(_as_d(u, 3 * n)), _d(out))
    return out


def compute_stress_field(dims, ux, uy, uz, solid, dx, mu):
    """stress.rs compute_stress_field (f64, SI fields, mu per cell or scalar):
    dict of s (n x 6), gamma_dot, viscous_stress, second_invariant, von_mises."""
    n = int(np.prod(dims))
    d = (C.c_int * 3)(*[int(v) for v in dims])
    mu = np.full(n, float(mu)) if np.isscalar(mu) else _as_d(mu, n)
    sol = np.ascontiguousarray(solid, dtype=np.uint8)
    out = {k: np.zeros(n) for k in ("gamma_dot", "viscous_stress", "second_invariant", "von_mises")}
    s6 = np.zeros(6 * n)
    lib().lbmo_compute_stress_field(d, _d(_as_d(ux, n)), _d(_as_d(uy, n)), _d(_as_d(uz, n)),
                                    sol.ctypes.data_as(_u8p), float(dx), _d(mu), _d(s6), _d(out["gamma_dot"]),
                                    _d(out["viscous_stress"]), _d(out["second_invariant"]), _d(out["von_mises"]))
    out["s"] = s6.reshape(n, 6)
    return out


def percentile_summary(values, threshold=None):
    """stress.rs percentile_summary: {p50, p90, p95, p99, max,
    fraction_above_threshold} over the finite values, or None."""
    v = _as_d(values)
    out = np.zeros(6)
    ok = lib().lbmo_percentile_summary(_d(v), v.size, 0 if threshold is None else 1,
                                       0.0 if threshold is None else float(threshold), _d(out))
    if not ok:
        return None
    keys = ("p50", "p90", "p95", "p99", "max", "fraction_above_threshold")
    r = dict(zip(keys, out.tolist()))
    if threshold is None:
        r["fraction_above_threshold"] = None
    return r


def wall_shear_proxy(dims, ux, uy, uz, solid, wall_u, dx, rho, mu):
    """stress.rs wall_shear_proxy: per wall-adjacent fluid cell (cell order)
    cell_index, tau_w, y_plus, u_parallel, normal (x3)."""
    n = int(np.prod(dims))
    d = (C.c_int * 3)(*[int(v) for v in dims])
    sol = np.ascontiguousarray(solid, dtype=np.uint8)
    wu = _as_d(wall_u, 3 * n)
    cap = n
    cell = np.zeros(cap, dtype=np.int64)
    tau, yp, up, nrm = np.zeros(cap), np.zeros(cap), np.zeros(cap), np.zeros(3 * cap)
    k = lib().lbmo_wall_shear_proxy(d, _d(_as_d(ux, n)), _d(_as_d(uy, n)), _d(_as_d(uz, n)),
                                    sol.ctypes.data_as(_u8p), _d(wu), float(dx), float(rho), float(mu), cap,
                                    cell.ctypes.data_as(C.POINTER(C.c_int64)), _d(tau), _d(yp), _d(up), _d(nrm))
    return {"cell_index": cell[:k], "tau_w": tau[:k], "y_plus": yp[:k], "u_parallel": up[:k],
            "normal": nrm[:3 * k].reshape(k, 3)}


OUR_KIND = {"constant": 0, "monod": 1, "cell_density_scaled": 2}


def _diag(d):
    return {"clipped_cells": int(d[0]), "clipped_fraction": d[1], "min_before_clip": d[2]}


def interfacial_flux(c, c_star, area, volume, dt, kl, cumulative=0.0):
    """oxygen.rs apply_interfacial_flux_sources on a copy of c: (c_new,
    ledger, diag), or raises ValueError with the error code."""
    c = _as_d(c).copy()
    n = c.size
    ledger = np.array([cumulative, 0.0, 0.0, 0.0])
    diag = np.zeros(3)
    cs = np.full(n, float(c_star)) if np.isscalar(c_star) else _as_d(c_star, n)
    vol = np.full(n, float(volume)) if np.isscalar(volume) else _as_d(volume, n)
    e = lib().lbmo_interfacial_flux(_d(c), _d(cs), _d(_as_d(area, n)), _d(vol), n, float(dt), float(kl), _d(ledger),
                                    _d(diag))
    if e:
        raise ValueError(f"oxygen source error {e}")
    return c, {"cumulative_mol": ledger[0], "last_step_mol": ledger[1], "source_integral_mol_s": ledger[2],
               "active_interface_cells": int(ledger[3])}, _diag(diag)


def oxygen_uptake(c, volume, dt, kind="constant", our=0.0, our_max=0.0, ks=0.0, c_ref=0.0, specific_our=0.0,
                  density=None, cumulative=0.0):
    """reaction.rs apply_oxygen_reaction_source on a copy of c."""
    c = _as_d(c).copy()
    n = c.size
    vol = np.full(n, float(volume)) if np.isscalar(volume) else _as_d(volume, n)
    ledger = np.array([cumulative, 0.0])
    diag = np.zeros(3)
    params = np.array([our, our_max, ks, c_ref, specific_our], dtype=np.float64)
    dens = None if density is None else _as_d(density, n)
    e = lib().lbmo_oxygen_uptake(_d(c), _d(vol), n, float(dt), OUR_KIND[kind], _d(params), _d(dens), _d(ledger),
                                 _d(diag))
    if e:
        raise ValueError(f"reaction source error {e}")
    return c, {"cumulative_kmol_consumed": ledger[0], "last_step_kmol_consumed": ledger[1]}, _diag(diag)


def henry_equilibrium(h, p):
    return lib().lbmo_henry_equilibrium(float(h), float(p))


def interfacial_area_density(phi, grad, width):
    return lib().lbmo_interfacial_area_density(float(phi), _d(_as_d(grad, 3)), float(width))

