"""lbmflow_b200: B200 (sm_100a) LBMFlow single-GPU time step.

Python mirror of the reference's stepping API (lbm-core ``Solver`` over the
``Backend`` trait) on top of the C ABI in ``include/lbmb.h``. All compute
runs in ``_build/liblbmb.so`` (hand-written CUDA for sm_100a); there is no
CPU fallback: every call fails loudly when the library or a CUDA device is
missing.
"""
from __future__ import annotations

import ctypes as C
import os
from dataclasses import dataclass, field

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_build", "liblbmb.so")

_dp = C.POINTER(C.c_double)
_u8p = C.POINTER(C.c_uint8)
_i32p = C.POINTER(C.c_int32)
_i64p = C.POINTER(C.c_int64)

OK, ERR_INVALID, ERR_CUDA, ERR_UNSUPPORTED, ERR_DIVERGED, ERR_STATE, ERR_NOMEM = 0, -1, -2, -3, -4, -5, -6
ERR_CHECKPOINT = -7
COLLISION = {"bgk": 0, "trt": 1, "cm": 2, "central_moment": 2}
STORAGE = {"f32": 0, "f16": 1, "bf16": 2, "f64": 3}
SWEEP = {"direct": 0, "bulk": 1, "async": 2, "pair": 3, "tile": 4, "lean": 5, "window": 6}
IMPELLER = {"rushton": 0, "pitched": 1, "flat_blade": 2}
MAGIC_STD = 3.0 / 16.0
RED_FLUID_CELLS, RED_MASS_DEV, RED_MOMENTUM = 0, 1, 2

# Symbols the library exports; kept in sync with include/lbmb.h (checked by
# tests/test_abi.py).
EXPORTS = (
    "lbmb_last_error", "lbmb_version", "lbmb_create", "lbmb_destroy", "lbmb_shape", "lbmb_init_fields",
    "lbmb_stage_in", "lbmb_stage_out", "lbmb_step", "lbmb_run_guarded", "lbmb_read_moments", "lbmb_reduce",
    "lbmb_total_mass", "lbmb_clear_body_force_field", "lbmb_get_force_field", "lbmb_ibm_set_body",
    "lbmb_apply_rotating_ibm", "lbmb_runner_step", "lbmb_enable_scalar", "lbmb_set_scalar_concentration",
    "lbmb_gather_scalar_concentration", "lbmb_scalar_cv", "lbmb_run_impeller", "lbmb_last_timing",
    "lbmb_build_wall_rims", "lbmb_build_stirred_tank", "lbmb_sync", "lbmb_reduce_populations_noalloc",
    "lbmb_set_sweep_kernel", "lbmb_get_sweep_kernel", "lbmb_set_sweep_variant", "lbmb_autotune_sweep",
    "lbmb_batch_create", "lbmb_batch_autotune", "lbmb_batch_run", "lbmb_batch_destroy", "lbmb_adjoint_torque",
    "lbmb_gather_strain_rate", "lbmb_stress_field", "lbmb_stress_summary", "lbmb_wall_shear_proxy",
    "lbmb_scalar_interfacial_flux", "lbmb_scalar_oxygen_uptake", "lbmb_set_omega_field",
    "lbmb_gather_velocity_gradient", "lbmb_wale_update", "lbmb_get_time", "lbmb_set_scalar_name",
    "lbmb_set_qoi_checkpoint_state", "lbmb_get_qoi_checkpoint_state", "lbmb_checkpoint_save",
    "lbmb_checkpoint_restore", "lbmb_checkpoint_write_host", "lbmb_checkpoint_read_host", "lbmb_fnv1a64",
    "lbmb_run_impeller_status", "lbmb_power_qois", "lbmb_power_from_torque_series", "lbmb_unit_report",
    "lbmb_scalar_top_hat_pulse", "lbmb_scalar_diffusivity_lu", "lbmb_capabilities", "lbmb_set_wait_limit",
)


class LbmbError(RuntimeError):
    """A failed lbmb call; .code is the lbmb_status."""

    def __init__(self, code, msg):
        super().__init__(f"[{code}] {msg}")
        self.code = code


class SpecError(LbmbError, ValueError):
    """Invalid specification (the reference's SpecError)."""


class UnsupportedError(LbmbError):
    """UnsupportedReason::NotImplemented."""


class CheckpointError(LbmbError):
    """CheckpointError (solver.rs:46-82): .code is the reference's stable
    code ("CKPT_IO", "CKPT_BAD_MAGIC", ...), .message its text, .status the
    lbmb_status (-7)."""

    def __init__(self, status, msg):
        code, _, message = msg.partition(": ")
        super().__init__(status, msg)
        self.status = status
        self.code = code
        self.message = message


class Diverged(LbmbError):
    """Non-finite mass detected by run_guarded; .completed steps ran."""

    def __init__(self, code, msg, completed):
        super().__init__(code, msg)
        self.completed = completed


class _CkptSpec(C.Structure):
    _fields_ = [("lattice", C.c_int32), ("collision", C.c_int32), ("dtype_bits", C.c_int32),
                ("dims", C.c_int32 * 3), ("periodic", C.c_int32 * 3), ("nu", C.c_double), ("magic", C.c_double),
                ("omega_shear", C.c_double), ("force", C.c_double * 3)]


class _CkptScalar(C.Structure):
    _fields_ = [("name", C.c_char * 64), ("diffusivity", C.c_double), ("q", C.c_int32), ("h", _dp),
                ("h_capacity", C.c_int64), ("conc", _dp)]


class _CkptData(C.Structure):
    _fields_ = [("step", C.c_uint64), ("f", _dp), ("moments", _dp), ("has_force_field", C.c_int32),
                ("force_field", _dp), ("n_scalars", C.c_int32), ("scalar_capacity", C.c_int32),
                ("scalars", C.POINTER(_CkptScalar)), ("has_qoi", C.c_int32), ("qoi_json", C.POINTER(C.c_char)),
                ("qoi_len", C.c_int64), ("qoi_capacity", C.c_int64)]


class _Config(C.Structure):
    _fields_ = [("lattice", C.c_int32), ("collision", C.c_int32), ("storage", C.c_int32),
                ("dims", C.c_int32 * 3), ("periodic", C.c_int32 * 3), ("device", C.c_int32),
                ("nu", C.c_double), ("magic", C.c_double), ("omega_shear", C.c_double),
                ("force", C.c_double * 3), ("smagorinsky_cs", C.c_double), ("free_slip_top", C.c_int32)]


class _AutotuneResult(C.Structure):
    _fields_ = [("kind", C.c_int32), ("even_blocks_per_sm", C.c_int32), ("odd_blocks_per_sm", C.c_int32),
                ("n_trials", C.c_int32), ("best_ms_per_step", C.c_double), ("default_ms_per_step", C.c_double)]


class _AdjointConfig(C.Structure):
    _fields_ = [("steps", C.c_int64), ("window_begin", C.c_int64), ("checkpoint_every", C.c_int32),
                ("body", C.c_int32)]


class _AdjointResult(C.Structure):
    _fields_ = [("J", C.c_double), ("dJ_dnu", C.c_double), ("dJ_domega_z", C.c_double),
                ("dJ_domega_plus", C.c_double), ("dJ_domega_minus", C.c_double), ("forward_ms", C.c_double),
                ("adjoint_ms", C.c_double), ("markers", C.c_int64)]


class _IbmConfig(C.Structure):
    _fields_ = [("max_iterations", C.c_int32), ("slip_tolerance", C.c_double),
                ("kernel_radius", C.c_int32), ("relaxation", C.c_double)]


class _IbmDiag(C.Structure):
    _fields_ = [("iterations", C.c_int32), ("slip_max", C.c_double), ("slip_rms", C.c_double),
                ("slip_max_rel", C.c_double), ("slip_rms_rel", C.c_double), ("torque", C.c_double * 3),
                ("fluid_force", C.c_double * 3), ("marker_force", C.c_double * 3),
                ("momentum_error_rel", C.c_double)]


class _Percentiles(C.Structure):
    _fields_ = [("p50", C.c_double), ("p90", C.c_double), ("p95", C.c_double), ("p99", C.c_double),
                ("max", C.c_double), ("fraction_above_threshold", C.c_double), ("count", C.c_int64),
                ("valid", C.c_int32)]

    def as_dict(self):
        if not self.valid:
            return None
        f = self.fraction_above_threshold
        return {"p50": self.p50, "p90": self.p90, "p95": self.p95, "p99": self.p99, "max": self.max,
                "fraction_above_threshold": None if np.isnan(f) else f, "count": self.count}


class _WaleDiag(C.Structure):
    _fields_ = [("clipped_cells", C.c_int64), ("clipped_fraction", C.c_double),
                ("max_nu_t_before_clipping", C.c_double), ("tau_eff_max", C.c_double), ("nu_t_max", C.c_double)]


class _OxygenDiag(C.Structure):
    _fields_ = [("clipped_cells", C.c_int64), ("clipped_fraction", C.c_double), ("min_before_clip", C.c_double)]

    def as_dict(self):
        return {"clipped_cells": self.clipped_cells, "clipped_fraction": self.clipped_fraction,
                "min_before_clip": self.min_before_clip}


class _OxygenLedger(C.Structure):
    _fields_ = [("cumulative_mol", C.c_double), ("last_step_mol", C.c_double),
                ("source_integral_mol_s", C.c_double), ("active_interface_cells", C.c_int64)]


class _OurLedger(C.Structure):
    _fields_ = [("cumulative_kmol_consumed", C.c_double), ("last_step_kmol_consumed", C.c_double)]


class _OurModel(C.Structure):
    _fields_ = [("kind", C.c_int32), ("our_kmol_m3_s", C.c_double), ("our_max", C.c_double), ("ks", C.c_double),
                ("c_ref", C.c_double), ("specific_our", C.c_double)]


OUR_KIND = {"constant": 0, "monod": 1, "cell_density_scaled": 2}


class _WallShear(C.Structure):
    _fields_ = [("cell_index", C.c_int64), ("tau_w_pa", C.c_double), ("y_plus", C.c_double),
                ("u_parallel_m_s", C.c_double), ("y_m", C.c_double), ("normal", C.c_double * 3)]


class _TankSpec(C.Structure):
    _fields_ = [("dims", C.c_int32 * 3), ("dx_m", C.c_double), ("vessel_diameter_m", C.c_double),
                ("liquid_height_m", C.c_double), ("baffle_count", C.c_int32),
                ("baffle_width_m", C.c_double), ("baffle_thickness_m", C.c_double),
                ("impeller_kind", C.c_int32), ("impeller_diameter_m", C.c_double),
                ("clearance_m", C.c_double), ("blade_count", C.c_int32), ("omega_rad_s", C.c_double),
                ("marker_spacing_cells", C.c_double), ("min_cells", C.c_double)]


class _PowerResult(C.Structure):
    _fields_ = [("torque_n_m", C.c_double), ("power_w", C.c_double), ("rotational_speed_hz", C.c_double),
                ("np", C.c_double), ("p_over_v_w_m3", C.c_double)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


class _UnitInput(C.Structure):
    _fields_ = [("vessel_diameter_m", C.c_double), ("liquid_height_m", C.c_double),
                ("impeller_diameter_m", C.c_double), ("rotational_speed_rpm", C.c_double),
                ("liquid_density_kg_m3", C.c_double), ("liquid_viscosity_pa_s", C.c_double), ("dt_s", C.c_double),
                ("grid", C.c_int32 * 3), ("scalar_diffusivity_m2_s", C.c_double)]


class _UnitMapping(C.Structure):
    _fields_ = [("dx_m", C.c_double), ("dt_s", C.c_double), ("u_ref_lu", C.c_double), ("nu_lu", C.c_double),
                ("tau_lu", C.c_double), ("cs2_lu", C.c_double), ("reynolds", C.c_double), ("froude", C.c_double),
                ("mach_lattice", C.c_double), ("schmidt", C.c_double), ("peclet", C.c_double),
                ("scalar_diffusivity_lu", C.c_double), ("grid_reynolds", C.c_double), ("warnings", C.c_uint32),
                ("rejections", C.c_uint32)]


class _BackendCaps(C.Structure):
    _fields_ = [("handles_single_part_periodic_halo", C.c_int32), ("supports_localized_features", C.c_int32),
                ("supports_d3q27_open_faces", C.c_int32), ("supports_two_pass", C.c_int32),
                ("supports_gravity_body_force", C.c_int32), ("distribution_hydro", C.c_int32),
                ("distribution_phase", C.c_int32), ("distribution_scalar", C.c_int32),
                ("run_chunk_size", C.c_int64), ("lattices", C.c_uint32), ("storages", C.c_uint32),
                ("collisions", C.c_uint32), ("adjoint", C.c_int32), ("batch", C.c_int32), ("checkpoint", C.c_int32)]


# Feasibility codes of the unit report (crates/lbm-scenario/src/units.rs), by bit.
UNIT_ISSUES = {1: "MA_LATTICE_HIGH", 2: "MA_LATTICE_TOO_HIGH", 4: "TAU_NEAR_HALF", 8: "TAU_NON_POSITIVE_VISCOSITY",
               16: "GRID_REYNOLDS_HIGH", 32: "SCALAR_DIFFUSION_UNSTABLE"}

_lib = None


def lib():
    """The loaded CUDA library (raises if it was never built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(f"lbmflow_b200 CUDA library not built: {LIB_PATH} (run lbmflow_b200/build.py)")
        L = C.CDLL(LIB_PATH)
        L.lbmb_last_error.restype = C.c_char_p
        L.lbmb_version.restype = C.c_char_p
        L.lbmb_create.argtypes = [C.POINTER(_Config), _u8p, _dp, C.POINTER(C.c_void_p)]
        vp = C.c_void_p
        L.lbmb_destroy.argtypes = [vp]
        L.lbmb_shape.argtypes = [vp, _i64p, _i32p]
        L.lbmb_init_fields.argtypes = [vp, _dp, _dp]
        L.lbmb_stage_in.argtypes = [vp, _dp]
        L.lbmb_stage_out.argtypes = [vp, _dp]
        L.lbmb_step.argtypes = [vp, C.c_int64]
        L.lbmb_run_guarded.argtypes = [vp, C.c_int64, C.c_int64, _i64p]
        L.lbmb_read_moments.argtypes = [vp, _dp, _dp, _dp, _dp]
        L.lbmb_reduce.argtypes = [vp, C.c_int32, C.c_int32, _dp]
        L.lbmb_total_mass.argtypes = [vp, _dp]
        L.lbmb_clear_body_force_field.argtypes = [vp]
        L.lbmb_get_force_field.argtypes = [vp, _dp]
        L.lbmb_ibm_set_body.argtypes = [vp, C.c_int32, _dp, _dp, C.c_int64, _dp, _dp]
        L.lbmb_apply_rotating_ibm.argtypes = [vp, C.c_int32, C.POINTER(_IbmConfig), C.POINTER(_IbmDiag)]
        L.lbmb_runner_step.argtypes = [vp, C.c_int32, _dp, _dp, C.c_int64, _dp, _dp, C.POINTER(_IbmConfig),
                                       C.POINTER(_IbmDiag)]
        L.lbmb_enable_scalar.argtypes = [vp, C.c_int32, C.c_double, _i32p]
        L.lbmb_set_scalar_concentration.argtypes = [vp, C.c_int32, _dp]
        L.lbmb_gather_scalar_concentration.argtypes = [vp, C.c_int32, _dp]
        L.lbmb_scalar_cv.argtypes = [vp, C.c_int32, _dp]
        L.lbmb_run_impeller.argtypes = [vp, C.c_int32, C.POINTER(_IbmConfig), C.c_int64, C.c_int32,
                                        C.c_int64, _dp, _dp, _dp, _i32p]
        L.lbmb_run_impeller_status.argtypes = [vp, _i64p, _i32p]
        L.lbmb_last_timing.argtypes = [vp, _dp, _dp, _i64p]
        L.lbmb_build_wall_rims.argtypes = [_i32p, _i32p, _dp, _u8p, _dp]
        L.lbmb_build_stirred_tank.argtypes = [C.POINTER(_TankSpec), _u8p, _u8p, _dp, _dp, _dp, C.c_int64,
                                              _i64p, _dp, _dp]
        L.lbmb_sync.argtypes = [vp]
        L.lbmb_gather_strain_rate.argtypes = [vp, _dp, _dp]
        L.lbmb_set_omega_field.argtypes = [vp, _dp]
        L.lbmb_gather_velocity_gradient.argtypes = [vp, _dp]
        L.lbmb_wale_update.argtypes = [vp, C.c_double, _dp, C.POINTER(_WaleDiag)]
        L.lbmb_scalar_interfacial_flux.argtypes = [vp, C.c_int32, _dp, C.c_double, _dp, _dp, C.c_double, C.c_double,
                                                   C.c_double, C.POINTER(_OxygenLedger), C.POINTER(_OxygenDiag)]
        L.lbmb_scalar_oxygen_uptake.argtypes = [vp, C.c_int32, C.POINTER(_OurModel), _dp, _dp, C.c_double,
                                                C.c_double, C.POINTER(_OurLedger), C.POINTER(_OxygenDiag)]
        L.lbmb_stress_field.argtypes = [vp, C.c_double, C.c_double, C.c_double, _dp, _dp, _dp]
        L.lbmb_stress_summary.argtypes = [vp, C.c_double, C.c_double, C.c_double, C.c_double, C.c_double,
                                          C.POINTER(_Percentiles), C.POINTER(_Percentiles), _dp]
        L.lbmb_wall_shear_proxy.argtypes = [vp, C.c_double, C.c_double, C.c_double, C.c_double,
                                            C.POINTER(_WallShear), C.c_int64, _i64p]
        L.lbmb_set_sweep_kernel.argtypes = [vp, C.c_int32]
        L.lbmb_get_sweep_kernel.argtypes = [vp, _i32p]
        L.lbmb_set_sweep_variant.argtypes = [vp, C.c_int32, C.c_int32]
        L.lbmb_autotune_sweep.argtypes = [vp, C.c_int32, C.POINTER(_AutotuneResult), _i32p, _dp, C.c_int32]
        L.lbmb_batch_create.argtypes = [C.POINTER(vp), _i32p, C.c_int32, C.POINTER(_IbmConfig), C.POINTER(vp)]
        L.lbmb_batch_autotune.argtypes = [vp, C.c_int32, _i32p, _i32p, _dp]
        L.lbmb_batch_run.argtypes = [vp, C.c_int64, _dp, _dp]
        L.lbmb_batch_destroy.argtypes = [vp]
        L.lbmb_adjoint_torque.argtypes = [vp, C.POINTER(_IbmConfig), C.POINTER(_AdjointConfig),
                                          C.POINTER(_AdjointResult), _dp, _dp]
        L.lbmb_reduce_populations_noalloc.argtypes = [vp, C.c_int32, C.c_int32, C.c_int64, C.c_int64, vp, _dp,
                                                      _dp, vp]
        L.lbmb_get_time.argtypes = [vp, C.POINTER(C.c_uint64)]
        L.lbmb_set_scalar_name.argtypes = [vp, C.c_int32, C.c_char_p]
        L.lbmb_set_qoi_checkpoint_state.argtypes = [vp, C.c_char_p, C.c_int64]
        L.lbmb_get_qoi_checkpoint_state.argtypes = [vp, C.c_char_p, C.c_int64, _i64p]
        L.lbmb_checkpoint_save.argtypes = [vp, C.c_char_p]
        L.lbmb_checkpoint_restore.argtypes = [vp, C.c_char_p]
        L.lbmb_checkpoint_write_host.argtypes = [C.c_char_p, C.POINTER(_CkptSpec), _u8p, _dp, C.POINTER(_CkptData)]
        L.lbmb_checkpoint_read_host.argtypes = [C.c_char_p, C.POINTER(_CkptSpec), _u8p, _dp, C.POINTER(_CkptData)]
        L.lbmb_fnv1a64.argtypes = [C.c_char_p, C.c_uint64]
        L.lbmb_fnv1a64.restype = C.c_uint64
        L.lbmb_power_qois.argtypes = [C.c_double] * 5 + [C.POINTER(_PowerResult)]
        L.lbmb_power_from_torque_series.argtypes = [_dp, C.c_int64, C.c_int64, C.c_int64] + [C.c_double] * 6 + [
            C.POINTER(_PowerResult), _i64p]
        L.lbmb_unit_report.argtypes = [C.POINTER(_UnitInput), C.POINTER(_UnitMapping)]
        L.lbmb_scalar_top_hat_pulse.argtypes = [_i32p, _u8p, C.c_double, _dp, C.c_double, C.c_double, _dp]
        L.lbmb_scalar_diffusivity_lu.argtypes = [C.c_double, C.c_double, C.c_double, _dp]
        L.lbmb_capabilities.argtypes = [vp, C.POINTER(_BackendCaps)]
        L.lbmb_set_wait_limit.argtypes = [vp, C.c_int64]
        _lib = L
    return _lib


def _check(rc, completed=None):
    if rc == OK:
        return
    msg = lib().lbmb_last_error().decode()
    if rc == ERR_INVALID:
        raise SpecError(rc, msg)
    if rc == ERR_UNSUPPORTED:
        raise UnsupportedError(rc, msg)
    if rc == ERR_DIVERGED:
        raise Diverged(rc, msg, completed)
    if rc == ERR_CHECKPOINT:
        raise CheckpointError(rc, msg)
    raise LbmbError(rc, msg)


def _d(a):
    return None if a is None else a.ctypes.data_as(_dp)


def _f64(a, n=None):
    a = np.ascontiguousarray(a, dtype=np.float64)
    if n is not None and a.size != n:
        raise ValueError(f"expected {n} values, got {a.size}")
    return a


@dataclass
class DirectForcingConfig:
    """rotating_ibm.rs:106-130 (defaults: 3 sweeps, tol 1e-2, radius 1, relax 1)."""
    max_iterations: int = 3
    slip_tolerance: float = 1.0e-2
    kernel_radius: int = 1
    relaxation: float = 1.0

    def _c(self):
        return _IbmConfig(self.max_iterations, self.slip_tolerance, self.kernel_radius, self.relaxation)


@dataclass
class IbmDiagnostics:
    """rotating_ibm.rs:134-153."""
    iterations: int
    slip_max: float
    slip_rms: float
    slip_max_rel: float
    slip_rms_rel: float
    torque: np.ndarray
    fluid_force: np.ndarray
    marker_force: np.ndarray
    momentum_error_rel: float


@dataclass
class RotatingBody:
    """rotating_ibm.rs:24-102: markers at lattice coordinates, Omega x r target."""
    center: np.ndarray
    omega: np.ndarray
    positions: np.ndarray  # (n, 3)
    weights: np.ndarray  # (n,)

    def __post_init__(self):
        self.center = _f64(self.center, 3)
        self.omega = _f64(self.omega, 3)
        self.positions = _f64(self.positions).reshape(-1, 3)
        self.weights = _f64(self.weights).ravel()

    @staticmethod
    def circle_2d(center, radius, omega_z, n_markers, z=0.0):
        th = 2.0 * np.pi * np.arange(n_markers) / n_markers
        pos = np.stack([center[0] + radius * np.cos(th), center[1] + radius * np.sin(th),
                        np.full(n_markers, z)], axis=1)
        w = np.full(n_markers, 2.0 * np.pi * radius / n_markers)
        return RotatingBody([center[0], center[1], z], [0.0, 0.0, omega_z], pos, w)


class Solver:
    """One device solver (Solver<L, T, B, H>, crates/lbm-core/src/solver.rs:1503)."""

    def __init__(self, dims, lattice=19, collision="trt", storage="f32", nu=1.0 / 6.0, magic=MAGIC_STD,
                 omega_shear=None, periodic=(False, False, False), force=(0.0, 0.0, 0.0), solid=None,
                 wall_u=None, device=0, smagorinsky_cs=0.0, free_slip_top=False):
        L = lib()
        self.dims = tuple(int(d) for d in dims)
        self.n = self.dims[0] * self.dims[1] * self.dims[2]
        self.q = int(lattice)
        if omega_shear is None:
            omega_shear = 1.0 / (3.0 * nu + 0.5)
        cfg = _Config(int(lattice), COLLISION[collision], STORAGE[storage], (C.c_int32 * 3)(*self.dims),
                      (C.c_int32 * 3)(*[int(bool(p)) for p in periodic]), int(device), float(nu),
                      float(magic), float(omega_shear), (C.c_double * 3)(*[float(f) for f in force]),
                      float(smagorinsky_cs), int(bool(free_slip_top)))
        self._solid = None if solid is None else np.ascontiguousarray(solid, dtype=np.uint8).ravel()
        if self._solid is not None and self._solid.size != self.n:
            raise ValueError("solid mask size does not match the grid")
        self._wall = None if wall_u is None else _f64(wall_u, 3 * self.n)
        h = C.c_void_p()
        _check(L.lbmb_create(C.byref(cfg), None if self._solid is None else self._solid.ctypes.data_as(_u8p),
                             _d(self._wall), C.byref(h)))
        self.h = h
        self._bodies = {}
        self._runner_args = None
        self._lib = L  # kept for close() during interpreter shutdown

    def close(self):
        if getattr(self, "h", None):
            (getattr(self, "_lib", None) or lib()).lbmb_destroy(self.h)
            self.h = None

    __del__ = close

    # --- state ------------------------------------------------------------
    def init_with(self, rho, u):
        _check(lib().lbmb_init_fields(self.h, _d(_f64(rho, self.n)), _d(_f64(u, 3 * self.n))))

    def stage_in(self, f):
        _check(lib().lbmb_stage_in(self.h, _d(_f64(f, self.q * self.n))))

    def stage_out(self):
        out = np.empty(self.q * self.n)
        _check(lib().lbmb_stage_out(self.h, _d(out)))
        return out.reshape(self.q, self.n)

    # --- stepping ---------------------------------------------------------
    def step(self):
        self.run(1)

    def run(self, steps):
        _check(lib().lbmb_step(self.h, int(steps)))

    def run_guarded(self, steps, check_every):
        done = C.c_int64(0)
        rc = lib().lbmb_run_guarded(self.h, int(steps), int(check_every), C.byref(done))
        _check(rc, completed=done.value)
        return done.value

    def sync(self):
        _check(lib().lbmb_sync(self.h))

    def set_wait_limit(self, cycles):
        """Bound (SM cycles) on the bulk-copy sweeps' mbarrier waits; 0 = the
        default, negative = the timeout self-test on the next such sweep."""
        _check(lib().lbmb_set_wait_limit(self.h, int(cycles)))

    def set_sweep_kernel(self, kind):
        """Pick the collide-stream kernel ("direct", "bulk", "async", "pair", "tile", "lean", "window");
        UnsupportedError if it cannot run this configuration."""
        _check(lib().lbmb_set_sweep_kernel(self.h, SWEEP[kind] if isinstance(kind, str) else int(kind)))

    def set_sweep_variant(self, even_blocks_per_sm, odd_blocks_per_sm):
        """Register budget of the current sweep kernel per parity, as resident
        blocks per SM: 6..10 for "lean", 4..6 for "async" (fp32 storage), 2..4
        for "window" (256-thread blocks), 3..5 for "pair" (13..15: the same
        with the next tile's populations staged by cp.async)."""
        _check(lib().lbmb_set_sweep_variant(self.h, int(even_blocks_per_sm), int(odd_blocks_per_sm)))

    def autotune_sweep(self, steps_per_trial=20):
        """Time every applicable sweep kernel on this solver's grid and keep
        the fastest (state preserved). Returns the choice and the trials."""
        cap = 256
        r = _AutotuneResult()
        desc = np.zeros(3 * cap, dtype=np.int32)
        ms = np.zeros(cap)
        _check(lib().lbmb_autotune_sweep(self.h, int(steps_per_trial), C.byref(r), desc.ctypes.data_as(_i32p),
                                         _d(ms), cap))
        names = {v: k for k, v in SWEEP.items()}
        trials = [(names[int(desc[3 * i])], int(desc[3 * i + 1]), int(desc[3 * i + 2]), float(ms[i]))
                  for i in range(min(r.n_trials, cap))]
        return {"kind": names[r.kind], "even_blocks_per_sm": r.even_blocks_per_sm,
                "odd_blocks_per_sm": r.odd_blocks_per_sm, "best_ms_per_step": r.best_ms_per_step,
                "default_ms_per_step": r.default_ms_per_step, "trials": trials}

    @property
    def sweep_kernel(self):
        k = C.c_int32()
        _check(lib().lbmb_get_sweep_kernel(self.h, C.byref(k)))
        return {v: n for n, v in SWEEP.items()}[k.value]

    def last_timing(self):
        t, hy, k = C.c_double(), C.c_double(), C.c_int64()
        _check(lib().lbmb_last_timing(self.h, C.byref(t), C.byref(hy), C.byref(k)))
        return t.value, hy.value, k.value

    # --- readback -----------------------------------------------------------
    def read_moments(self):
        out = [np.empty(self.n) for _ in range(4)]
        _check(lib().lbmb_read_moments(self.h, *[_d(a) for a in out]))
        return out

    def reduce(self, kind, axis=0):
        v = C.c_double()
        _check(lib().lbmb_reduce(self.h, int(kind), int(axis), C.byref(v)))
        return v.value

    def total_mass_f64(self):
        v = C.c_double()
        _check(lib().lbmb_total_mass(self.h, C.byref(v)))
        return v.value

    def total_momentum(self):
        return np.array([self.reduce(RED_MOMENTUM, a) for a in range(3)])

    # --- forcing / IBM ------------------------------------------------------
    # --- per-cell relaxation field and WALE -------------------------------
    def set_omega_field(self, omega):
        """Solver::set_omega_field: per-cell omega+ (TRT/BGK) or shear rate
        (central moment) for the following collisions; None removes it."""
        _check(lib().lbmb_set_omega_field(self.h, None if omega is None else _d(_f64(omega, self.n))))

    def velocity_gradient(self):
        """Solver::gather_velocity_gradient: n x 3 x 3, g[i][j] = du_i/dx_j."""
        g = np.empty(9 * self.n)
        _check(lib().lbmb_gather_velocity_gradient(self.h, _d(g)))
        return g.reshape(self.n, 3, 3)

    def wale_update(self, tau_eff_max=None):
        """WaleLes::update (Cw 0.325): nu_t per cell and diagnostics; the
        omega+ field is installed on the device for the next collision."""
        nu_t, d = np.empty(self.n), _WaleDiag()
        _check(lib().lbmb_wale_update(self.h, float("nan") if tau_eff_max is None else float(tau_eff_max), _d(nu_t),
                                      C.byref(d)))
        return nu_t, {"clipped_cells": d.clipped_cells, "clipped_fraction": d.clipped_fraction,
                      "max_nu_t_before_clipping": d.max_nu_t_before_clipping,
                      "tau_eff_max": None if np.isnan(d.tau_eff_max) else d.tau_eff_max,
                      "nu_t_max": None if np.isnan(d.nu_t_max) else d.nu_t_max}

    # --- oxygen transfer and uptake on a scalar --------------------------
    def apply_interfacial_flux_sources(self, scalar, area_density, c_star, cell_volume, dt_s, kl_m_s,
                                       cumulative_mol=0.0):
        """oxygen.rs apply_interfacial_flux_sources on scalar `scalar` (gather,
        C += kL a (C* - C) dt, clip, set). c_star / cell_volume: per-cell
        arrays or one value. Returns (ledger, diagnostics)."""
        led, dg = _OxygenLedger(), _OxygenDiag()
        led.cumulative_mol = float(cumulative_mol)
        cs = None if np.isscalar(c_star) else _f64(c_star, self.n)
        vol = None if np.isscalar(cell_volume) else _f64(cell_volume, self.n)
        _check(lib().lbmb_scalar_interfacial_flux(
            self.h, int(scalar), _d(cs), float(c_star) if cs is None else 0.0, _d(_f64(area_density, self.n)),
            _d(vol), float(cell_volume) if vol is None else 0.0, float(dt_s), float(kl_m_s), C.byref(led),
            C.byref(dg)))
        return ({"cumulative_mol": led.cumulative_mol, "last_step_mol": led.last_step_mol,
                 "source_integral_mol_s": led.source_integral_mol_s,
                 "active_interface_cells": led.active_interface_cells}, dg.as_dict())

    def apply_oxygen_reaction_source(self, scalar, cell_volume, dt_s, kind="constant", our=0.0, our_max=0.0, ks=0.0,
                                     c_ref=0.0, specific_our=0.0, cell_density=None, cumulative_kmol=0.0):
        """reaction.rs apply_oxygen_reaction_source on scalar `scalar`
        (gather, C -= OUR(C) dt, clip, set). Returns (ledger, diagnostics)."""
        m = _OurModel(OUR_KIND[kind], float(our), float(our_max), float(ks), float(c_ref), float(specific_our))
        led, dg = _OurLedger(), _OxygenDiag()
        led.cumulative_kmol_consumed = float(cumulative_kmol)
        vol = None if np.isscalar(cell_volume) else _f64(cell_volume, self.n)
        dens = None if cell_density is None else _f64(cell_density, self.n)
        _check(lib().lbmb_scalar_oxygen_uptake(self.h, int(scalar), C.byref(m), _d(dens), _d(vol),
                                               float(cell_volume) if vol is None else 0.0, float(dt_s),
                                               C.byref(led), C.byref(dg)))
        return ({"cumulative_kmol_consumed": led.cumulative_kmol_consumed,
                 "last_step_kmol_consumed": led.last_step_kmol_consumed}, dg.as_dict())

    # --- shear-rate and stress QOIs ---------------------------------------
    def strain_rate(self):
        """Native strain rate (n x 6: xx yy zz xy xz yz) and shear rate
        sqrt(2 S:S) per cell in lattice units (Solver::gather_strain_rate /
        gather_shear_rate, solver.rs:5464-5599)."""
        s6, g = np.empty(6 * self.n), np.empty(self.n)
        _check(lib().lbmb_gather_strain_rate(self.h, _d(s6), _d(g)))
        return s6.reshape(self.n, 6), g

    def stress_field(self, dx_m, dt_s, mu_pa_s):
        """stress.rs compute_stress_field on the SI velocity (u x dx/dt):
        strain-rate tensor (n x 6), gamma_dot [1/s], viscous stress [Pa]."""
        s6, g, v = np.empty(6 * self.n), np.empty(self.n), np.empty(self.n)
        _check(lib().lbmb_stress_field(self.h, float(dx_m), float(dt_s), float(mu_pa_s), _d(s6), _d(g), _d(v)))
        return {"s": s6.reshape(self.n, 6), "gamma_dot": g, "viscous_stress": v}

    def stress_summary(self, dx_m, dt_s, mu_pa_s, gamma_threshold=0.0, tau_threshold=0.0):
        """Percentile summaries of gamma_dot and viscous stress over the fluid
        cells (runner.rs:1648-1690; thresholds None for none). Returns
        (gamma, viscous, device_ms); a summary is None without fluid values."""
        pg, pt, ms = _Percentiles(), _Percentiles(), C.c_double()
        tg = float("nan") if gamma_threshold is None else float(gamma_threshold)
        tt = float("nan") if tau_threshold is None else float(tau_threshold)
        _check(lib().lbmb_stress_summary(self.h, float(dx_m), float(dt_s), float(mu_pa_s), tg, tt, C.byref(pg),
                                         C.byref(pt), C.byref(ms)))
        return pg.as_dict(), pt.as_dict(), ms.value

    def wall_shear_proxy(self, dx_m, dt_s, rho_kg_m3, mu_pa_s):
        """stress.rs wall_shear_proxy: wall-adjacent fluid cells in cell order
        with tau_w [Pa], y+, |u_parallel| [m/s] and the unit wall normal."""
        cnt = C.c_int64()
        _check(lib().lbmb_wall_shear_proxy(self.h, float(dx_m), float(dt_s), float(rho_kg_m3), float(mu_pa_s),
                                           None, 0, C.byref(cnt)))
        k = cnt.value
        buf = (_WallShear * max(k, 1))()
        _check(lib().lbmb_wall_shear_proxy(self.h, float(dx_m), float(dt_s), float(rho_kg_m3), float(mu_pa_s),
                                           buf, k, C.byref(cnt)))
        a = np.ctypeslib.as_array(buf)[:k] if k else None
        if k == 0:
            return {"cell_index": np.zeros(0, np.int64), "tau_w": np.zeros(0), "y_plus": np.zeros(0),
                    "u_parallel": np.zeros(0), "normal": np.zeros((0, 3))}
        return {"cell_index": a["cell_index"].copy(), "tau_w": a["tau_w_pa"].copy(), "y_plus": a["y_plus"].copy(),
                "u_parallel": a["u_parallel_m_s"].copy(), "normal": np.array(a["normal"]).reshape(k, 3)}

    def clear_body_force_field(self):
        _check(lib().lbmb_clear_body_force_field(self.h))

    def force_field(self):
        out = np.empty(3 * self.n)
        _check(lib().lbmb_get_force_field(self.h, _d(out)))
        return out.reshape(self.n, 3)

    def set_body(self, slot, body: RotatingBody):
        _check(lib().lbmb_ibm_set_body(self.h, int(slot), _d(body.positions), _d(body.weights),
                                       body.weights.size, _d(body.center), _d(body.omega)))
        self._bodies[slot] = body

    def _slot_for(self, body):
        for k, b in self._bodies.items():
            if b is body:
                return k
        slot = len(self._bodies)
        self.set_body(slot, body)
        return slot

    def apply_rotating_ibm(self, body: RotatingBody, cfg: DirectForcingConfig = None) -> IbmDiagnostics:
        cfg = cfg or DirectForcingConfig()
        d = _IbmDiag()
        _check(lib().lbmb_apply_rotating_ibm(self.h, self._slot_for(body), C.byref(cfg._c()), C.byref(d)))
        return IbmDiagnostics(d.iterations, d.slip_max, d.slip_rms, d.slip_max_rel, d.slip_rms_rel,
                              np.array(d.torque[:]), np.array(d.fluid_force[:]), np.array(d.marker_force[:]),
                              d.momentum_error_rel)

    def runner_step(self, slot, body: RotatingBody, cfg: DirectForcingConfig = None) -> IbmDiagnostics:
        """One iteration of the runner loop (runner.rs:1080-1085) with this
        marker set in body slot `slot`: clear the force field, upload the
        markers, apply the direct forcing, step; the IBM runs beside the
        full-grid sweep, and the call returns once the diagnostics are on the
        host (the sweep may still run, as after run())."""
        cfg = cfg or DirectForcingConfig()
        # the host arrays' pointers are kept while the caller passes the same
        # arrays (a runner loop passes one marker set every step; their
        # contents are read at each call)
        arrays = (body.positions, body.weights, body.center, body.omega)
        c = self._runner_args
        if c is None or c[0] != int(slot) or any(a is not b for a, b in zip(c[1], arrays)):
            pos = np.ascontiguousarray(body.positions, dtype=np.float64)
            w = np.ascontiguousarray(body.weights, dtype=np.float64)
            ctr = np.ascontiguousarray(body.center, dtype=np.float64)
            om = np.ascontiguousarray(body.omega, dtype=np.float64)
            c = (int(slot), arrays, (pos, w, ctr, om), (_d(pos), _d(w), int(w.size), _d(ctr), _d(om)), _IbmDiag())
            self._runner_args = c
        ptr, d = c[3], c[4]
        _check(lib().lbmb_runner_step(self.h, int(slot), ptr[0], ptr[1], ptr[2], ptr[3], ptr[4], C.byref(cfg._c()),
                                      C.byref(d)))
        self._bodies[int(slot)] = body
        return IbmDiagnostics(d.iterations, d.slip_max, d.slip_rms, d.slip_max_rel, d.slip_rms_rel,
                              np.array(d.torque[:]), np.array(d.fluid_force[:]), np.array(d.marker_force[:]),
                              d.momentum_error_rel)

    def run_impeller(self, body: RotatingBody, steps, cfg: DirectForcingConfig = None, scalar=-1,
                     probe_every=1):
        """Runner hot loop (runner.rs:1079-1129) on the device. The f64 total
        mass is checked after every 1000th step; a non-finite value stops the
        run with status "diverged" (runner.rs:1125-1128), and the series
        after the executed steps read NaN."""
        cfg = cfg or DirectForcingConfig()
        torque = np.empty(steps)
        ff = np.empty(3 * steps)
        iters = np.empty(steps, dtype=np.int32)
        cv = np.full(steps, np.nan) if scalar >= 0 else None
        rc = lib().lbmb_run_impeller(self.h, self._slot_for(body), C.byref(cfg._c()), int(steps), int(scalar),
                                     int(probe_every), _d(torque), _d(ff), _d(cv), iters.ctypes.data_as(_i32p))
        if rc != ERR_DIVERGED:
            _check(rc)
        executed = C.c_int64()
        diverged = C.c_int32()
        _check(lib().lbmb_run_impeller_status(self.h, C.byref(executed), C.byref(diverged)))
        return {"torque_lu": torque, "fluid_force": ff.reshape(steps, 3), "ibm_iterations": iters, "cv": cv,
                "executed": executed.value, "status": "diverged" if diverged.value else "completed"}

    def adjoint_torque(self, body: RotatingBody, steps, window_begin=None, checkpoint_every=100,
                       cfg: DirectForcingConfig = None):
        """Gradient of J = mean torque over steps [window_begin, steps) of the
        runner loop (fixed IBM sweep count) w.r.t. nu, Omega_z and the marker
        positions, by the discrete adjoint with checkpointed recomputation."""
        cfg = cfg or DirectForcingConfig()
        if window_begin is None:
            window_begin = steps // 2
        slot = self._slot_for(body)
        nm = int(np.asarray(body.weights).size)
        ac = _AdjointConfig(int(steps), int(window_begin), int(checkpoint_every), int(slot))
        r = _AdjointResult()
        dpos = np.zeros(3 * max(nm, 1))
        tq = np.zeros(int(steps))
        _check(lib().lbmb_adjoint_torque(self.h, C.byref(cfg._c()), C.byref(ac), C.byref(r), _d(dpos), _d(tq)))
        return {"J": r.J, "dJ_dnu": r.dJ_dnu, "dJ_domega_z": r.dJ_domega_z, "dJ_domega_plus": r.dJ_domega_plus,
                "dJ_domega_minus": r.dJ_domega_minus, "dJ_dpos": dpos[:3 * nm].reshape(nm, 3), "torque": tq,
                "forward_ms": r.forward_ms, "adjoint_ms": r.adjoint_ms}

    # --- checkpoint/restart ---------------------------------------------------
    @property
    def time(self):
        """Solver::time: hydro steps taken since creation (or restored)."""
        t = C.c_uint64()
        _check(lib().lbmb_get_time(self.h, C.byref(t)))
        return t.value

    def save(self, directory):
        """Solver::save (solver.rs:4715-4724): manifest.json plus
        rank_0000_part_0000.bin in the reference's v3 format."""
        _check(lib().lbmb_checkpoint_save(self.h, os.fsencode(directory)))

    def restore(self, directory):
        """Solver::restore (solver.rs:4739-4742): CheckpointError with the
        reference's code on any mismatch, before anything is installed."""
        _check(lib().lbmb_checkpoint_restore(self.h, os.fsencode(directory)))

    @classmethod
    def load(cls, directory, dims, **kw):
        """Solver::load (solver.rs:4726-4737): build from the spec, restore."""
        s = cls(dims, **kw)
        s.restore(directory)
        return s

    def set_scalar_name(self, k, name):
        _check(lib().lbmb_set_scalar_name(self.h, int(k), name.encode()))

    @property
    def qoi_checkpoint_state(self):
        """QoiCheckpointState carried through checkpoints (JSON text or None)."""
        n = C.c_int64()
        _check(lib().lbmb_get_qoi_checkpoint_state(self.h, None, 0, C.byref(n)))
        if n.value < 0:
            return None
        buf = C.create_string_buffer(n.value + 1)
        _check(lib().lbmb_get_qoi_checkpoint_state(self.h, buf, n.value, C.byref(n)))
        return buf.raw[:n.value].decode()

    @qoi_checkpoint_state.setter
    def qoi_checkpoint_state(self, text):
        if text is None:
            _check(lib().lbmb_set_qoi_checkpoint_state(self.h, None, 0))
        else:
            b = text.encode()
            _check(lib().lbmb_set_qoi_checkpoint_state(self.h, b, len(b)))

    # --- passive scalar -----------------------------------------------------
    def enable_scalar_distribution(self, diffusivity, q=None, name=None):
        k = C.c_int32()
        _check(lib().lbmb_enable_scalar(self.h, int(self.q if q is None else q), float(diffusivity),
                                        C.byref(k)))
        if name is not None:
            self.set_scalar_name(k.value, name)
        return k.value

    def set_scalar_concentration(self, k, values):
        _check(lib().lbmb_set_scalar_concentration(self.h, int(k), _d(_f64(values, self.n))))

    def gather_scalar_concentration(self, k):
        out = np.empty(self.n)
        _check(lib().lbmb_gather_scalar_concentration(self.h, int(k), _d(out)))
        return out

    def scalar_cv(self, k):
        v = C.c_double()
        _check(lib().lbmb_scalar_cv(self.h, int(k), C.byref(v)))
        return None if np.isnan(v.value) else v.value


class Batch:
    """Solvers of one lattice/storage type advanced in lockstep by batched
    kernels (one launch per kernel family per step for every case); each case
    runs the runner step of its own rotating body (lbmb_batch_*)."""

    def __init__(self, solvers, bodies, cfg: DirectForcingConfig = None):
        cfg = cfg or DirectForcingConfig()
        self.solvers = list(solvers)
        self.n = len(self.solvers)
        slots = np.array([s._slot_for(b) for s, b in zip(self.solvers, bodies)], dtype=np.int32)
        hs = (C.c_void_p * self.n)(*[s.h.value for s in self.solvers])
        h = C.c_void_p()
        _check(lib().lbmb_batch_create(C.cast(hs, C.POINTER(C.c_void_p)), slots.ctypes.data_as(_i32p), self.n,
                                       C.byref(cfg._c()), C.byref(h)))
        self.h = h
        self._lib = lib()

    def autotune(self, steps_per_trial=6):
        e, o, ms = C.c_int32(), C.c_int32(), C.c_double()
        _check(lib().lbmb_batch_autotune(self.h, int(steps_per_trial), C.byref(e), C.byref(o), C.byref(ms)))
        return {"even_blocks_per_sm": e.value, "odd_blocks_per_sm": o.value, "best_ms_per_step": ms.value}

    def run(self, steps):
        """Advance every case; returns (torque_lu [ncases x steps], device ms)."""
        tq = np.empty((self.n, max(int(steps), 1)))
        ms = C.c_double()
        _check(lib().lbmb_batch_run(self.h, int(steps), _d(tq), C.byref(ms)))
        return tq[:, :int(steps)], ms.value

    def close(self):
        if getattr(self, "h", None):
            (getattr(self, "_lib", None) or lib()).lbmb_batch_destroy(self.h)
            self.h = None

    def __del__(self):
        self.close()


def mixing_time_from_cv(times, cv):
    """Mixing times from a CV series (crates/lbm-core/src/qoi.rs:534-556):
    CV0 = the first finite positive value; t95 / t99 = the first time with
    CV <= 0.05 / 0.01 CV0 (None when never reached). Returns None when no
    finite positive CV exists."""
    times = np.asarray(times, dtype=np.float64)
    cv = np.asarray(cv, dtype=np.float64)
    ok = np.isfinite(cv) & (cv > 0.0)
    if not ok.any():
        return None
    cv0 = float(cv[np.argmax(ok)])
    fin = np.isfinite(cv)
    hit95 = fin & (cv <= 0.05 * cv0)
    hit99 = fin & (cv <= 0.01 * cv0)
    return {"cv0": cv0, "t95": float(times[np.argmax(hit95)]) if hit95.any() else None,
            "t99": float(times[np.argmax(hit99)]) if hit99.any() else None}


def power_qois(torque_n_m, omega_rad_s, rho_kg_m3, impeller_diameter_m, working_volume_m3):
    """qoi::power_qois (crates/lbm-core/src/qoi.rs:477-505)."""
    r = _PowerResult()
    _check(lib().lbmb_power_qois(float(torque_n_m), float(omega_rad_s), float(rho_kg_m3),
                                 float(impeller_diameter_m), float(working_volume_m3), C.byref(r)))
    return r.as_dict()


def power_from_torque_series(torque_lu, run_steps, probe_every, rho_kg_m3, dx_m, dt_s, omega_rad_s,
                             impeller_diameter_m, working_volume_m3, executed=None):
    """The runner's power QOIs (crates/lbm-cli/src/runner.rs:1396-1425,
    1514-1543) from the per-step lattice torque series of run_impeller:
    records at probe steps, SI torque, mean over the last half of the run."""
    t = _f64(torque_lu)
    executed = t.size if executed is None else int(executed)
    r = _PowerResult()
    used = C.c_int64()
    _check(lib().lbmb_power_from_torque_series(_d(t), executed, int(run_steps), int(probe_every), float(rho_kg_m3),
                                               float(dx_m), float(dt_s), float(omega_rad_s),
                                               float(impeller_diameter_m), float(working_volume_m3), C.byref(r),
                                               C.byref(used)))
    out = r.as_dict()
    out["records_used"] = used.value
    return out


def unit_report(vessel_diameter_m, liquid_height_m, impeller_diameter_m, rotational_speed_rpm, liquid_density_kg_m3,
                liquid_viscosity_pa_s, dt_s, grid, scalar_diffusivity_m2_s=None, checked=True):
    """bioprocess_unit_report (crates/lbm-scenario/src/units.rs:96-325),
    single-phase subset. checked=True raises UnsupportedError when a
    rejection fires (compute_unit_report); False returns the report with its
    rejections (unit_report_with_diagnostics)."""
    i = _UnitInput(float(vessel_diameter_m), float(liquid_height_m), float(impeller_diameter_m),
                   float(rotational_speed_rpm), float(liquid_density_kg_m3), float(liquid_viscosity_pa_s), float(dt_s),
                   (C.c_int32 * 3)(*[int(g) for g in grid]),
                   float(scalar_diffusivity_m2_s) if scalar_diffusivity_m2_s else 0.0)
    m = _UnitMapping()
    rc = lib().lbmb_unit_report(C.byref(i), C.byref(m))
    if rc != ERR_UNSUPPORTED or checked:
        _check(rc)
    out = {k: getattr(m, k) for k, _ in _UnitMapping._fields_ if k not in ("warnings", "rejections")}
    out["warnings"] = [v for b, v in UNIT_ISSUES.items() if m.warnings & b]
    out["rejections"] = [v for b, v in UNIT_ISSUES.items() if m.rejections & b]
    return out


def scalar_top_hat_pulse(dims, solid, dx_m, center_m, radius_m, concentration=1.0):
    """scalar_initial_condition, pulse branch (crates/lbm-cli/src/runner.rs:
    1317-1377): `concentration` on fluid cells within radius_m of center_m."""
    dims = [int(d) for d in dims]
    n = dims[0] * dims[1] * dims[2]
    so = None if solid is None else np.ascontiguousarray(solid, dtype=np.uint8).ravel()
    out = np.empty(n)
    _check(lib().lbmb_scalar_top_hat_pulse((C.c_int32 * 3)(*dims), None if so is None else so.ctypes.data_as(_u8p),
                                           float(dx_m), _d(_f64(center_m, 3)), float(radius_m), float(concentration),
                                           _d(out)))
    return out


def scalar_diffusivity_lu(diffusivity_m2_s, dt_s, dx_m):
    """D dt / dx^2 (crates/lbm-cli/src/runner.rs:1371-1375)."""
    v = C.c_double()
    _check(lib().lbmb_scalar_diffusivity_lu(float(diffusivity_m2_s), float(dt_s), float(dx_m), C.byref(v)))
    return v.value


def capabilities(solver=None):
    """The Backend trait's capability hooks (crates/lbm-core/src/backend.rs:
    162-199, 343-345) for this backend (and a solver's configuration)."""
    c = _BackendCaps()
    _check(lib().lbmb_capabilities(None if solver is None else solver.h, C.byref(c)))
    return {k: getattr(c, k) for k, _ in _BackendCaps._fields_}


def gaussian_pulse(dims, solid, center, sigma):
    """Concentration exp(-r^2 / (2 sigma^2)) around `center` (cell
    coordinates) on the fluid cells, zero on solids."""
    nx, ny, nz = dims
    z, y, x = np.meshgrid(np.arange(nz), np.arange(ny), np.arange(nx), indexing="ij")
    r2 = (x - center[0]) ** 2 + (y - center[1]) ** 2 + (z - center[2]) ** 2
    c = np.exp(-r2.ravel() / (2.0 * sigma * sigma))
    c[np.asarray(solid).ravel() != 0] = 0.0
    return c


def build_wall_rims(dims, is_wall, wall_u):
    dims = [int(d) for d in dims]
    n = dims[0] * dims[1] * dims[2]
    solid = np.empty(n, dtype=np.uint8)
    wu = np.empty(3 * n)
    u = _f64(wall_u, 18)
    _check(lib().lbmb_build_wall_rims((C.c_int32 * 3)(*dims), (C.c_int32 * 6)(*[int(bool(w)) for w in is_wall]),
                                      _d(u), solid.ctypes.data_as(_u8p), _d(wu)))
    return solid, wu.reshape(n, 3)


@dataclass
class TankSpec:
    """Stirred-tank set-up in SI units (geometry.rs:84-132)."""
    dims: tuple
    dx_m: float
    vessel_diameter_m: float
    liquid_height_m: float
    impeller_diameter_m: float
    clearance_m: float
    omega_rad_s: float
    blade_count: int = 6
    impeller: str = "rushton"
    baffle_count: int = 0
    baffle_width_m: float = 0.0
    baffle_thickness_m: float = 0.0
    marker_spacing_cells: float = 0.7
    min_cells: float = 32.0

    def _c(self):
        return _TankSpec((C.c_int32 * 3)(*self.dims), self.dx_m, self.vessel_diameter_m, self.liquid_height_m,
                         self.baffle_count, self.baffle_width_m, self.baffle_thickness_m,
                         IMPELLER[self.impeller], self.impeller_diameter_m, self.clearance_m, self.blade_count,
                         self.omega_rad_s, self.marker_spacing_cells, self.min_cells)


def build_stirred_tank(spec: TankSpec):
    L = lib()
    c = spec._c()
    n = spec.dims[0] * spec.dims[1] * spec.dims[2]
    m = C.c_int64()
    _check(L.lbmb_build_stirred_tank(C.byref(c), None, None, None, None, None, 0, C.byref(m), None, None))
    solid = np.empty(n, dtype=np.uint8)
    baffle = np.empty(n, dtype=np.uint8)
    wv = np.empty(3 * n)
    pos = np.empty(3 * m.value)
    w = np.empty(m.value)
    center = np.empty(3)
    omega = np.empty(3)
    _check(L.lbmb_build_stirred_tank(C.byref(c), solid.ctypes.data_as(_u8p), baffle.ctypes.data_as(_u8p),
                                     _d(wv), _d(pos), _d(w), m.value, C.byref(m), _d(center), _d(omega)))
    return {"solid": solid, "baffle": baffle, "wall_velocity": wv.reshape(n, 3),
            "marker_pos": pos.reshape(-1, 3), "marker_w": w, "center": center, "omega": omega}


# ---------------------------------------------------------------------------
# Checkpoint format on host arrays (no device): the reference's
# write_part_checkpoint / read_rank_file for one part.
# ---------------------------------------------------------------------------
def _ckpt_spec(spec):
    dims = tuple(int(d) for d in spec["dims"])
    nu = float(spec.get("nu", 1.0 / 6.0))
    om = spec.get("omega_shear")
    return _CkptSpec(int(spec.get("lattice", 19)), COLLISION[spec.get("collision", "trt")],
                     64 if spec.get("dtype", "f64") == "f64" else 32, (C.c_int32 * 3)(*dims),
                     (C.c_int32 * 3)(*[int(bool(p)) for p in spec.get("periodic", (False, False, False))]), nu,
                     float(spec.get("magic", MAGIC_STD)), float(1.0 / (3.0 * nu + 0.5) if om is None else om),
                     (C.c_double * 3)(*[float(f) for f in spec.get("force", (0.0, 0.0, 0.0))])), dims


def _masks(n, solid, wall_u):
    s = None if solid is None else np.ascontiguousarray(solid, dtype=np.uint8).ravel()
    w = None if wall_u is None else _f64(wall_u, 3 * n)
    return s, w


def checkpoint_write_host(directory, spec, state, solid=None, wall_u=None):
    """Write a checkpoint from host arrays. spec: dims, lattice, collision,
    dtype ("f32" | "f64"), nu, magic, omega_shear, periodic, force. state:
    step, f (Q x n), moments (4 x n), force_field (n x 3 or None), scalars
    (list of dicts name, diffusivity, q, h (q x n), conc), qoi (JSON text or
    None)."""
    cs, dims = _ckpt_spec(spec)
    n = dims[0] * dims[1] * dims[2]
    q = cs.lattice
    f = _f64(state["f"], q * n)
    mo = _f64(state["moments"], 4 * n)
    ff = state.get("force_field")
    ff = None if ff is None else _f64(ff, 3 * n)
    scal = state.get("scalars") or []
    keep = []
    arr = (_CkptScalar * max(len(scal), 1))()
    for i, x in enumerate(scal):
        h = _f64(x["h"], int(x["q"]) * n)
        c = _f64(x["conc"], n)
        keep += [h, c]
        arr[i].name = x["name"].encode()
        arr[i].diffusivity = float(x["diffusivity"])
        arr[i].q = int(x["q"])
        arr[i].h = _d(h)
        arr[i].h_capacity = h.size
        arr[i].conc = _d(c)
    qoi = state.get("qoi")
    qb = None if qoi is None else C.create_string_buffer(qoi.encode(), len(qoi.encode()))
    data = _CkptData(int(state.get("step", 0)), _d(f), _d(mo), int(ff is not None), _d(ff), len(scal), len(scal),
                     arr, int(qoi is not None), None if qb is None else C.cast(qb, C.POINTER(C.c_char)),
                     0 if qoi is None else len(qoi.encode()), 0 if qoi is None else len(qoi.encode()))
    s, w = _masks(n, solid, wall_u)
    _check(lib().lbmb_checkpoint_write_host(os.fsencode(directory), C.byref(cs),
                                            None if s is None else s.ctypes.data_as(_u8p), _d(w), C.byref(data)))


def checkpoint_read_host(directory, spec, solid=None, wall_u=None, max_scalars=2, max_qoi_bytes=1 << 20):
    """Read and validate a checkpoint against spec and masks; returns the
    state dict of checkpoint_write_host. CheckpointError on any mismatch
    (including more scalar distributions than max_scalars)."""
    cs, dims = _ckpt_spec(spec)
    n = dims[0] * dims[1] * dims[2]
    q = cs.lattice
    f = np.zeros(q * n)
    mo = np.zeros(4 * n)
    ff = np.zeros(3 * n)
    hs = [np.zeros(max(q, 7) * n) for _ in range(max_scalars)]
    cs_ = [np.zeros(n) for _ in range(max_scalars)]
    arr = (_CkptScalar * max_scalars)()
    for i in range(max_scalars):
        arr[i].h = _d(hs[i])
        arr[i].h_capacity = hs[i].size
        arr[i].conc = _d(cs_[i])
    qb = C.create_string_buffer(max_qoi_bytes)
    data = _CkptData(0, _d(f), _d(mo), 0, _d(ff), 0, max_scalars, arr, 0, C.cast(qb, C.POINTER(C.c_char)), 0,
                     max_qoi_bytes)
    s, w = _masks(n, solid, wall_u)
    _check(lib().lbmb_checkpoint_read_host(os.fsencode(directory), C.byref(cs),
                                           None if s is None else s.ctypes.data_as(_u8p), _d(w), C.byref(data)))
    return {"step": data.step, "f": f.reshape(q, n), "moments": mo.reshape(4, n),
            "force_field": ff.reshape(n, 3) if data.has_force_field else None,
            "scalars": [{"name": arr[i].name.decode(), "diffusivity": arr[i].diffusivity, "q": arr[i].q,
                         "h": hs[i][:arr[i].q * n].reshape(arr[i].q, n).copy(), "conc": cs_[i].copy()}
                        for i in range(data.n_scalars)],
            "qoi": qb.raw[:data.qoi_len].decode() if data.has_qoi else None}


def fnv1a64(data):
    """FNV-1a 64 of bytes (the checkpoint payload hash)."""
    b = bytes(data)
    return int(lib().lbmb_fnv1a64(b, len(b)))
