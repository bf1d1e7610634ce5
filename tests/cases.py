"""Shared seeded cases for the GPU-vs-oracle parity tests."""
import math

import numpy as np

# Tolerances (stated per precision; crates/lbm-core/tests/backend_simd_equiv.rs
# uses 1e-11 (f64) / 1e-6 (f32) per cell for CPU<->CPU and
# t14_backend_equiv.rs 1e-5 relative for CPU<->GPU fields).
TOL = {"f64": 1e-11, "f32": 1e-5}


def cavity(n, u_lid=0.05, re=100.0, lid_face=5):
    """3D lid-driven cavity: all walls half-way bounce-back, ZPos lid moving +x
    (crates/lbm-core/tests/t15_5_cavity3d.rs:148-182, nu = U (N-2) / Re)."""
    from oracle import oracle as o
    dims = (n, n, n)
    u = np.zeros((6, 3))
    u[lid_face] = [u_lid, 0.0, 0.0]
    solid, wall_u = o.wall_rims(dims, [True] * 6, u.ravel())
    nu = u_lid * (n - 2) / re
    return dims, solid, wall_u, nu


def tgv_fields(dims, amp=0.02, rho0=1.0):
    """Taylor-Green vortex velocity on a periodic box (lattice.rs:742-755)."""
    nx, ny, nz = dims
    z, y, x = np.meshgrid(np.arange(nz), np.arange(ny), np.arange(nx), indexing="ij")
    sx, cx = np.sin(2 * math.pi * x / nx), np.cos(2 * math.pi * x / nx)
    sy, cy = np.sin(2 * math.pi * y / ny), np.cos(2 * math.pi * y / ny)
    cz = np.cos(2 * math.pi * z / nz)
    u = np.stack([amp * sx * cy * cz, -amp * cx * sy * cz, np.zeros_like(sx)], axis=-1).reshape(-1, 3)
    rho = np.full(nx * ny * nz, rho0)
    return rho, u


def seeded_state(q, n, seed, scale=1e-3):
    """Random deviation populations around a mild flow (for staging)."""
    rng = np.random.default_rng(seed)
    return rng.normal(0.0, scale, size=(q, n))


def rel_err(a, b, mask=None):
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    if mask is not None:
        a = a[..., mask]
        b = b[..., mask]
    den = max(np.abs(b).max(), 1e-300)
    return np.abs(a - b).max() / den


PREC_BITS = {"f64": 64, "f32": 32}


class Pair:
    """GPU solver + oracle in the same precision (+ an f64 oracle for f32)."""

    def __init__(self, dims, q, prec, collision="trt", nu=0.05, periodic=(False,) * 3, force=(0, 0, 0),
                 solid=None, wall_u=None, omega_shear=None, smagorinsky_cs=0.0, sweep=None, free_slip_top=False):
        import lbmflow_b200 as lb
        from oracle import oracle as o
        if omega_shear is None:
            omega_shear = 1.0 / (3.0 * nu + 0.5)
        self.prec = prec
        kw = dict(collision=collision, nu=nu, periodic=periodic, force=force, solid=solid, wall_u=wall_u,
                  omega_shear=omega_shear, smagorinsky_cs=smagorinsky_cs, free_slip_top=free_slip_top)
        self.g = lb.Solver(dims, lattice=q, storage=prec, **kw)
        if sweep is not None:
            self.g.set_sweep_kernel(sweep)
        self.oracles = [o.OracleSolver(dims, q=q, real_bits=PREC_BITS[prec], **kw)]
        if prec == "f32":
            self.oracles.append(o.OracleSolver(dims, q=q, real_bits=64, **kw))
        self.n = self.g.n

    def init_with(self, rho, u):
        self.g.init_with(rho, u)
        for c in self.oracles:
            c.init_with(rho, u)

    def stage_in(self, f):
        self.g.stage_in(f)
        for c in self.oracles:
            c.stage_in(f)

    def run(self, steps):
        self.g.run(steps)
        for c in self.oracles:
            c.step(steps)

    def check(self, fluid):
        """f64: populations within 1e-11 of the max population, moments
        within 1e-10. f32: the GPU's distance to the f64 oracle is at most
        3x the reference f32 path's own distance to it (+1e-9): the GPU is as
        accurate as the reference CPU path in the same precision."""
        fg = self.g.stage_out()[:, fluid]
        rg, ug = self._mom(self.g.read_moments(), fluid)
        c = self.oracles[0]
        fc = c.stage_out()[:, fluid]
        rc, uc = self._mom(c.moments(), fluid)
        if self.prec == "f64":
            scale = max(np.abs(fc).max(), 1e-30)
            assert np.abs(fg - fc).max() / scale < TOL["f64"]
            assert np.abs(rg - rc).max() < 1e-10
            assert np.abs(ug - uc).max() / max(np.abs(uc).max(), 1e-30) < 1e-10
            return
        c64 = self.oracles[1]
        f64 = c64.stage_out()[:, fluid]
        r64, u64 = self._mom(c64.moments(), fluid)
        for gpu, ref, exact in ((fg, fc, f64), (rg, rc, r64), (ug, uc, u64)):
            e_gpu = np.abs(gpu - exact).max()
            e_ref = np.abs(ref - exact).max()
            assert e_gpu <= 3.0 * e_ref + 1e-9, (e_gpu, e_ref)

    @staticmethod
    def _mom(m, fluid):
        return m[0][fluid], np.stack([m[1][fluid], m[2][fluid], m[3][fluid]])
