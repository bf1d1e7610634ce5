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
