"""The allocation-free reduction entry point, checked against lbmb_reduce.

lbmb_reduce_populations_noalloc exists for callers that cannot allocate
device memory while they run: an application that hands out every device
byte from its own arena, a process under a hard device-memory quota, or a
time-stepping loop that must not call cudaMalloc/cudaFree because those
calls can synchronize the device. Here the test (the caller) owns the
device buffers through torch; the entry point only reads them and keeps
its partial sums in the library's fixed device array.

This file is collected last so that a stopping run has executed every other
test first; it also passes alone in a fresh process.
"""
import ctypes as C

import numpy as np
import pytest

import lbmflow_b200 as lb
from cases import cavity

pytestmark = pytest.mark.gpu

MAX_CELLS = 1 << 25


def noalloc_reduce(f_dev, storage, q, ncells, plane, solid_dev, force):
    out = np.full(5, np.nan)
    g = np.ascontiguousarray(force, dtype=np.float64)
    rc = lb.lib().lbmb_reduce_populations_noalloc(
        C.c_void_p(f_dev.data_ptr()), lb.STORAGE[storage], q, ncells, plane,
        None if solid_dev is None else C.c_void_p(solid_dev.data_ptr()),
        g.ctypes.data_as(C.POINTER(C.c_double)), out.ctypes.data_as(C.POINTER(C.c_double)), None)
    return rc, out


def handle_reduce(s):
    return np.array([s.reduce(lb.RED_FLUID_CELLS), s.reduce(lb.RED_MASS_DEV)] +
                    [s.reduce(lb.RED_MOMENTUM, a) for a in range(3)])


@pytest.mark.parametrize("q,prec", [(19, "f32"), (27, "f64"), (19, "f16"), (27, "bf16")])
def test_noalloc_reduction_matches_handle_reduce(q, prec):
    import torch
    dims, solid, wall_u, nu = cavity(24, re=30.0)
    force = (1e-6, -2e-6, 5e-7)
    s = lb.Solver(dims, lattice=q, storage=prec, nu=nu, solid=solid, wall_u=wall_u, force=force)
    dtype = {"f32": torch.float32, "f64": torch.float64, "f16": torch.float16, "bf16": torch.bfloat16}[prec]
    solid_dev = torch.from_numpy(solid.astype(np.uint8)).cuda()
    for call in range(2):  # two calls in a row share the fixed scratch array
        s.run(17 + call)
        ref = handle_reduce(s)
        # stage_out is the exact f64 view of the stored values, so the cast
        # back to the storage type reproduces the device populations.
        f_dev = torch.from_numpy(s.stage_out()).to(dtype).cuda().contiguous()
        # the solver keeps the uniform force in its arithmetic precision
        # (fp32 for fp32 and 16-bit storage, fp64 for fp64), so pass the same
        # rounded value
        force_t = np.asarray(force, dtype=np.float64 if prec == "f64" else np.float32).astype(np.float64)
        rc, out = noalloc_reduce(f_dev, prec, q, s.n, s.n, solid_dev, force_t)
        assert rc == lb.OK, lb.lib().lbmb_last_error()
        assert out[0] == ref[0]
        assert np.abs(out[1:] - ref[1:]).max() < 1e-12, (out, ref)
    s.close()


def test_noalloc_rejects_oversized_grid():
    import torch
    f_dev = torch.zeros(8, dtype=torch.float32, device="cuda")
    rc, out = noalloc_reduce(f_dev, "f32", 19, MAX_CELLS + 1, MAX_CELLS + 1, None, (0.0, 0.0, 0.0))
    assert rc == lb.ERR_INVALID
    assert b"exceeds the no-alloc maximum" in lb.lib().lbmb_last_error()
    assert np.isnan(out).all()
