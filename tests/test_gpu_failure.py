"""Failure detection on the device without a GPU fault.

Every mbarrier wait of the bulk-copy sweep kernels is bounded; a wait that
runs out sets a device error flag and the kernel returns, so the host reads
an error status and the context stays usable. The test makes a wait run out
on purpose: with a negative wait limit the sweep waits on a barrier that
nothing arrives at (a flag that nothing sets), for a short bounded time.
No test here faults, traps or hangs a GPU.
"""
import numpy as np
import pytest

import lbmflow_b200 as lb
from cases import cavity

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("storage", ["f32", "f16"])
def test_bounded_wait_timeout_reports_error_and_context_survives(storage):
    kind = "bulk"
    dims, solid, wall_u, nu = cavity(16, re=20.0)
    g = lb.Solver(dims, storage=storage, nu=nu, solid=solid, wall_u=wall_u)
    try:
        g.set_sweep_kernel(kind)
    except lb.UnsupportedError:
        pytest.skip(f"{kind} sweep not available for this form")
    f0 = g.stage_out()
    g.set_wait_limit(-200000)  # ~0.1 ms on a barrier nothing arrives at
    with pytest.raises(lb.LbmbError) as e:
        g.run(1)
        g.sync()
    assert "timed out" in str(e.value)
    # nothing was written by the sweep that timed out
    g.set_wait_limit(0)
    # the context is usable: a fresh solver steps and matches a direct-load run
    a = lb.Solver(dims, storage=storage, nu=nu, solid=solid, wall_u=wall_u)
    b = lb.Solver(dims, storage=storage, nu=nu, solid=solid, wall_u=wall_u)
    a.set_sweep_kernel(kind)
    b.set_sweep_kernel("direct")
    a.run(6)
    b.run(6)
    ra, rb = a.read_moments()[1], b.read_moments()[1]
    assert np.abs(ra - rb).max() <= 1e-3 * max(np.abs(rb).max(), 1e-12)
    assert np.isfinite(f0).all()
