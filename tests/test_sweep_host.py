"""Host logic of the sweep: case expansion, aggregation, seeded cases, LPT
sharding and the rank-0 gather (world_size 2 over gloo on the CPU)."""
import os
import socket

import pytest

from lbmflow_b200 import sweep


def test_expand_grid_order_matches_reference():
    # crates/lbm-scenario/src/sweep.rs grid_sweep_expands_expected_cases
    cases = sweep.expand_grid([("operation.duration_s", [1.0, 2.0]), ("run.dt_s", [0.1, 0.2, 0.3])])
    assert len(cases) == 6
    assert cases[0][0][1] == 1.0
    assert cases[5][1][1] == 0.3
    assert [c[1][1] for c in cases[:3]] == [0.1, 0.2, 0.3]  # last parameter varies fastest


def test_aggregate_matches_reference_roundtrip():
    # crates/lbm-cli/src/sweep.rs aggregation_roundtrip: two bundles 2.0 / 4.0
    agg = sweep.aggregate([{"power.power_w": 2.0}, {"power.power_w": 4.0}])
    assert agg["power.power_w"] == {"count": 2, "min": 2.0, "mean": 3.0, "max": 4.0}
    agg = sweep.aggregate([{"Np": 1.0}, None, {"Np": float("nan")}])
    assert agg["Np"]["count"] == 1


def test_seeded_cases_reproducible_and_in_range():
    a = sweep.seeded_cases()
    b = sweep.seeded_cases()
    assert len(a) == 64
    assert [(c.T, c.u_tip, c.re) for c in a] == [(c.T, c.u_tip, c.re) for c in b]
    for c in a:
        assert 48 <= c.T <= 128 and 0.02 <= c.u_tip <= 0.06 and 500 <= c.re <= 5000
        assert c.dims == (c.T, c.T, int(round(1.25 * c.T)))
        # Re = N D^2 / nu with N = Omega / 2 pi and Omega = u_tip / (D / 2)
        assert abs((c.omega / (2 * 3.141592653589793)) * c.D ** 2 / c.nu - c.re) < 1e-9 * c.re
    assert len({c.T for c in a}) > 20


def test_lpt_assign_covers_every_case_once_and_balances():
    cases = sweep.seeded_cases()
    for world in (1, 2, 3, 8):
        parts = sweep.lpt_assign(cases, world, steps=5000)
        flat = sorted(i for p in parts for i in p)
        assert flat == list(range(len(cases)))
        loads = [sum(cases[i].cells for i in p) for p in parts]
        assert max(loads) - min(loads) <= max(c.cells for c in cases)


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _rank_main(rank, world, port, q):
    import torch.distributed as dist

    from lbmflow_b200 import sweep as sw
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)

    def fake_run(cases, steps, **kw):
        # stands in for the device runner: deterministic per-case values
        per = [{"index": c.index, "T": c.T, "u_tip": c.u_tip, "re": c.re, "Np": 1.0 + c.index} for c in cases]
        return {"per_case": per, "device_ms": 10.0 * (rank + 1), "cells": sum(c.cells for c in cases)}

    sw.run_sweep = fake_run

    def gather(obj):
        out = [None] * world
        dist.all_gather_object(out, obj)
        return out

    cases = sw.seeded_cases(n=10)
    res = sw.run_sharded(cases, 100, rank, world, gather)
    q.put((rank, res))
    dist.barrier()
    dist.destroy_process_group()


def test_run_sharded_gathers_every_case_on_rank0():
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    out = dict(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert out[1] is None
    res = out[0]
    assert [d["index"] for d in res["per_case"]] == list(range(10))
    assert [d["Np"] for d in res["per_case"]] == [1.0 + i for i in range(10)]
    assert res["device_ms_max"] == 20.0  # max over ranks
    assert res["aggregate"]["Np"]["count"] == 10
