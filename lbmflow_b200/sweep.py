"""Stirred-tank parameter sweeps on the batched device runner.

Mirrors the reference sweep driver: cartesian case expansion
(crates/lbm-scenario/src/sweep.rs:52-71 ``expand_grid``), one runner per case
(crates/lbm-cli/src/sweep.rs:47-106 ``run`` / ``run_case``) and the per-QOI
count/min/mean/max summary (sweep.rs:142-175 ``aggregate_qoi_bundles``).
Where the reference runs the cases one after another, ``run_sweep`` advances
all of them in lockstep with ``Batch`` (one launch per kernel family per step
for every case); ``mode="sequential"`` keeps the reference's one-case-at-a-time
order on the device for comparison. Across GPUs the cases are independent:
``lpt_assign`` shards them by longest-processing-time on cells x steps and
``run_sharded`` gathers the per-case results on rank 0, with no collective on
the data path.
"""
from __future__ import annotations

import itertools
import math
from dataclasses import dataclass, field

import numpy as np

SEED = 0x5EED


def expand_grid(params):
    """Cartesian product in the reference's order: the first parameter varies
    slowest (each parameter multiplies the case list built so far,
    sweep.rs:52-71). ``params`` is a list of (parameter_path, values)."""
    cases = [[]]
    for path, values in params:
        cases = [c + [(path, float(v))] for c in cases for v in values]
    return cases


def aggregate(values_per_case):
    """count/min/mean/max per QOI key over the cases that produced it
    (sweep.rs:142-175); NaN results are dropped like failed cases."""
    keys = sorted({k for v in values_per_case if v for k in v})
    out = {}
    for k in keys:
        xs = [v[k] for v in values_per_case if v and k in v and np.isfinite(v[k])]
        if xs:
            out[k] = {"count": len(xs), "min": min(xs), "mean": sum(xs) / len(xs), "max": max(xs)}
    return out


@dataclass
class TankCase:
    """One tank of the sweep: diameter T cells (grid T x T x round(1.25 T)),
    six-blade flat-blade turbine D = T/3 at clearance T/3, four baffles of
    width T/10, tip speed u_tip (lattice units) and impeller Reynolds number."""
    T: int
    u_tip: float
    re: float
    index: int = 0
    dims: tuple = field(init=False)
    D: float = field(init=False)
    omega: float = field(init=False)
    nu: float = field(init=False)

    def __post_init__(self):
        self.dims = (int(self.T), int(self.T), int(round(1.25 * self.T)))
        self.D = self.T / 3.0
        self.omega = self.u_tip / (0.5 * self.D)  # rad/step
        self.nu = (self.omega / (2.0 * math.pi)) * self.D ** 2 / self.re

    @property
    def cells(self):
        return self.dims[0] * self.dims[1] * self.dims[2]


def seeded_cases(n=64, seed=SEED, t_range=(48, 128), u_tip_range=(0.02, 0.06), re_range=(500.0, 5000.0)):
    """n tanks with T ~ U{t_range} (integers, inclusive), u_tip ~ U(u_tip_range)
    and Re ~ U(re_range), drawn in that order per case from numpy's
    default_rng(seed)."""
    rng = np.random.default_rng(seed)
    out = []
    for i in range(n):
        T = int(rng.integers(t_range[0], t_range[1] + 1))
        u = float(rng.uniform(*u_tip_range))
        re = float(rng.uniform(*re_range))
        out.append(TankCase(T, u, re, index=i))
    return out


def tank_geometry(T, H_over_T=1.25, spacing=0.7, min_cells=6.0):
    """Voxel flags and impeller markers of a T-cell tank (1 m vessel, dx =
    1/T): flat bottom, solid lid, four baffles of width 0.1 m and thickness
    2.6 cells at T = 128 (scaled with T, at least one cell), flat-blade
    turbine D = T/3 at clearance T/3 sampled at ``spacing`` cells. The
    sweep's smallest tanks (T = 48, D = 16 cells) are below the geometry
    builder's default resolution floor (32 cells), so the floor is lowered
    to ``min_cells``."""
    import lbmflow_b200 as lb
    nz = int(round(H_over_T * T))
    dx = 1.0 / T
    spec = lb.TankSpec(dims=(T, T, nz), dx_m=dx, vessel_diameter_m=1.0, liquid_height_m=nz * dx,
                       impeller_diameter_m=1.0 / 3.0, clearance_m=1.0 / 3.0, omega_rad_s=1.0,
                       impeller="flat_blade", marker_spacing_cells=spacing, baffle_count=4,
                       baffle_width_m=0.1, baffle_thickness_m=max(2.6 * T / 128.0, 1.0) * dx,
                       min_cells=min_cells)
    return lb.build_stirred_tank(spec)


def build_case(case: TankCase, storage="f32", lattice=19, collision="trt", les_cs=0.1, device=0):
    """Solver + rotating body of one sweep case."""
    import lbmflow_b200 as lb
    geo = tank_geometry(case.T)
    body = lb.RotatingBody(geo["center"], [0.0, 0.0, case.omega], geo["marker_pos"], geo["marker_w"])
    g = lb.Solver(case.dims, lattice=lattice, collision=collision, storage=storage, nu=case.nu,
                  solid=geo["solid"], device=device, smagorinsky_cs=les_cs)
    return g, body


def power_number(torque_lu, omega, D):
    """Np from the last-half mean torque (runner.rs:1523-1530, qoi.rs:477-505),
    lattice units with rho = 1."""
    t = np.asarray(torque_lu)
    tq = float(np.mean(t[t.size // 2:]))
    n_rev = omega / (2.0 * math.pi)
    return omega * tq / (n_rev ** 3 * D ** 5)


def lpt_assign(cases, world, steps=1):
    """Longest-processing-time assignment of cases to ranks on cells x steps:
    cases in decreasing cost, each to the currently least-loaded rank (ties to
    the lowest rank). Returns one list of case indices per rank."""
    load = [0.0] * world
    parts = [[] for _ in range(world)]
    order = sorted(range(len(cases)), key=lambda i: (-cases[i].cells * steps, i))
    for i in order:
        r = min(range(world), key=lambda k: (load[k], k))
        parts[r].append(i)
        load[r] += cases[i].cells * steps
    return [sorted(p) for p in parts]


def run_sweep(cases, steps, mode="batch", storage="f32", les_cs=0.1, autotune=True, device=0, warmup=0):
    """Run every case for ``steps`` runner steps. Returns per-case Np and
    torque, and the aggregate MLUPS = sum(N_i) * steps / device time."""
    import lbmflow_b200 as lb
    built = [build_case(c, storage=storage, les_cs=les_cs, device=device) for c in cases]
    solvers = [b[0] for b in built]
    bodies = [b[1] for b in built]
    total_cells = sum(c.cells for c in cases)
    res = {"mode": mode, "cases": len(cases), "cells": total_cells, "steps": steps}
    torques = []
    if mode == "batch":
        batch = lb.Batch(solvers, bodies)
        if autotune:
            res["autotune"] = batch.autotune()
        if warmup:
            batch.run(warmup)
        tq, ms = batch.run(steps)
        torques = list(tq)
        batch.close()
    else:
        ms = 0.0
        for g, b in zip(solvers, bodies):
            if autotune:
                g.autotune_sweep(6)
            if warmup:
                g.run_impeller(b, warmup)
            r = g.run_impeller(b, steps)
            ms += g.last_timing()[0]
            torques.append(r["torque_lu"])
    for g in solvers:
        g.close()
    res["device_ms"] = ms
    res["mlups"] = total_cells * steps / (ms * 1e-3) / 1e6 if ms > 0 else float("nan")
    res["per_case"] = [{"index": c.index, "T": c.T, "u_tip": c.u_tip, "re": c.re,
                        "Np": power_number(t, c.omega, c.D)} for c, t in zip(cases, torques)]
    res["aggregate"] = aggregate([{"Np": p["Np"]} for p in res["per_case"]])
    return res


def run_sharded(cases, steps, rank, world, gather, **kw):
    """This rank's LPT share of the sweep, then the per-case results of every
    rank on rank 0 via ``gather(obj) -> list`` (e.g. a torch.distributed
    all_gather_object wrapper); no collective touches the device data."""
    mine = lpt_assign(cases, world, steps)[rank]
    part = run_sweep([cases[i] for i in mine], steps, **kw) if mine else {"per_case": [], "device_ms": 0.0,
                                                                          "cells": 0}
    allp = gather({"per_case": part["per_case"], "device_ms": part["device_ms"], "cells": part["cells"]})
    if rank != 0:
        return None
    per_case = sorted(itertools.chain.from_iterable(p["per_case"] for p in allp), key=lambda d: d["index"])
    worst_ms = max(p["device_ms"] for p in allp)
    cells = sum(p["cells"] for p in allp)
    return {"per_case": per_case, "device_ms_max": worst_ms,
            "mlups": cells * steps / (worst_ms * 1e-3) / 1e6 if worst_ms > 0 else float("nan"),
            "aggregate": aggregate([{"Np": p["Np"]} for p in per_case])}
