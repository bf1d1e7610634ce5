"""Benchmark of the LBMFlow stirred-tank time step on B200.

Workload (the single-GPU tank configuration): cylindrical tank T = 128
cells on a 128 x 128 x 160 grid, flat bottom, four wall baffles of width
T/10 and thickness 2.6 cells, a six-blade flat-blade disc turbine of
diameter T/3 at clearance T/3 sampled by ~6k direct-forcing IBM markers at
0.7-cell spacing, tip speed 0.05, nu for impeller Re = 2000, D3Q27
central-moment collision, fp32 populations. One step = the reference
runner step (clear force field -> IBM direct forcing -> collide/stream/
moments), synthetic seeded geometry, quiescent start after a warm-up.

Prints one JSON line (rank 0). `--impl reference` times the reference's CPU
path (the C++ restatement in oracle/, the reference being Rust that cannot
be built here) on the host cores instead.
"""
from __future__ import annotations

import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

PEAKS_FILE = os.path.join(ROOT, "MEASURED_PEAKS.json")
FALLBACK_HBM_GBS = 6650.0


# ---------------------------------------------------------------------------
# Workload
# ---------------------------------------------------------------------------
def tank_case(T=128, H_over_T=1.25, u_tip=0.05, re=2000.0, spacing=0.7):
    import lbmflow_b200 as lb
    nz = int(round(H_over_T * T))
    dims = (T, T, nz)
    dx = 1.0 / T  # lattice units: vessel diameter 1 m, dt chosen so Omega is in rad/step
    D = T / 3.0
    spec = lb.TankSpec(dims=dims, dx_m=dx, vessel_diameter_m=1.0, liquid_height_m=nz * dx,
                       impeller_diameter_m=1.0 / 3.0, clearance_m=1.0 / 3.0, omega_rad_s=1.0,
                       impeller="flat_blade", marker_spacing_cells=spacing, baffle_count=4,
                       baffle_width_m=0.1, baffle_thickness_m=2.6 * dx)
    geo = lb.build_stirred_tank(spec)
    omega = u_tip / (0.5 * D)  # rad/step
    n_rev = omega / (2.0 * math.pi)
    nu = n_rev * D * D / re
    body = lb.RotatingBody(geo["center"], [0.0, 0.0, omega], geo["marker_pos"], geo["marker_w"])
    return dims, geo["solid"], body, nu


def b_lu(q, storage):
    return 2 * q * {"f32": 4, "f16": 2, "bf16": 2, "f64": 8}[storage]


# ---------------------------------------------------------------------------
# Clocks sampled during the timed region
# ---------------------------------------------------------------------------
class ClockSampler:
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device=0):
        self.device = device
        self.proc = None
        self.lines = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.device), f"--query-gpu={self.FIELDS}",
                                          "--format=csv,noheader,nounits", "-lms", "100"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except OSError:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            p = [x.strip() for x in ln.split(",")]
            if len(p) < 9:
                continue
            try:
                sm.append(float(p[1]))
                mx = float(p[2])
            except ValueError:
                continue
            for nm, v in zip(names, p[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(nm)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"], "samples": 0}
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


def peak_hbm():
    try:
        with open(PEAKS_FILE) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    except (OSError, KeyError, ValueError):
        return FALLBACK_HBM_GBS, "fallback"


# ---------------------------------------------------------------------------
# CPU baseline (oracle), bounded sample
# ---------------------------------------------------------------------------
def cpu_tank_sample(dims, solid, body, nu, q=27, collision="cm", bits=32, steps=3, warmup=1):
    from oracle import oracle as o
    os_ = 1.0 / (3.0 * nu + 0.5)
    c = o.OracleSolver(dims, q=q, real_bits=bits, collision=collision, nu=nu, omega_shear=os_, solid=solid)
    c.run_tank(body.positions, body.weights, body.center, body.omega, warmup)
    t0 = time.perf_counter()
    c.run_tank(body.positions, body.weights, body.center, body.omega, steps)
    dt = time.perf_counter() - t0
    n = dims[0] * dims[1] * dims[2]
    return n * steps / dt / 1e6, dt


# ---------------------------------------------------------------------------
# Distributed plumbing (replicas: one independent tank per GPU)
# ---------------------------------------------------------------------------
def dist_init(n_gpus):
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime

        import torch
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
    return rank, world, local


def allmax(v, world):
    if world == 1:
        return v
    import torch
    import torch.distributed as dist
    t = torch.tensor([v], dtype=torch.float64, device="cuda")
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def barrier(world):
    if world > 1:
        import torch.distributed as dist
        dist.barrier()


def run_b200(args, rank, world, local):
    import lbmflow_b200 as lb

    dims, solid, body, nu = tank_case(T=args.tank_T)
    q, coll, storage = args.lattice, args.collision, args.storage
    os_ = 1.0 / (3.0 * nu + 0.5)
    n_cells = dims[0] * dims[1] * dims[2]
    n_fluid = int((solid == 0).sum())
    g = lb.Solver(dims, lattice=q, collision=coll, storage=storage, nu=nu, omega_shear=os_, solid=solid,
                  device=local)
    cfg = lb.DirectForcingConfig()
    # warm-up (untimed)
    g.run_impeller(body, max(args.warmup, 3))
    barrier(world)
    g.sync()
    # timed region: K runner steps, device time by CUDA events on the solver stream
    with ClockSampler(local) as clk:
        out = g.run_impeller(body, args.steps)
        t_total_ms, _, _ = g.last_timing()
    t_ms = allmax(t_total_ms, world)
    barrier(world)
    ms_per_step = t_ms / args.steps
    value = world * n_cells * args.steps / (t_ms * 1e-3) / 1e6
    # hydro-kernel-only launches (same stream, CUDA events) for the roofline
    g.run(4)
    g.run(args.hydro_steps)
    hydro_ms, _, launches = g.last_timing()
    per_launch_ms = hydro_ms / max(launches, 1)
    alg_bytes = b_lu(q, storage) * n_fluid
    achieved = alg_bytes / (per_launch_ms * 1e-3) / 1e9
    peak, peak_kind = peak_hbm()
    # e2e through the reference-facing API with host buffers: per step the
    # caller passes the rotating body (host arrays) to apply_rotating_ibm,
    # reads the diagnostics back and advances one step.
    e2e_steps = args.e2e_steps
    g2 = lb.Solver(dims, lattice=q, collision=coll, storage=storage, nu=nu, omega_shear=os_, solid=solid,
                   device=local)
    h2d = body.positions.nbytes + body.weights.nbytes + 48
    d2h = 100
    for _ in range(3):
        g2.clear_body_force_field()
        g2.set_body(0, body)
        g2.apply_rotating_ibm(body, cfg)
        g2.run(1)
    g2.sync()
    barrier(world)
    t0 = time.perf_counter()
    for _ in range(e2e_steps):
        g2.clear_body_force_field()
        g2.set_body(0, body)  # host -> device upload of the marker set
        g2.apply_rotating_ibm(body, cfg)  # device -> host diagnostics
        g2.run(1)
    g2.sync()
    e2e_s = allmax(time.perf_counter() - t0, world)
    e2e_value = world * n_cells * e2e_steps / e2e_s / 1e6
    g2.close()
    # low-precision storage variants (same workload, short timing)
    extra = {}
    if args.variants:
        for st in ("f16", "bf16"):
            gv = lb.Solver(dims, lattice=q, collision=coll, storage=st, nu=nu, omega_shear=os_, solid=solid,
                           device=local)
            gv.run_impeller(body, 8)
            gv.run_impeller(body, max(args.steps // 2, 16))
            tv, _, _ = gv.last_timing()
            extra[f"{st}_mlups"] = n_cells * max(args.steps // 2, 16) / (tv * 1e-3) / 1e6
            gv.run(args.hydro_steps)
            hv, _, lv = gv.last_timing()
            extra[f"{st}_hydro_gbs"] = b_lu(q, st) * n_fluid / (hv / lv * 1e-3) / 1e9
            gv.close()
        extra["fp16_over_fp32"] = extra["f16_mlups"] / (value / world)
        # D3Q19 TRT on the same tank (the reference runner's collision), fp32
        # and fp16-storage: runner step MLUPS and the hydro sweep's fraction
        # of the HBM roofline (152 / 76 bytes per fluid cell).
        peak, _ = peak_hbm()
        for st in ("f32", "f16"):
            gv = lb.Solver(dims, lattice=19, collision="trt", storage=st, nu=nu, solid=solid, device=local)
            gv.run_impeller(body, 8)
            k = max(args.steps // 2, 16)
            gv.run_impeller(body, k)
            tv, _, _ = gv.last_timing()
            extra[f"d3q19_trt_{st}_mlups"] = n_cells * k / (tv * 1e-3) / 1e6
            gv.run(args.hydro_steps)
            hv, _, lv = gv.last_timing()
            gbs = b_lu(19, st) * n_fluid / (hv / lv * 1e-3) / 1e9
            extra[f"d3q19_trt_{st}_hydro_gbs"] = gbs
            extra[f"d3q19_trt_{st}_hydro_frac"] = gbs / peak
            gv.close()
        extra["d3q19_fp16_over_fp32"] = extra["d3q19_trt_f16_mlups"] / extra["d3q19_trt_f32_mlups"]
    torque = out["torque_lu"]
    res = {
        "metric": "MLUPS (stirred-tank runner step, D3Q27 central moment, fp32 populations)",
        "value": value, "unit": "MLUPS", "n_gpus": world, "steps": args.steps, "warmup": max(args.warmup, 3),
        "ms_per_step": ms_per_step, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": {"f32": "f32", "f16": "f16-storage/f32", "bf16": "bf16-storage/f32", "f64": "f64"}[storage],
        "data": "synthetic (seeded tank geometry, quiescent start)",
        "config": {"workload": "tank128x128x160_d3q27_cm_ibm6k", "grid": list(dims), "cells": n_cells,
                   "fluid_cells": n_fluid, "markers": int(body.weights.size), "lattice": "D3Q27",
                   "collision": "central_moment", "storage": storage, "nu": nu, "u_tip": 0.05, "re": 2000,
                   "ibm": "3 sweeps, tol 1e-2, radius 1", "top": "solid lid (reference)",
                   "l2": "inputs larger than L2 (populations %.0f MB)" % (q * 4 * n_cells / 1e6),
                   "parallelism": f"replicas x{world}"},
        "e2e": {"value": e2e_value, "unit": "MLUPS", "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
                "path": "C ABI per step: ibm_set_body(host markers) + apply_rotating_ibm(diag to host) + step"},
        "gpu_launches": int(12 * args.steps),
        "roofline": {"bound": "hbm", "kernel": "hydro_aa_kernel<27,float,CM>", "achieved": achieved,
                     "peak": peak, "unit": "GB/s", "frac": achieved / peak, "traffic": None,
                     "peak_kind": peak_kind, "bytes_per_fluid_cell": b_lu(q, storage),
                     "launch_ms": per_launch_ms},
        "qoi": {"torque_lu_last": float(torque[-1]), "finite": bool(np.isfinite(torque).all())},
        "clocks": clk.summary(),
    }
    res.update(extra)
    if rank == 0 and world == 1 and not args.no_cpu:
        mlups, dt = cpu_tank_sample(dims, solid, body, nu, steps=args.cpu_steps)
        res["cpu_baseline"] = {"value": mlups, "unit": "MLUPS", "cores": os.cpu_count(), "kind": "port",
                               "sample": f"{args.cpu_steps} runner steps of the full tank, fp32, OpenMP "
                                         f"({dt:.1f} s)"}
    g.close()
    return res


def run_reference(args, rank, world):
    if rank != 0:
        return None
    dims, solid, body, nu = tank_case(T=args.tank_T)
    steps = max(1, min(args.steps, args.cpu_steps))
    mlups, dt = cpu_tank_sample(dims, solid, body, nu, steps=steps, warmup=1)
    return {"impl": "reference", "metric": "MLUPS (stirred-tank runner step, D3Q27 central moment, fp32 populations)",
            "value": mlups, "unit": "MLUPS", "n_gpus": world, "steps": steps, "warmup": 1,
            "ms_per_step": dt / steps * 1e3, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f32", "data": "synthetic (seeded tank geometry, quiescent start)",
            "config": {"workload": "tank128x128x160_d3q27_cm_ibm6k", "grid": list(dims)},
            "cpu_baseline": {"value": mlups, "unit": "MLUPS", "cores": os.cpu_count(), "kind": "port",
                             "sample": f"{steps} runner steps of the full tank on the host cores (C++ "
                                       f"restatement of the reference CpuScalar path; the Rust reference "
                                       f"cannot be built here)"},
            "e2e": {"value": mlups, "unit": "MLUPS", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=6000)
    ap.add_argument("--warmup", type=int, default=20)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--storage", default="f32", choices=["f32", "f16", "bf16"])
    ap.add_argument("--hydro-steps", type=int, default=200)
    ap.add_argument("--e2e-steps", type=int, default=100)
    ap.add_argument("--tank-T", type=int, default=128, help="tank diameter in cells (128 = the benchmark case)")
    ap.add_argument("--lattice", type=int, default=27, choices=[19, 27])
    ap.add_argument("--collision", default="cm", choices=["cm", "trt"])
    ap.add_argument("--cpu-steps", type=int, default=12)
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--variants", type=int, default=1)
    args = ap.parse_args()
    rank, world, local = dist_init(args.gpus)
    if args.impl == "reference":
        res = run_reference(args, rank, world)
    else:
        res = run_b200(args, rank, world, local)
    if rank == 0 and res is not None:
        print(json.dumps(res), flush=True)
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
