"""Benchmark of the LBMFlow stirred-tank time step on B200.

Workload (the single-GPU tank configuration): cylindrical tank T = 128
cells on a 128 x 128 x 160 grid, flat bottom, free-slip (specular) liquid surface on top (``--lid`` for the
reference's no-slip lid), four wall baffles of width
T/10 and thickness 2.6 cells, a six-blade flat-blade disc turbine of
diameter T/3 at clearance T/3 sampled by ~6k direct-forcing IBM markers at
0.7-cell spacing, tip speed 0.05, nu for impeller Re = 2000, D3Q27
central-moment collision, fp32 populations, 20k steps, with the library's
optional Smagorinsky model (Cs = 0.1; the reference operators diverge on
this under-resolved tank). One step = the reference runner step (clear
force field -> IBM direct forcing -> collide/stream/moments), synthetic
seeded geometry, quiescent start after a warm-up; the sweep kernel is
picked by the library's autotuner on the tank itself.

Besides the headline line the output carries the precision study (power
number of the same schedule with f64 / f32 / f16 / bf16 populations for the
D3Q27 central-moment and D3Q19 TRT forms, errors against the f64 path) and
the throughput of every form at T = 256 (256 x 256 x 320, populations
larger than L2).

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

# DRAM traffic per launch (dram__bytes_read.sum + dram__bytes_write.sum, mean of
# one even and one odd launch) from an ncu full-set capture of the sweep kernel
# the autotuner picks for the form, on the tank of the given diameter.
NCU_TRAFFIC = {("hydro_async_kernel", 27, "cm", "f32", 128): 448.2e6,
               ("hydro_pair_kernel", 27, "cm", "f32", 128): 466.0e6,
               ("hydro_pair_kernel", 19, "trt", "f32", 256): 2720.2e6,
               ("hydro_pair_kernel", 19, "trt", "f16", 256): 1406.1e6,
               ("hydro_pair_kernel", 19, "trt", "bf16", 256): 1403.9e6,
               ("hydro_pair_kernel", 27, "cm", "f32", 256): 3916.6e6,
               ("hydro_pair_kernel", 27, "cm", "f16", 256): 2006.1e6,
               ("hydro_pair_kernel", 27, "cm", "bf16", 256): 2016.5e6}
KERNEL_NAME = {"lean": "hydro_lean_kernel", "pair": "hydro_pair_kernel", "tile": "hydro_tile_kernel",
               "window": "hydro_window_kernel", "async": "hydro_async_kernel", "direct": "hydro_aa_kernel",
               "bulk": "hydro_tma_kernel"}
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


def tank_case_oracle(T=128, H_over_T=1.25, u_tip=0.05, re=2000.0, spacing=0.7):
    """The tank of tank_case built by the oracle's restatement of the same
    generators (bit-identical to lbmb_build_stirred_tank, tests/
    test_runner_qoi.py), so that a CPU leg loads nothing of the product."""
    from types import SimpleNamespace

    from oracle import oracle as o
    nz = int(round(H_over_T * T))
    dims = (T, T, nz)
    dx = 1.0 / T
    D = T / 3.0
    geo = o.build_tank(dims, dx, 1.0, nz * dx, 1.0 / 3.0, 1.0 / 3.0, 6, 1.0, baffle_w=0.1, baffle_t=2.6 * dx,
                       kind=2, spacing=spacing)
    omega = u_tip / (0.5 * D)
    nu = omega / (2.0 * math.pi) * D * D / re
    body = SimpleNamespace(center=geo["center"], omega=np.array([0.0, 0.0, omega]),
                           positions=geo["marker_pos"], weights=geo["marker_w"])
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
                                          "--format=csv,noheader,nounits", "-lms", "50"],
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
def cpu_tank_sample(dims, solid, body, nu, q=27, collision="cm", bits=32, steps=3, warmup=1, cs=0.0,
                    store16=None):
    """The oracle's runner loop (OpenMP over the host cores) from rest:
    `warmup` untimed steps, then `steps` timed ones. Returns (MLUPS, seconds,
    the torque series of all warmup + steps steps). store16: "f16" | "bf16"
    rounds every stored population to that type (fp32 arithmetic)."""
    from oracle import oracle as o
    os_ = 1.0 / (3.0 * nu + 0.5)
    c = o.OracleSolver(dims, q=q, real_bits=bits, collision=collision, nu=nu, omega_shear=os_, solid=solid,
                       smagorinsky_cs=cs, free_slip_top=FREE_SLIP_TOP, store16=store16)
    r0 = c.run_tank(body.positions, body.weights, body.center, body.omega, warmup)
    t0 = time.perf_counter()
    r1 = c.run_tank(body.positions, body.weights, body.center, body.omega, steps)
    dt = time.perf_counter() - t0
    n = dims[0] * dims[1] * dims[2]
    return n * steps / dt / 1e6, dt, np.concatenate([r0["torque_lu"], r1["torque_lu"]])


def shear_study(g, dims, solid, nu, T, q, storage):
    """The bioprocess runner's stress QOI (runner.rs:1648-1690) on the final
    headline state: gamma_dot and viscous-stress percentiles over the fluid
    cells, on the device (moments, f64 finite differences, device sort) and
    through the oracle's restatement of stress.rs on the same velocity (the
    CPU leg, single thread). Units: a water-filled 1 m vessel (dx = 1 / T m,
    nu = 1e-6 m^2/s, mu = 1e-3 Pa s; dt from nu_lattice = nu dt / dx^2)."""
    from oracle import oracle as o
    dx = 1.0 / T
    dt = nu * dx * dx / 1.0e-6
    mu = 1.0e-3
    g.stress_summary(dx, dt, mu)  # warm-up (first-call set-up)
    runs = [g.stress_summary(dx, dt, mu, 0.0, 0.0) for _ in range(3)]
    gam, tau, _ = runs[-1]
    dev_ms = min(r[2] for r in runs)
    _, ux, uy, uz = g.read_moments()
    vs = dx / dt
    t0 = time.perf_counter()
    ref = o.compute_stress_field(dims, ux * vs, uy * vs, uz * vs, solid, dx, mu)
    fl = solid == 0
    rg = o.percentile_summary(ref["gamma_dot"][fl], 0.0)
    cpu_ms = (time.perf_counter() - t0) * 1e3
    n_fluid = int(fl.sum())
    pop_bytes = q * {"f32": 4, "f16": 2, "bf16": 2, "f64": 8}[storage] * n_fluid
    return {"what": "gamma_dot / viscous-stress percentiles over fluid cells (stress.rs, runner.rs:1648-1690)",
            "units": {"dx_m": dx, "dt_s": dt, "mu_pa_s": mu}, "fluid_cells": n_fluid,
            "gamma_dot_1_s": gam, "viscous_stress_pa": tau, "device_ms": dev_ms,
            "device_populations_gbs": pop_bytes / (dev_ms * 1e-3) / 1e9,
            "cpu_ms": cpu_ms, "cpu_kind": "port (oracle restatement, 1 thread, same velocity field)",
            "p95_rel_diff_vs_cpu": abs(gam["p95"] - rg["p95"]) / rg["p95"]}


def oxygen_study(g, dims, solid, T):
    """Oxygen transfer on a D3Q7 scalar of the final headline state (the
    reference composition gather -> apply_interfacial_flux_sources -> set,
    oxygen.rs:124-191): Henry C* = 1.3e-5 x 21 kPa, kL = 2e-4 m/s, interface
    area density 1/dx on the top fluid layer, dx = 1/T m, dt = 1 ms. Timed
    through the public call (host arrays in, ledger out) against the
    oracle's restatement of the host function on the same arrays."""
    from oracle import oracle as o
    n = dims[0] * dims[1] * dims[2]
    dx = 1.0 / T
    fl = solid == 0
    z = np.arange(n) // (dims[0] * dims[1])
    top = int(z[fl].max())
    import torch
    area = torch.empty(n, dtype=torch.float64, pin_memory=True).numpy()  # caller's array in pinned memory
    area[...] = np.where(fl & (z == top), 1.0 / dx, 0.0)
    k = g.enable_scalar_distribution(1e-2, q=7)
    g.set_scalar_concentration(k, np.where(fl, 0.05, 0.0))
    c_star, kl, vol, dt = 1.3e-5 * 21000.0, 2.0e-4, dx ** 3, 1.0e-3
    g.apply_interfacial_flux_sources(k, area, c_star, vol, dt, kl)  # warm-up
    g.sync()
    times = []
    for _ in range(7):
        t0 = time.perf_counter()
        led, diag = g.apply_interfacial_flux_sources(k, area, c_star, vol, dt, kl)
        times.append((time.perf_counter() - t0) * 1e3)
    dev_ms = float(np.median(times))
    c = g.gather_scalar_concentration(k)
    led, diag = g.apply_interfacial_flux_sources(k, area, c_star, vol, dt, kl)  # on the state c holds
    t0 = time.perf_counter()
    _, led_c, _ = o.interfacial_flux(c, c_star, area, vol, dt, kl)
    cpu_ms = (time.perf_counter() - t0) * 1e3
    return {"what": "kL a (C* - C) transfer step on a D3Q7 scalar, gather + source + clip + set (oxygen.rs)",
            "cells": n, "interface_cells": led["active_interface_cells"], "source_integral_mol_s":
            led["source_integral_mol_s"], "call_ms": dev_ms,
            "call_path": "C ABI, median of 7 calls, host area array (pinned) uploaded every call (8 B per cell)",
            "cpu_ms": cpu_ms, "cpu_kind": "port (oracle restatement of the host function, 1 thread, source only)",
            "ledger_rel_diff_vs_cpu": abs(led["source_integral_mol_s"] - led_c["source_integral_mol_s"]) /
            abs(led_c["source_integral_mol_s"])}


def checkpoint_study(g):
    """Solver::save / restore (the reference's v3 checkpoint files,
    solver.rs:4536-5066) of the final headline state: populations, moments,
    the IBM force field and the D3Q7 scalar, through the C ABI into a
    temporary directory; then a full-size resume check: 2 steps from the
    saved state, restore, the same 2 steps again, moments bit for bit."""
    import shutil
    import tempfile
    d = tempfile.mkdtemp(prefix="lbmb_ckpt_")
    try:
        g.sync()
        save_ms = []
        for _ in range(2):  # the first call also allocates the pinned staging buffer
            t0 = time.perf_counter()
            g.save(d)
            save_ms.append((time.perf_counter() - t0) * 1e3)
        nbytes = sum(os.path.getsize(os.path.join(d, f)) for f in os.listdir(d))
        step0 = g.time
        g.run(2)
        a = g.read_moments()
        t0 = time.perf_counter()
        g.restore(d)
        restore_ms = (time.perf_counter() - t0) * 1e3
        restored_step = g.time
        g.run(2)
        b = g.read_moments()
        exact = all(np.array_equal(x, y) for x, y in zip(a, b))
    finally:
        shutil.rmtree(d, ignore_errors=True)
    return {"what": "checkpoint save + restore of the final state (manifest.json + rank_0000_part_0000.bin, "
                    "reference v3 format: padded f32/f64 planes, zero stash, FNV-1a 64 payload hash)",
            "bytes": nbytes, "save_ms": save_ms[1], "first_save_ms": save_ms[0], "restore_ms": restore_ms,
            "save_GBps": nbytes / save_ms[1] / 1e6, "restore_GBps": nbytes / restore_ms / 1e6,
            "path": "device packs the padded planes in the file type, one pinned copy each way; the host "
                    "hashes (FNV-1a 64, byte-serial; all-zero 64-byte blocks as one multiply) while a second "
                    "thread writes / reads the rank file",
            "step": step0, "restored_step": restored_step, "resume_bit_exact_2_steps": bool(exact),
            "directory": "tempfile.mkdtemp() on the bench host"}


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


def power_number(torque_lu, omega, D):
    """Np from the last-half mean torque (runner.rs:1523-1530; qoi.rs:477-505),
    lattice units with rho = 1: P = Omega Tq, N = Omega / 2 pi, Np = P / (N^3 D^5)."""
    t = np.asarray(torque_lu)
    tq = float(np.mean(t[t.size // 2:]))
    n_rev = omega / (2.0 * math.pi)
    return omega * tq / (n_rev ** 3 * D ** 5)


FREE_SLIP_TOP = True


def make_solver(lb, dims, solid, nu, q, coll, storage, cs, local):
    os_ = 1.0 / (3.0 * nu + 0.5)
    return lb.Solver(dims, lattice=q, collision=coll, storage=storage, nu=nu, omega_shear=os_, solid=solid,
                     device=local, smagorinsky_cs=cs, free_slip_top=FREE_SLIP_TOP)


def qoi_study(lb, args, local, dims, solid, body, nu, D, headline_np):
    """QOI errors of every storage precision against the f64 path on a fixed
    schedule, independent of --steps: qoi_revs impeller revolutions from
    rest; the power number from the mean torque over the last half of the
    run (the runner's window, runner.rs:1523-1530), the kinetic energy of
    the fluid averaged over that half, and the L2 error of the velocity
    field averaged over that half (sampled every 200 steps). The flow at
    Re = 2000 is chaotic, so time averages rather than instantaneous fields
    are compared; the integral quantities (Np, energy) converge within two
    revolutions, the mean field does not fully. The f64 path is the one the parity tests pin to the
    C++ oracle (tests/test_gpu_configs.py: the 128 x 128 x 160 tank's first
    100 steps to 1e-9 of the torque, the 64^3 cavity's 1000 steps to 1e-11)."""
    out = {}
    omega = float(body.omega[2])
    rev = 2.0 * math.pi / omega
    steps = int(round(args.qoi_revs * rev))
    half = steps // 2
    every = 200
    fluid = solid == 0
    out["schedule"] = {"revolutions": args.qoi_revs, "steps": steps, "window": [half + 1, steps],
                       "velocity_samples_every": every}
    for q, coll, label in ((27, "cm", "d3q27_cm"), (19, "trt", "d3q19_trt")):
        res = {}
        for st in ("f64", "f32", "f16", "bf16"):
            g = make_solver(lb, dims, solid, nu, q, coll, st, args.les_cs, local)
            g.autotune_sweep(6)
            r = g.run_impeller(body, half)
            tq = [r["torque_lu"]]
            ok = r["status"] == "completed"
            usum, nsum, done, ke = None, 0, half, 0.0
            while ok and done < steps:
                k = min(every, steps - done)
                r = g.run_impeller(body, k)
                ok = r["status"] == "completed"
                tq.append(r["torque_lu"])
                done += k
                u = np.stack(g.read_moments()[1:4])[:, fluid]
                usum = u if usum is None else usum + u
                ke += 0.5 * float(np.sum(u * u))
                nsum += 1
            tq = np.concatenate(tq)
            fin = ok and np.isfinite(tq).all()
            res[st] = {"Np": power_number(tq, omega, D) if fin else None,
                       "torque_mean": float(np.mean(tq[half:])) if fin else None,
                       "ke_mean": ke / nsum if (fin and nsum) else None,
                       "u_mean": usum / nsum if (fin and nsum) else None}
            g.close()
        ref = res["f64"]
        errs = {}
        for st in ("f32", "f16", "bf16"):
            r = res[st]
            e = {"Np": abs(r["Np"] - ref["Np"]) / abs(ref["Np"]) if r["Np"] and ref["Np"] else None,
                 "mean_kinetic_energy": (abs(r["ke_mean"] - ref["ke_mean"]) / ref["ke_mean"]
                                         if r["ke_mean"] and ref["ke_mean"] else None)}
            if r["u_mean"] is not None and ref["u_mean"] is not None:
                e["mean_velocity_L2"] = float(np.linalg.norm(r["u_mean"] - ref["u_mean"]) /
                                              np.linalg.norm(ref["u_mean"]))
            errs[st] = e
        out[label] = {"Np": {k_: v["Np"] for k_, v in res.items()}, "rel_err_vs_f64": errs}
    return out


def mixing_study(lb, args, local):
    """95% / 99% mixing time of a D3Q7 passive-scalar pulse (Gaussian, sigma
    4 cells, centred on the axis just under the liquid surface) in the
    T = mix_T tank, D3Q27 central-moment form, every storage precision
    against the f64 path; CV probed every 200 steps, run until CV <= 0.01
    CV0 or mix_steps. The stated diffusivity (mix_D, 1e-3 lattice units,
    grid Peclet u_tip / D = 50, tau_s = 4 D + 1/2 = 0.504) is run first; a
    precision whose run stops (non-finite CV or mass) is recorded with the
    step it stopped at (none has: the runs stay bounded and reach t99 within
    about 150,000 steps), and the study is then repeated at 1e-2. mix_D2 > 0
    adds a second diffusivity. Each run reports the CV / CV0 it reached."""
    from lbmflow_b200 import sweep
    c = sweep.TankCase(args.mix_T, 0.05, 2000.0)
    geo = sweep.tank_geometry(args.mix_T)
    dims, solid = c.dims, geo["solid"]
    body = lb.RotatingBody(geo["center"], [0.0, 0.0, c.omega], geo["marker_pos"], geo["marker_w"])
    c0 = lb.gaussian_pulse(dims, solid, ((dims[0] - 1) / 2.0, (dims[1] - 1) / 2.0, dims[2] - 2.0), 4.0)
    probe, chunk = 200, 5000

    finals = {}

    def run(D):
        res, stops = {}, {}
        for st in ("f64", "f32", "f16", "bf16"):
            g = make_solver(lb, dims, solid, c.nu, 27, "cm", st, args.les_cs, local)
            k = g.enable_scalar_distribution(D, q=7)
            g.set_scalar_concentration(k, c0)
            cvs, done, mix, stop = [], 0, None, None
            while done < args.mix_steps:
                r = g.run_impeller(body, chunk, scalar=k, probe_every=probe)
                cv = r["cv"][:r["executed"]]
                cvs.append(cv)
                done += r["executed"]
                bad = [i for i in range(probe - 1, cv.size, probe) if not np.isfinite(cv[i])]
                if r["status"] != "completed" or bad:
                    stop = int(done - cv.size + (bad[0] + 1 if bad else cv.size))
                    break
                allcv = np.concatenate(cvs)
                mix = lb.mixing_time_from_cv(np.arange(1, allcv.size + 1, dtype=np.float64), allcv)
                if mix is not None and mix["t99"] is not None:
                    break
            res[st] = None if stop is not None else mix
            stops[st] = stop
            allcv = np.concatenate(cvs) if cvs else np.array([np.nan])
            fin = allcv[np.isfinite(allcv)]
            finals[st] = {"steps": int(done), "cv_over_cv0": float(fin[-1] / fin[0]) if fin.size > 1 else None}
            g.close()
        return res, stops

    def errs(res):
        ref = res["f64"]
        out = {}
        for st in ("f32", "f16", "bf16"):
            e = {}
            for key in ("t95", "t99"):
                a, b = (res[st] or {}).get(key), (ref or {}).get(key)
                e[key] = abs(a - b) / b if a and b else None
            out[st] = e
        return out

    out = {"grid": list(dims), "sigma_cells": 4.0, "probe_every": probe, "step_cap": args.mix_steps,
           "revolution_steps": 2 * math.pi / c.omega, "form": "D3Q27 central moment + D3Q7 scalar"}
    Ds = [args.mix_D] + ([args.mix_D2] if args.mix_D2 > 0 else [])
    for D in Ds:
        res, stops = run(D)
        out[f"D={D:g}"] = {"grid_peclet": 0.05 / D, "tau_s": 4.0 * D + 0.5,
                           "t95_steps": {k_: (v or {}).get("t95") for k_, v in res.items()},
                           "t99_steps": {k_: (v or {}).get("t99") for k_, v in res.items()},
                           "stopped_at_step": stops, "final": dict(finals),
                           "rel_err_vs_f64": errs(res)}
        if D == args.mix_D and any(v is not None for v in stops.values()) and 1e-2 not in Ds:
            Ds.append(1e-2)  # the loop picks it up
    return out


def throughput_study(lb, args, local, peak):
    """Sweep throughput at the precision-variant grid (tank T = big_T,
    populations larger than L2): hydro kernel GB/s against the HBM roofline
    and runner-step MLUPS, autotuned kernel per configuration."""
    dims, solid, body, nu = tank_case(T=args.big_T)
    n_cells = dims[0] * dims[1] * dims[2]
    n_fluid = int((solid == 0).sum())
    res = {"grid": list(dims), "fluid_cells": n_fluid, "markers": int(body.weights.size)}
    for q, coll in ((19, "trt"), (27, "cm")):
        for st in ("f32", "f16", "bf16"):
            g = make_solver(lb, dims, solid, nu, q, coll, st, args.les_cs, local)
            tune = g.autotune_sweep(6)
            g.run(4)
            g.run(args.hydro_steps)
            hms, _, L = g.last_timing()
            per = hms / max(L, 1)
            gbs = b_lu(q, st) * n_fluid / (per * 1e-3) / 1e9
            g.run_impeller(body, 8)
            g.run_impeller(body, args.big_steps)
            tms, _, _ = g.last_timing()
            traffic = NCU_TRAFFIC.get((KERNEL_NAME[tune["kind"]], q, coll, st, args.big_T))
            res[f"d3q{q}_{coll}_{st}"] = {"kernel": tune["kind"],
                                          "variant": [tune["even_blocks_per_sm"], tune["odd_blocks_per_sm"]],
                                          "hydro_ms": per, "hydro_gbs": gbs, "hydro_frac": gbs / peak,
                                          "traffic": traffic,
                                          "traffic_over_algorithmic": (traffic / (b_lu(q, st) * n_fluid)
                                                                       if traffic else None),
                                          "runner_mlups": n_cells * args.big_steps / (tms * 1e-3) / 1e6}
            g.close()
    for q, coll in ((19, "trt"), (27, "cm")):
        a, b = res[f"d3q{q}_{coll}_f16"], res[f"d3q{q}_{coll}_f32"]
        res[f"d3q{q}_{coll}_fp16_over_fp32_runner"] = a["runner_mlups"] / b["runner_mlups"]
        res[f"d3q{q}_{coll}_fp16_over_fp32_hydro"] = b["hydro_ms"] / a["hydro_ms"]
    return res


def sweep_study(args, rank, world, local):
    """Batched sweep (64 seeded D3Q19 TRT fp32 tanks, T ~ U{48..128}, height
    1.25 T, u_tip ~ U(0.02, 0.06), Re ~ U(500, 5000), seed 0x5EED): all of a
    rank's cases in lockstep through the batched runner, autotuned; cases are
    sharded over ranks by LPT and per-case Np gathered on rank 0. The
    reference's sequential per-case loop is timed on a bounded sample."""
    from lbmflow_b200 import sweep

    cases = sweep.seeded_cases()

    def gather(obj):
        if world == 1:
            return [obj]
        import torch.distributed as dist
        out = [None] * world
        dist.all_gather_object(out, obj)
        return out

    res = sweep.run_sharded(cases, args.sweep_steps, rank, world, gather, mode="batch", les_cs=args.les_cs,
                            device=local, warmup=16)
    if rank != 0:
        return None
    out = {"cases": len(cases), "steps_per_case": args.sweep_steps, "cells_total": sum(c.cells for c in cases),
           "mlups": res["mlups"], "device_ms_max_over_ranks": res["device_ms_max"],
           "Np": res["aggregate"].get("Np"), "finite_cases": sum(1 for p in res["per_case"] if np.isfinite(p["Np"])),
           "seed": "0x5EED", "storage": "f32", "lattice": "D3Q19 TRT", "sharding": f"LPT over {world} rank(s)"}
    if world == 1 and args.sweep_seq_steps > 0:
        seq = sweep.run_sweep(cases, args.sweep_seq_steps, mode="sequential", les_cs=args.les_cs, autotune=False,
                              device=local)
        out["sequential_sample"] = {"steps_per_case": args.sweep_seq_steps, "mlups": seq["mlups"],
                                    "what": "one case after another (sweep.rs:61-68 order), each through the "
                                            "device runner loop"}
        out["batch_over_sequential"] = res["mlups"] / seq["mlups"]
    return out


def adjoint_study(args, local):
    """Adjoint of the runner loop on the D3Q19 TRT tank T = 96 (96 x 96 x
    120), fp32 forward with f64 reductions, 2000 steps, a checkpoint every
    100, J = mean torque over steps 1001-2000, fixed 3 IBM sweeps. Gradient
    w.r.t. (nu, Omega, marker positions) checked against central differences
    of the f64 forward on seeded random directions in (nu / nu0, Omega /
    Omega0, x / cell), relative step 1e-4, and against the f64 adjoint. The
    markers get a seeded jitter of at most 0.1 cell (no marker on a kink of
    the linear IBM kernel). Re = adj_re keeps the flow laminar so that J is
    smooth in the parameters."""
    import lbmflow_b200 as lb
    from lbmflow_b200 import sweep

    T, steps, K = args.adj_T, args.adj_steps, 100
    win = steps // 2
    c = sweep.TankCase(T, 0.05, args.adj_re)
    geo = sweep.tank_geometry(T)
    rng = np.random.default_rng(0x5EED)
    pos0 = geo["marker_pos"] + rng.uniform(-0.1, 0.1, size=geo["marker_pos"].shape)
    cfg = lb.DirectForcingConfig(max_iterations=3, slip_tolerance=0.0)

    def solver(storage, nu):
        return lb.Solver(c.dims, lattice=19, collision="trt", storage=storage, nu=nu, solid=geo["solid"],
                         device=local)

    def body(omega, pos):
        return lb.RotatingBody(geo["center"], [0.0, 0.0, omega], pos, geo["marker_w"])

    g = solver("f32", c.nu)
    r32 = g.adjoint_torque(body(c.omega, pos0), steps, win, K, cfg)
    g.close()
    # plain forward (graph-captured runner) for the cost ratio
    g = solver("f32", c.nu)
    g.run_impeller(body(c.omega, pos0), steps, cfg)
    fwd_ms, _, _ = g.last_timing()
    g.close()
    g = solver("f64", c.nu)
    r64 = g.adjoint_torque(body(c.omega, pos0), steps, win, K, cfg)
    g.close()

    def J(nu, omega, pos):
        s_ = solver("f64", nu)
        t = s_.run_impeller(body(omega, pos), steps, cfg)["torque_lu"]
        s_.close()
        return float(np.mean(t[win:]))

    nm = pos0.shape[0]
    h = 1e-4
    errs, errs64 = [], []
    for k in range(args.adj_dirs):
        d = rng.normal(size=2 + 3 * nm)
        d /= np.linalg.norm(d)
        dn, do, dp = d[0] * c.nu, d[1] * c.omega, d[2:].reshape(nm, 3)
        fd = (J(c.nu + h * dn, c.omega + h * do, pos0 + h * dp) -
              J(c.nu - h * dn, c.omega - h * do, pos0 - h * dp)) / (2 * h)
        ad32 = r32["dJ_dnu"] * dn + r32["dJ_domega_z"] * do + float(np.sum(r32["dJ_dpos"] * dp))
        ad64 = r64["dJ_dnu"] * dn + r64["dJ_domega_z"] * do + float(np.sum(r64["dJ_dpos"] * dp))
        errs.append(abs(ad32 - fd) / abs(fd))
        errs64.append(abs(ad64 - fd) / abs(fd))
    g32 = np.concatenate([[r32["dJ_dnu"], r32["dJ_domega_z"]], r32["dJ_dpos"].ravel()])
    g64 = np.concatenate([[r64["dJ_dnu"], r64["dJ_domega_z"]], r64["dJ_dpos"].ravel()])
    return {"grid": list(c.dims), "steps": steps, "checkpoint_every": K, "window": [win, steps],
            "re": args.adj_re, "u_tip": 0.05, "markers": int(nm), "J_f32": r32["J"], "J_f64": r64["J"],
            "dJ_dnu": r32["dJ_dnu"], "dJ_domega": r32["dJ_domega_z"],
            "fd_directions": args.adj_dirs, "fd_rel_step": h,
            "fd_rel_err_f32_adjoint_max": max(errs) if errs else None,
            "fd_rel_err_f64_adjoint_max": max(errs64) if errs64 else None,
            "f32_vs_f64_gradient_rel": float(np.linalg.norm(g32 - g64) / np.linalg.norm(g64)),
            "forward_ms_runner": fwd_ms, "forward_ms_checkpointed": r32["forward_ms"],
            "recompute_plus_adjoint_ms": r32["adjoint_ms"],
            "cost_ratio": r32["adjoint_ms"] / fwd_ms,
            "cost_note": "(recomputation + backward pass) / plain forward runner, device time"}


def run_b200(args, rank, world, local):
    import lbmflow_b200 as lb

    dims, solid, body, nu = tank_case(T=args.tank_T)
    q, coll, storage = args.lattice, args.collision, args.storage
    n_cells = dims[0] * dims[1] * dims[2]
    n_fluid = int((solid == 0).sum())
    D = args.tank_T / 3.0
    omega = float(body.omega[2])
    g = make_solver(lb, dims, solid, nu, q, coll, storage, args.les_cs, local)
    if args.sweep_kernel:
        # a fixed kernel (profiling runs: timings under a profiler would
        # mislead the autotuner)
        g.set_sweep_kernel(args.sweep_kernel)
        ev, od = 0, 0
        if args.sweep_variant:
            ev, od = (int(v) for v in args.sweep_variant.split("/"))
            g.set_sweep_variant(ev, od)
        tune = {"kind": args.sweep_kernel, "even_blocks_per_sm": ev, "odd_blocks_per_sm": od,
                "best_ms_per_step": None, "default_ms_per_step": None}
    else:
        # tune on a developed flow: on the quiescent start the central-moment
        # exact-rest skip makes every kernel unrepresentatively cheap
        if args.tune_after > 0:
            g.run_impeller(body, args.tune_after)
        tune = g.autotune_sweep(8)
    cfg = lb.DirectForcingConfig()
    # clocks are sampled (every 50 ms) from the warm-up through the timed
    # steps, the hydro-only launches and the e2e loop: a short timed span
    # alone would hold no sample
    clk = ClockSampler(local).__enter__()
    # warm-up (untimed)
    g.run_impeller(body, max(args.warmup, 3))
    barrier(world)
    g.sync()
    # timed region: K runner steps, device time by CUDA events on the solver stream
    out = g.run_impeller(body, args.steps)
    t_total_ms, _, _ = g.last_timing()
    t_ms = allmax(t_total_ms, world)
    barrier(world)
    ms_per_step = t_ms / args.steps
    value = world * n_cells * args.steps / (t_ms * 1e-3) / 1e6
    torque = out["torque_lu"]
    np_head = power_number(torque, omega, D) if np.isfinite(torque).all() else None
    # hydro-kernel-only launches (same stream, CUDA events) for the roofline
    g.run(4)
    g.run(args.hydro_steps)
    hydro_ms, _, launches = g.last_timing()
    per_launch_ms = hydro_ms / max(launches, 1)
    alg_bytes = b_lu(q, storage) * n_fluid
    achieved = alg_bytes / (per_launch_ms * 1e-3) / 1e9
    peak, peak_kind = peak_hbm()
    # e2e through the reference-facing API with host buffers: per step the
    # caller uploads the rotating body (host arrays), runs the IBM (its
    # diagnostics come back to the host) and advances one step.
    e2e_steps = args.e2e_steps
    g2 = make_solver(lb, dims, solid, nu, q, coll, storage, args.les_cs, local)
    g2.set_sweep_kernel(tune["kind"])
    if tune["even_blocks_per_sm"] and tune["kind"] in ("lean", "pair", "window", "async") and storage != "f64":
        g2.set_sweep_variant(tune["even_blocks_per_sm"], tune["odd_blocks_per_sm"])
    # the caller's marker arrays live in pinned host memory (copied to the
    # device every step); the step's result is the IBM diagnostics record
    # read back to the host. Timed two ways: one lbmb_runner_step per step
    # (the runner loop body in one call, the IBM beside the sweep), and the
    # reference loop's four calls (clear field, upload markers, apply with
    # the diagnostics, step).
    import torch
    pos_pin = torch.empty(body.positions.shape, dtype=torch.float64, pin_memory=True).numpy()
    w_pin = torch.empty(body.weights.shape, dtype=torch.float64, pin_memory=True).numpy()
    pos_pin[...] = body.positions
    w_pin[...] = body.weights
    body = lb.RotatingBody(body.center, body.omega, pos_pin, w_pin)
    h2d = body.positions.nbytes + body.weights.nbytes
    d2h = 128

    def calls_step():
        g2.clear_body_force_field()
        g2.set_body(0, body)  # host -> device upload of the marker set
        g2.apply_rotating_ibm(body, cfg)  # device -> host diagnostics
        g2.run(1)

    def fused_step():
        g2.runner_step(0, body, cfg)

    e2e_per = {}
    for name, fn in (("calls", calls_step), ("runner_step", fused_step)):
        for _ in range(3):
            fn()
        g2.sync()
        barrier(world)
        t0 = time.perf_counter()
        for _ in range(e2e_steps):
            fn()
        g2.sync()
        e2e_per[name] = allmax(time.perf_counter() - t0, world)
    e2e_s = e2e_per["runner_step"]
    e2e_value = world * n_cells * e2e_steps / e2e_s / 1e6
    e2e_calls_value = world * n_cells * e2e_steps / e2e_per["calls"] / 1e6
    g2.close()
    clk.__exit__()
    extra = {}
    if world == 1 and args.shear:
        extra["shear_qoi"] = shear_study(g, dims, solid, nu, args.tank_T, q, storage)
        extra["oxygen_transfer"] = oxygen_study(g, dims, solid, args.tank_T)
    if world == 1 and args.ckpt:
        extra["checkpoint"] = checkpoint_study(g)
    g.close()
    if args.sweep_steps > 0:
        sw = sweep_study(args, rank, world, local)
        if sw is not None:
            extra["sweep"] = sw
    if args.adj_steps > 0 and world == 1:
        extra["adjoint"] = adjoint_study(args, local)
    if args.variants and world == 1:
        if args.qoi_revs > 0:
            extra["qoi_precision"] = qoi_study(lb, args, local, dims, solid, body, nu, D, np_head)
        if args.mix_steps > 0:
            extra["mixing_precision"] = mixing_study(lb, args, local)
        if args.big_steps > 0:
            extra["throughput_T%d" % args.big_T] = throughput_study(lb, args, local, peak)
    kname = KERNEL_NAME[tune["kind"]]
    coll_name = {"cm": "central_moment", "trt": "trt"}[coll]
    res = {
        "metric": f"MLUPS (stirred-tank runner step, D3Q{q} {coll_name}, {storage} populations)",
        "value": value, "unit": "MLUPS", "n_gpus": world, "steps": args.steps, "warmup": max(args.warmup, 3),
        "ms_per_step": ms_per_step, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": {"f32": "f32", "f16": "f16-storage/f32", "bf16": "bf16-storage/f32", "f64": "f64"}[storage],
        "data": "synthetic (seeded tank geometry, quiescent start)",
        "config": {"workload": f"tank{dims[0]}x{dims[1]}x{dims[2]}_d3q{q}_{coll}_ibm{body.weights.size}",
                   "grid": list(dims), "cells": n_cells, "fluid_cells": n_fluid, "markers": int(body.weights.size),
                   "lattice": f"D3Q{q}", "collision": coll_name, "storage": storage, "nu": nu, "u_tip": 0.05,
                   "re": 2000, "smagorinsky_cs": args.les_cs,
                   "les_note": "library option; without it the reference operators diverge on this "
                               "under-resolved Re=2000 tank (D3Q27 CM at step ~2390, D3Q19 TRT at ~186); "
                               "the reference's WALE closure (lbmb_wale_update every 10 steps) also keeps "
                               "it finite but is a host-driven per-step call outside the runner loop",
                   "ibm": "3 sweeps, tol 1e-2, radius 1",
                   "top": "free-slip (specular) liquid surface" if FREE_SLIP_TOP else "solid lid (reference)",
                   "sweep_kernel": tune["kind"], "autotune": {k: tune[k] for k in
                                                              ("even_blocks_per_sm", "odd_blocks_per_sm",
                                                               "best_ms_per_step", "default_ms_per_step")}
                   | {"tuned_after_runner_steps": args.tune_after},
                   "l2": "inputs larger than L2 (populations %.0f MB)" % (q * 4 * n_cells / 1e6),
                   "parallelism": f"replicas x{world}"},
        "e2e": {"value": e2e_value, "unit": "MLUPS", "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
                "path": "C ABI per step: lbmb_runner_step (clear field, upload the host marker set, direct "
                        "forcing beside the sweep, diagnostics to the host)",
                "calls_value": e2e_calls_value,
                "calls_path": "the same step as four C ABI calls: clear_body_force_field + ibm_set_body(host "
                              "markers) + apply_rotating_ibm(diagnostics to host) + step"},
        "gpu_launches": int(13 * args.steps),
        "roofline": {"bound": "hbm", "kernel": kname, "achieved": achieved,
                     "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                     "traffic": NCU_TRAFFIC.get((kname, q, coll, storage, args.tank_T)),
                     "traffic_unit": "bytes per launch (ncu capture)", "algorithmic_bytes_per_launch": alg_bytes,
                     "peak_kind": peak_kind, "bytes_per_fluid_cell": b_lu(q, storage),
                     "launch_ms": per_launch_ms},
        "qoi": {"Np": np_head, "torque_lu_last": float(torque[-1]), "finite": bool(np.isfinite(torque).all())},
        "clocks": clk.summary() | {"window": "warm-up, timed steps, hydro-only launches and e2e loop"},
    }
    res.update(extra)
    if rank == 0 and world == 1 and not args.no_cpu:
        # the oracle's runner on the same tank from rest: timed (the CPU
        # baseline) and, as the checker, its torque series against the
        # device runner's first steps from rest in the same precision
        dims_o, solid_o, body_o, nu_o = tank_case_oracle(T=args.tank_T)
        warm = 3
        mlups, dt, tq_cpu = cpu_tank_sample(dims_o, solid_o, body_o, nu_o, q=q, collision=coll,
                                            steps=args.cpu_steps, warmup=warm, cs=args.les_cs)
        same_geo = bool(np.array_equal(solid_o, solid) and np.array_equal(body_o.positions, body.positions))
        nsteps = warm + args.cpu_steps

        def rel(a, b):
            return float(np.abs(a - b).max() / np.abs(b).max())

        # every storage precision of the device runner against the oracle
        # run in the same precision (16-bit: the oracle's storage-rounding
        # mode) and against the oracle in f64, over the same steps from rest
        oracle_tq = {storage: tq_cpu}
        for st, bits, s16 in (("f64", 64, None), ("f32", 32, None), ("f16", 32, "f16"), ("bf16", 32, "bf16")):
            if st not in oracle_tq:
                oracle_tq[st] = cpu_tank_sample(dims_o, solid_o, body_o, nu_o, q=q, collision=coll, bits=bits,
                                                steps=nsteps - 1, warmup=1, cs=args.les_cs, store16=s16)[2]
        per = {}
        for st in ("f64", "f32", "f16", "bf16"):
            g3 = make_solver(lb, dims, solid, nu, q, coll, st, args.les_cs, local)
            tq_gpu = g3.run_impeller(body, nsteps)["torque_lu"]
            g3.close()
            per[st] = {"torque_max_rel_diff_vs_oracle_same_precision": rel(tq_gpu, oracle_tq[st]),
                       "torque_max_rel_diff_vs_oracle_f64": rel(tq_gpu, oracle_tq["f64"])}
        res["cpu_baseline"] = {"value": mlups, "unit": "MLUPS", "cores": os.cpu_count(), "kind": "port",
                               "sample": f"{args.cpu_steps} runner steps of the full tank after {warm} untimed, "
                                         f"{storage}, OpenMP ({dt:.1f} s)",
                               "check": {"same_geometry_as_device": same_geo, "steps_from_rest": nsteps,
                                         "torque_max_rel_diff_vs_device": per[storage][
                                             "torque_max_rel_diff_vs_oracle_same_precision"],
                                         "per_storage": per}}
    return res


def run_reference(args, rank, world):
    """The reference's CPU path (the oracle's C++ restatement of the
    CpuScalar runner loop, OpenMP over every host core) on this arm's
    workload; geometry from the oracle's generators, so nothing of the
    product is loaded. Bounded sample: the arm's --steps (at most 40) after
    its --warmup (at most 5) untimed steps."""
    if rank != 0:
        return None
    dims, solid, body, nu = tank_case_oracle(T=args.tank_T)
    steps = max(1, min(args.steps, 40))
    q, coll = args.lattice, args.collision
    warm = max(1, min(args.warmup, 5))  # untimed runner steps before the timed sample
    mlups, dt, _ = cpu_tank_sample(dims, solid, body, nu, q=q, collision=coll, steps=steps, warmup=warm,
                                   cs=args.les_cs)
    coll_name = {"cm": "central_moment", "trt": "trt"}[coll]
    return {"impl": "reference",
            "metric": f"MLUPS (stirred-tank runner step, D3Q{q} {coll_name}, {args.storage} populations)",
            "value": mlups, "unit": "MLUPS", "n_gpus": world, "steps": steps, "warmup": warm,
            "ms_per_step": dt / steps * 1e3, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f32", "data": "synthetic (seeded tank geometry, quiescent start)",
            "config": {"workload": f"tank{dims[0]}x{dims[1]}x{dims[2]}_d3q{q}_{coll}_ibm{body.weights.size}",
                       "grid": list(dims), "smagorinsky_cs": args.les_cs,
                       "top": "free-slip (specular) liquid surface" if FREE_SLIP_TOP else "solid lid (reference)"},
            "cpu_baseline": {"value": mlups, "unit": "MLUPS", "cores": os.cpu_count(), "kind": "port",
                             "sample": f"{steps} runner steps of the full tank after {warm} untimed, on the host "
                                       f"cores (C++ restatement of the reference CpuScalar path, OpenMP; the Rust "
                                       f"reference cannot be built here) ({dt:.1f} s)"},
            "e2e": {"value": mlups, "unit": "MLUPS", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20000)
    ap.add_argument("--warmup", type=int, default=20)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--storage", default="f32", choices=["f32", "f16", "bf16"])
    ap.add_argument("--hydro-steps", type=int, default=200)
    ap.add_argument("--tune-after", type=int, default=300,
                    help="untimed runner steps before the autotuner runs (developed flow)")
    ap.add_argument("--e2e-steps", type=int, default=100)
    ap.add_argument("--tank-T", type=int, default=128, help="tank diameter in cells (128 = the benchmark case)")
    ap.add_argument("--lattice", type=int, default=27, choices=[19, 27])
    ap.add_argument("--collision", default="cm", choices=["cm", "trt"])
    ap.add_argument("--cpu-steps", type=int, default=12)
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--shear", type=int, default=1, help="stress QOI study on the final state (0: skip)")
    ap.add_argument("--ckpt", type=int, default=1, help="checkpoint save/restore study on the final state (0: skip)")
    ap.add_argument("--variants", type=int, default=1)
    ap.add_argument("--qoi-revs", type=float, default=4.0,
                    help="impeller revolutions of the precision study (Np over the last half; 0: skip)")
    ap.add_argument("--les-cs", type=float, default=0.1, help="Smagorinsky constant (0: reference operators)")
    ap.add_argument("--big-T", type=int, default=256, help="tank diameter of the throughput study")
    ap.add_argument("--big-steps", type=int, default=100, help="runner steps per form of the throughput study (0: skip)")
    ap.add_argument("--sweep-steps", type=int, default=5000, help="steps per case of the batched sweep (0: skip)")
    ap.add_argument("--adj-steps", type=int, default=2000, help="adjoint study steps (0: skip)")
    ap.add_argument("--adj-T", type=int, default=96)
    ap.add_argument("--adj-re", type=float, default=100.0)
    ap.add_argument("--adj-dirs", type=int, default=16)
    ap.add_argument("--mix-T", type=int, default=128, help="tank diameter of the mixing-time study")
    ap.add_argument("--mix-D", type=float, default=1e-3, help="scalar diffusivity of the mixing study (lattice)")
    ap.add_argument("--mix-D2", type=float, default=0.0,
                    help="second diffusivity of the mixing study (0: none; 1e-2 is added when a run at --mix-D stops)")
    ap.add_argument("--mix-steps", type=int, default=160000, help="step cap of the mixing study (0: skip)")
    ap.add_argument("--sweep-variant", default="",
                    help="with --sweep-kernel: resident blocks per SM, even/odd (e.g. 4/3)")
    ap.add_argument("--sweep-kernel", default=None, choices=["direct", "bulk", "async", "pair", "tile", "lean", "window"],
                    help="use this sweep kernel instead of the autotuner's choice")
    ap.add_argument("--lid", action="store_true", help="no-slip lid (the reference's tank) instead of a free-slip top")
    ap.add_argument("--sweep-seq-steps", type=int, default=200,
                    help="steps per case of the sequential-loop sample (0: skip)")
    args = ap.parse_args()
    global FREE_SLIP_TOP
    FREE_SLIP_TOP = not args.lid
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
