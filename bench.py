#!/usr/bin/env python
"""Benchmark of the B200 per-stage path: zone-updates/s of the SSP-RK3 step.

Workload (N=1): the 2.5D equatorial Fishbone-Moncrief torus in Kerr-Schild coordinates
(a = 0.9), log-r spheroidal grid 400 x 1 x 200, WENO5 + HLLE, r_in 6, r_max 12, Gamma 4/3,
1% seeded pressure noise -- synthetic initial data of the configuration's shape.  One
"step" is one full SSP-RK3 step (3 RHS evaluations, stage combinations, con2prim sweeps
and boundary fills) of the whole grid.  The headline value is the FP64 path (the parity
path); the mixed FP32/FP64 policy is reported beside it with its L1 against FP64.

Multi-GPU: one process per GPU (torchrun), each rank advances its own replica of the
workload ("replicas only": the reference path does not shard); the value is the
whole-job zone-updates/s, timed on the device as the max over ranks.

``--impl reference`` times the reference's CPU implementation of the path on the host
cores instead: the reference (Fortran) cannot be compiled in this image (no gfortran),
so its restatement in oracle/ is timed, with all host threads.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "zone-updates/s per SSP-RK3 step, FP32-mixed vs FP64 at stated L1; serve p50/p99"
WORKLOAD = "2.5D Kerr-Schild FM torus 400x1x200, WENO5+HLLE, a=0.9, r_in=6, r_max=12, Gamma=4/3"


def torus_problem(nx=400, nz=200):
    from grhd_b200.problem import Problem
    keys = dict(metric="kerr_schild", geometry="spheroidal", logarithmic_r=True, spin=0.9, bh_mass=1.0,
                nx=nx, ny=1, nz=nz, r_min=1.2, r_max=40.0, theta_min=0, theta_max=1, phi_min=0,
                phi_max=2, fm_inner_radius=6.0, fm_pressure_max_radius=12.0,
                fm_polytropic_constant=0.0015, adiabatic_index=1.3333333333333333,
                reconstruction="weno5", riemann_solver="hlle", shock_sensor=False, cfl=0.4,
                perturbation="pressure_noise", perturbation_amplitude=0.01, perturbation_time=0.0,
                perturbation_seed=3435)
    return Problem.from_keys("fishbone_equatorial", **keys)


def initial_state(pb):
    p = pb.initial_prims()
    pb.perturb(p)
    return p


# ------------------------------------------------------------------------------------
def dist_env():
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return rank, world, local


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled every 200 ms during the timed region."""

    FIELDS = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.gpu = gpu_index
        self.proc = None
        self.lines = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.gpu), f"--query-gpu={self.FIELDS}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except (FileNotFoundError, OSError):
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *a):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        sm, mx, reasons = [], None, set()
        names = ("hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap")
        for ln in self.lines:
            parts = [x.strip() for x in ln.split(",")]
            if len(parts) < 8:
                continue
            try:
                sm.append(float(parts[0]))
                mx = float(parts[1])
            except ValueError:
                continue
            for nm, val in zip(names, parts[4:8]):
                if val.lower() == "active":
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx,
                "reasons": sorted(reasons), "samples": len(sm)}


def measured_peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        with open(path) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def kernel_bytes(name: str, pb, mixed: bool) -> float:
    """Algorithmic DRAM bytes of one launch: every cell's state read or written once,
    every face flux written once by face_flux and read once by cell_update.  Metric
    tables (k-invariant, L2-resident) and stencil re-reads are excluded."""
    nx, ny, nz = pb.nx, pb.ny, pb.nz
    n = nx * ny * nz
    ep = 4 if mixed else 8   # primitive / flux element size
    nf = {"x": (nx + 1) * ny * nz, "y": nx * (ny + 1) * nz, "z": nx * ny * (nz + 1)}
    if name.startswith("face_flux_"):
        return 5 * ep * n + 5 * ep * nf[name[-1]]
    if name == "cell_update":
        flux_read = 5 * ep * (nf["x"] + (nf["y"] if ny > 1 else 0) + (nf["z"] if nz > 1 else 0))
        # P read+write, up read+write, u read (stages 2,3) or write (stage 1)
        return 2 * 5 * ep * n + 3 * 5 * 8 * n + flux_read
    return 0.0


# ------------------------------------------------------------------------------------
def run_ours(args):
    import torch
    import torch.distributed as dist
    from grhd_b200.solver import GpuGrid

    rank, world, local = dist_env()
    torch.cuda.set_device(local)
    if world > 1:
        dist.init_process_group("nccl", timeout=__import__("datetime").timedelta(seconds=120))
    pb = torus_problem()
    p0 = initial_state(pb)
    ncell = pb.n_cells
    l2_flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device="cuda")

    def timed_run(precision):
        g = GpuGrid(pb, precision=precision, upload_initial=False)
        g.upload(p=p0)
        g.prim_to_cons()
        dt = g.cfl()
        ext = torch.cuda.ExternalStream(g.stream_ptr)
        for _ in range(args.warmup):
            g.step(dt)
        g.synchronize()
        evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize()
        for s in range(args.steps):
            with torch.cuda.stream(ext):
                l2_flush.zero_()  # evict the ~20 MB working set from the 126 MB L2
            evs[s][0].record(ext)
            g.step(dt)
            evs[s][1].record(ext)
        g.synchronize()
        torch.cuda.synchronize()
        ms = sum(a.elapsed_time(b) for a, b in evs)
        if world > 1:
            t = torch.tensor([ms], device="cuda")
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
            ms = float(t.item())
        return g, dt, ms

    with ClockSampler(local) as clk:
        g64, dt, ms64 = timed_run("fp64")
    clocks = clk.summary()
    gmx, _, msmx = timed_run("mixed")
    # L1 of the mixed policy against FP64 after the same steps from the same state
    up64, _ = g64.download()
    upmx, _ = gmx.download()
    den = np.abs(up64.reshape(-1, 5)).sum(axis=0)
    l1_mixed = (np.abs(upmx - up64).reshape(-1, 5).sum(axis=0) / den).tolist()

    # per-kernel durations of one step (outside the timed region) -> dominant kernel
    prof = {}
    for _ in range(3):
        for name, t in g64.profile_step(dt):
            prof.setdefault(name, []).append(t)
    per_step = {k: sum(v) / 3.0 for k, v in prof.items()}
    launches = {k: len(v) // 3 for k, v in prof.items()}
    dom = max(per_step, key=per_step.get)
    dom_ms = per_step[dom] / launches[dom]
    dom_bytes = kernel_bytes(dom, pb, False)
    peak, peak_kind = measured_peaks()
    achieved = dom_bytes / (dom_ms * 1e-3) / 1e9
    traffic = None
    tr_path = os.path.join(ROOT, "profiles", "traffic.json")
    if os.path.exists(tr_path):
        with open(tr_path) as f:
            traffic = json.load(f).get(dom)

    # end to end through the C-ABI with host buffers (pinned), copies inside the timed region
    pin_p = torch.from_numpy(p0.copy()).pin_memory()
    pin_up = torch.empty(pb.cons_shape, dtype=torch.float64).pin_memory()
    g_e = GpuGrid(pb, precision="fp64", upload_initial=False)
    g_e.upload(p=p0)
    g_e.prim_to_cons()
    up_e, _ = g_e.download()
    pin_up.numpy()[...] = up_e
    ext = torch.cuda.ExternalStream(g_e.stream_ptr)
    h2d = pin_up.numel() * 8 + pin_p.numel() * 8
    lib, h = g_e.lib, g_e._h
    from grhd_b200 import native as N
    pu, pp = N.dptr(pin_up.numpy()), N.dptr(pin_p.numpy())
    for _ in range(args.warmup):
        lib.grhd2_gpu_upload(h, pu, pp)
        lib.grhd2_gpu_step(h, dt)
        lib.grhd2_gpu_download(h, pu, pp)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(ext)
    for _ in range(args.steps):
        assert lib.grhd2_gpu_upload(h, pu, pp) == 0
        assert lib.grhd2_gpu_step(h, dt) == 0
        assert lib.grhd2_gpu_download(h, pu, pp) == 0
    e1.record(ext)
    torch.cuda.synchronize()
    ms_e = e0.elapsed_time(e1)
    if world > 1:
        t = torch.tensor([ms_e], device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms_e = float(t.item())

    value = world * ncell * args.steps / (ms64 * 1e-3)
    out = {
        "metric": METRIC, "value": value, "unit": "zone-updates/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms64 / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic (analytic torus initial data, seeded pressure noise)",
        "config": {"workload": WORKLOAD, "nx": pb.nx, "ny": pb.ny, "nz": pb.nz, "cells": ncell,
                   "precision": "fp64 (parity path, no FMA)", "parallelism": f"replicas x{world}",
                   "l2": "256 MB buffer written between timed steps (working set ~20 MB < L2)"},
        "variants": {"mixed": {"value": world * ncell * args.steps / (msmx * 1e-3),
                               "ms_per_step": msmx / args.steps, "dtype": "f32 recon/Riemann/sources, f64 con2prim + RK",
                               "l1_vs_fp64": l1_mixed}},
        "clocks": clocks,
        "e2e": {"value": world * ncell * args.steps / (ms_e * 1e-3), "unit": "zone-updates/s",
                "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": h2d,
                "path": "grhd2_gpu_upload(up,p) + grhd2_gpu_step + grhd2_gpu_download(up,p), pinned host buffers"},
        "gpu_launches": sum(launches.values()) * args.steps,
        "kernels_ms_per_step": per_step,
        "roofline": {"bound": "hbm", "kernel": dom, "achieved": achieved, "peak": peak, "unit": "GB/s",
                     "frac": achieved / peak, "traffic": traffic, "peak_kind": peak_kind,
                     "algorithmic_bytes_per_launch": dom_bytes, "launch_ms": dom_ms},
    }
    if rank == 0 and not args.no_cpu_baseline:
        out["cpu_baseline"] = cpu_baseline(pb, p0, max_seconds=args.cpu_seconds)
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()
    if rank == 0:
        print(json.dumps(out), flush=True)


def cpu_baseline(pb, p0, max_seconds=15.0, steps=None):
    """The oracle (plain-C restatement of the reference path) on the host cores."""
    from oracle.binding import OracleRun, lib
    o = OracleRun(pb, p0)
    o.prim_to_cons()
    o.set_boundary()
    dt = o.cfl()
    o.step(dt)  # warm-up
    n, t0 = 0, time.perf_counter()
    while True:
        o.step(dt)
        n += 1
        el = time.perf_counter() - t0
        if (steps is not None and n >= steps) or (steps is None and el >= max_seconds):
            break
    return {"value": pb.n_cells * n / el, "unit": "zone-updates/s", "cores": int(lib().orc_num_threads()),
            "kind": "port", "sample": f"{n} RK3 steps of the {pb.nx}x{pb.ny}x{pb.nz} torus ({el:.1f} s)"}


def run_reference(args):
    rank, world, local = dist_env()
    if rank != 0:
        return
    pb = torus_problem()
    p0 = initial_state(pb)
    base = cpu_baseline(pb, p0, steps=args.steps)
    out = {"metric": METRIC, "value": base["value"], "unit": "zone-updates/s", "n_gpus": world,
           "steps": args.steps, "warmup": args.warmup, "ms_per_step": pb.n_cells / base["value"] * 1e3,
           "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
           "data": "synthetic (analytic torus initial data, seeded pressure noise)", "impl": "reference",
           "config": {"workload": WORKLOAD, "nx": pb.nx, "ny": pb.ny, "nz": pb.nz,
                      "note": "reference Fortran not buildable here (no gfortran); its C restatement (oracle/) "
                              "timed with all host threads"},
           "cpu_baseline": base,
           "e2e": {"value": base["value"], "unit": "zone-updates/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(out), flush=True)


def main():
    ap = argparse.ArgumentParser(description=__doc__.split("\n")[0])
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--cpu-seconds", type=float, default=15.0)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    if args.impl == "reference":
        run_reference(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
