#!/usr/bin/env python
"""Benchmark of the B200 per-stage path: zone-updates/s of the SSP-RK3 step.

Workload (N=1): the 2.5D equatorial Fishbone-Moncrief torus in Kerr-Schild coordinates
(a = 0.9), log-r spheroidal grid 400 x 1 x 200, WENO5 + HLLE, r_in 6, r_max 12, Gamma 4/3,
1% seeded pressure noise -- synthetic initial data of the configuration's shape.  A batch
of --batch such grids (default 32, one perturbation seed each) steps together: one launch
per kernel kind for all of them, each step replayed as one CUDA graph.  One "step" is one
full SSP-RK3 step (3 RHS evaluations, stage combinations, con2prim sweeps and boundary
fills) of every grid of the batch.  The headline value is the FP64 path (the parity
path); the mixed FP32/FP64 policy and a single grid alone are reported beside it.

Multi-GPU: one process per GPU (torchrun), each rank advances its own batch
("replicas only": the grids are independent, nothing is exchanged); the value is the
whole-job zone-updates/s, timed on the device as the max over ranks.

``--impl reference`` times the reference's CPU implementation of the path on the host
cores instead: the reference (Fortran) cannot be compiled here or on the GPU hosts (no
Fortran compiler), so its restatement in oracle/ is timed, built on the timing host with
the reference's own optimisation flags and run on all physical cores (oracle/stopwatch.py).
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


TORUS_KEYS = dict(metric="kerr_schild", geometry="spheroidal", logarithmic_r=True, spin=0.9, bh_mass=1.0,
                  nx=400, ny=1, nz=200, r_min=1.2, r_max=40.0, theta_min=0, theta_max=1, phi_min=0,
                  phi_max=2, fm_inner_radius=6.0, fm_pressure_max_radius=12.0,
                  fm_polytropic_constant=0.0015, adiabatic_index=1.3333333333333333,
                  reconstruction="weno5", riemann_solver="hlle", shock_sensor=False, cfl=0.4,
                  perturbation="pressure_noise", perturbation_amplitude=0.01, perturbation_time=0.0,
                  perturbation_seed=3435)


def torus_problem(nx=400, nz=200, seed=3435):
    from grhd_b200.problem import Problem
    keys = dict(TORUS_KEYS, nx=nx, nz=nz, perturbation_seed=seed)
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


def reduce_max(value: float, world: int, device: str = "cuda") -> float:
    """Maximum of a per-rank value over all ranks (the job's time is its slowest rank)."""
    if world <= 1:
        return value
    import torch
    import torch.distributed as dist
    t = torch.tensor([value], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


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


STAGE_BYTES_PER_ZONE = {"fp64": 200.0, "mixed": 160.0}
"""Algorithmic bytes of one cell through one RK stage: read P, u, up and write up, P, five
values each.  FP64: 5 x 8 x 5 = 200 B.  Mixed policy: P in FP32, u and up in FP64,
20 + 40 + 40 + 40 + 20 = 160 B.  Face fluxes, interface states, metric tables (k-invariant,
L2-resident), halo re-reads, ghosts and counters are not algorithmic bytes."""
STEP_BYTES_PER_ZONE = {k: 3.0 * v for k, v in STAGE_BYTES_PER_ZONE.items()}
"""Per zone-update (a cell through a full SSP-RK3 step): FP64 600 B, mixed 480 B."""


def kernel_bytes(name: str, pb, mixed: bool) -> float:
    """Algorithmic DRAM bytes of one launch for one grid.  The cell update (or a kernel that
    runs a whole stage) counts the stage's algorithmic bytes, STAGE_BYTES_PER_ZONE per cell;
    a face kernel counts P read once and what it must write (q_L, q_R or the fluxes)."""
    nx, ny, nz = pb.nx, pb.ny, pb.nz
    n = nx * ny * nz
    ep = 4 if mixed else 8   # primitive / interface / flux element size
    nf = {"x": (nx + 1) * ny * nz, "y": nx * (ny + 1) * nz, "z": nx * ny * (nz + 1)}
    if name.startswith("recon_"):
        return 5 * ep * n + 10 * ep * nf[name[-1]]
    if name.startswith("riemann_"):
        return 15 * ep * nf[name[-1]]
    if name.startswith("flux_"):  # fused recon + Riemann: reads P, writes the face fluxes
        return 5 * ep * n + 5 * ep * nf[name[-1]]
    if name in ("cell_update", "stage"):
        return STAGE_BYTES_PER_ZONE["mixed" if mixed else "fp64"] * n
    return 0.0


# ------------------------------------------------------------------------------------
def make_batch(nbatch, precision, stream, seed0=3435):
    """nbatch torus grids (perturbation seeds seed0, seed0+1, ...) on one stream, each
    running on its own device clock with its CFL dt."""
    from grhd_b200.solver import GpuBatch, GpuGrid
    grids = []
    for r in range(nbatch):
        pb = torus_problem(seed=seed0 + r)
        g = GpuGrid(pb, precision=precision, upload_initial=False, stream=stream.cuda_stream)
        g.upload(p=initial_state(pb))
        g.prim_to_cons()
        grids.append(g)
    b = GpuBatch(grids)
    for k in range(nbatch):
        b.set_clock(k, 0.0, 1e300, -1)
    b.tuned = b.autotune(reps=5)  # flux kernel variant per direction, timed on this batch
    return grids, b


def close_batch(grids, b):
    b.close()
    for g in grids:
        g.close()


def run_ours(args):
    import torch
    import torch.distributed as dist

    rank, world, local = dist_env()
    torch.cuda.set_device(local)
    if world > 1:
        dist.init_process_group("nccl", timeout=__import__("datetime").timedelta(seconds=120))
    pb = torus_problem()
    ncell = pb.n_cells
    stream = torch.cuda.Stream()
    l2_flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device="cuda")

    def max_over_ranks(ms):
        return reduce_max(ms, world, "cuda")

    def timed(b, flush, tag):
        """ms of args.steps batched steps (graph replays), CUDA events on the batch's stream."""
        b.step(args.warmup, graph=True)
        torch.cuda.synchronize()
        evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize()
        torch.cuda.nvtx.range_push(f"timed_{tag}")  # lets a profiler select the timed launches
        for s in range(args.steps):
            if flush:
                with torch.cuda.stream(stream):
                    l2_flush.zero_()
            evs[s][0].record(stream)
            b.step(1, graph=True)
            evs[s][1].record(stream)
        torch.cuda.nvtx.range_pop()
        torch.cuda.synchronize()
        return max_over_ranks(sum(a.elapsed_time(c) for a, c in evs))

    nb = args.batch
    with ClockSampler(local) as clk:
        g64, b64 = make_batch(nb, "fp64", stream)
        ms64 = timed(b64, flush=False, tag="fp64_batched")
    clocks = clk.summary()
    gmx, bmx = make_batch(nb, "mixed", stream)
    msmx = timed(bmx, flush=False, tag="mixed_batched")
    # L1 of the mixed policy against FP64 after the same steps from the same state
    up64 = g64[0].download(want_p=False)[0]
    upmx = gmx[0].download(want_p=False)[0]
    den = np.abs(up64.reshape(-1, 5)).sum(axis=0)
    num = np.abs(upmx - up64).reshape(-1, 5).sum(axis=0)
    # a variable that is zero everywhere (S_y of the equatorial torus) reports its absolute L1
    l1_mixed = np.where(den > 0, num / np.where(den > 0, den, 1.0), num).tolist()
    n_done = b64.clock(0)[1]
    b64_tuned, bmx_tuned = b64.tuned, bmx.tuned
    close_batch(gmx, bmx)

    # one grid alone (L2 flushed between steps: its ~22 MB working set fits in L2)
    singles = {}
    for prec in ("fp64", "mixed"):
        gs, bs = make_batch(1, prec, stream)
        ms = timed(bs, flush=True, tag=f"{prec}_single")
        singles[prec] = {"value": world * ncell * args.steps / (ms * 1e-3), "ms_per_step": ms / args.steps}
        close_batch(gs, bs)

    # per-kernel durations of one batched step (outside the timed region) -> dominant kernel
    prof = {}
    reps = 3
    for _ in range(reps):
        for name, t in b64.profile_step():
            prof.setdefault(name, []).append(t)
    per_step = {k: sum(v) / reps for k, v in prof.items()}
    launches = {k: len(v) // reps for k, v in prof.items()}
    dom = max(per_step, key=per_step.get)
    dom_ms = per_step[dom] / launches[dom]
    # every grid passes through each stage kernel once per stage (three times a step); a
    # large scheme group runs as two halves, each launched separately
    grids_per_launch = 3 * nb / launches[dom]
    dom_bytes = kernel_bytes(dom, pb, False) * grids_per_launch
    peak, peak_kind = measured_peaks()
    achieved = dom_bytes / (dom_ms * 1e-3) / 1e9
    traffic = None
    tr_path = os.path.join(ROOT, "profiles", "traffic.json")
    if os.path.exists(tr_path):
        with open(tr_path) as f:
            tr = json.load(f).get("torus2p5d_400x1x200", {}).get(dom)
        traffic = tr * grids_per_launch if tr is not None else None

    close_batch(g64, b64)

    # End to end through the C-ABI with page-locked host buffers: every step uploads each
    # grid's conserved state, recovers the primitives (one launch per sub-batch), steps,
    # and downloads the conserved state.  The grids are split into sub-batches on their own
    # streams and every call is asynchronous, so one sub-batch's copies overlap another's
    # kernels.
    from grhd_b200 import native as N
    nsub = max(1, min(args.e2e_streams, nb))
    subs = []
    for q in range(nsub):
        st = torch.cuda.Stream()
        grids, bq = make_batch(len(range(q, nb, nsub)), "fp64", st, seed0=3435 + 1000 * (q + 1))
        subs.append((st, grids, bq))
    lib = subs[0][1][0].lib
    pins, work = [], []
    for st, grids, bq in subs:
        for g in grids:
            up = torch.empty(pb.cons_shape, dtype=torch.float64).pin_memory()
            up.numpy()[...] = g.download(want_p=False)[0]
            pins.append(up)
            work.append(N.dptr(up.numpy()))
    h2d = sum(u.numel() * 8 for u in pins)

    def e2e_step():
        k = 0
        for st, grids, bq in subs:
            ptrs = work[k:k + len(grids)]
            for g, pu in zip(grids, ptrs):
                assert lib.grhd2_gpu_upload_async(g._h, pu, None) == 0
            assert lib.grhd2_gpu_batch_cons_to_prim(bq._b) == 0
            bq.step(1, graph=True)
            for g, pu in zip(grids, ptrs):
                assert lib.grhd2_gpu_download_async(g._h, pu, None) == 0
            k += len(grids)

    for _ in range(args.warmup):
        e2e_step()
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for st, _, _ in subs:
        st.wait_event(e0)
    for _ in range(args.steps):
        e2e_step()
    for st, _, _ in subs:
        ev = torch.cuda.Event()
        ev.record(st)
        stream.wait_event(ev)
    e1.record(stream)
    torch.cuda.synchronize()
    ms_e = max_over_ranks(e0.elapsed_time(e1))
    for st, grids, bq in subs:
        close_batch(grids, bq)

    value = world * nb * ncell * args.steps / (ms64 * 1e-3)
    mixed_value = world * nb * ncell * args.steps / (msmx * 1e-3)
    out = {
        "metric": METRIC, "value": value, "unit": "zone-updates/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms64 / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic (analytic torus initial data, seeded pressure noise, one seed per grid)",
        "config": {"workload": WORKLOAD, "grids_per_gpu": nb, "nx": pb.nx, "ny": pb.ny, "nz": pb.nz,
                   "cells_per_gpu": nb * ncell, "precision": "fp64 (parity path, no FMA)",
                   "parallelism": f"replicas x{world}", "graph": "one CUDA graph per batched step",
                   "flux_variant_xz": b64_tuned, "flux_variant_xz_mixed": bmx_tuned,
                   "l2": f"inputs larger than L2: {nb} grids x ~22 MB resident state, no flush"},
        "variants": {
            "mixed_batched": {"value": mixed_value, "ms_per_step": msmx / args.steps,
                              "dtype": "f32 recon/Riemann/sources, f64 con2prim + RK",
                              "l1_vs_fp64": l1_mixed, "steps_compared": n_done,
                              "speedup_vs_fp64_batched": mixed_value / value,
                              "speedup_vs_fp64_single": mixed_value / singles["fp64"]["value"]},
            "fp64_single_grid": dict(singles["fp64"], l2="256 MB buffer written between timed steps"),
            "mixed_single_grid": dict(singles["mixed"], l2="256 MB buffer written between timed steps"),
        },
        "clocks": clocks,
        "e2e": {"value": world * nb * ncell * args.steps / (ms_e * 1e-3), "unit": "zone-updates/s",
                "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": h2d,
                "path": f"the {nb} grids in {nsub} sub-batches on their own streams; per step "
                        "grhd2_gpu_upload_async(up) per grid, grhd2_gpu_batch_cons_to_prim and "
                        "grhd2_gpu_batch_step per sub-batch, grhd2_gpu_download_async(up) per grid; "
                        "page-locked host buffers"},
        "gpu_launches": sum(launches.values()) * args.steps,
        "kernels_ms_per_step": per_step,
        "roofline": {"bound": "hbm", "kernel": dom, "achieved": achieved, "peak": peak, "unit": "GB/s",
                     "frac": achieved / peak, "traffic": traffic, "peak_kind": peak_kind,
                     "algorithmic_bytes_per_launch": dom_bytes, "launch_ms": dom_ms,
                     "grids_per_launch": grids_per_launch,
                     "step": {"bytes_per_zone_update": STEP_BYTES_PER_ZONE["fp64"],
                              "achieved": STEP_BYTES_PER_ZONE["fp64"] * value / world / 1e9,
                              "frac": STEP_BYTES_PER_ZONE["fp64"] * value / world / 1e9 / peak,
                              "mixed_bytes_per_zone_update": STEP_BYTES_PER_ZONE["mixed"],
                              "mixed_achieved": STEP_BYTES_PER_ZONE["mixed"] * mixed_value / world / 1e9,
                              "mixed_frac": STEP_BYTES_PER_ZONE["mixed"] * mixed_value / world / 1e9 / peak}},
    }
    if args.serve_requests > 0:
        out["serve"] = run_serve(args)
        out["serve_mixed"] = run_serve(args, "mixed")
    if rank == 0 and not args.no_cpu_baseline:
        out["cpu_baseline"] = cpu_baseline(max_seconds=args.cpu_seconds)
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()
    if rank == 0:
        print(json.dumps(out), flush=True)


def run_serve(args, precision="fp64"):
    """A bounded sample of the serving stream (Poisson arrivals, 70 % Riemann problems of
    128-8192 cells to t = 0.4, 30 % Michel runs of 512-4096 cells) through the
    continuous-batching server on this GPU: time to solution p50/p99 and zone-updates/s.
    The host's load and CPU are recorded beside it: the server's host work (grid set-up,
    batch rebuilds) shares the host cores, and the sample's figures move with them."""
    from grhd_b200.serve import GpuEngine, SolveServer, make_stream, summarize
    reqs = make_stream(args.serve_requests, seed=20260901, rate=args.serve_rate,
                       michel_final_time=args.serve_michel_final_time)
    load0 = os.getloadavg()
    eng = GpuEngine(precision, metric=args.serve_metric)
    srv = SolveServer(eng, steps_per_round=16)
    res = srv.run(reqs)
    eng.close()
    out = summarize(res)
    out.update(peak_active=srv.peak_active, rounds=srv.rounds, batch_rebuilds=srv.rebuilds,
               host_s={k: round(v, 3) for k, v in {**srv.host_s, **eng.host_s}.items()},
               host={"nproc": os.cpu_count(), "loadavg_1min_before": round(load0[0], 2),
                     "loadavg_1min_after": round(os.getloadavg()[0], 2)},
               sample=f"{args.serve_requests} requests of the 4096-request stream (seed 20260901), "
                      f"{args.serve_rate:g} arrivals/s, Michel final time {args.serve_michel_final_time:g} M, "
                      f"{precision}, metric tables built on the {args.serve_metric}",
               timing="wall clock from each arrival to its result on the host")
    return out


def cpu_baseline(max_seconds=15.0, steps=None):
    """The reference path on the host cores: its restatement in oracle/, built with the
    reference's own optimisation flags on this host and run on all physical cores with
    OMP_PROC_BIND=close, in a process of its own (oracle/stopwatch.py)."""
    cmd = [sys.executable, "-m", "oracle.stopwatch", "run", "--problem", "fishbone_equatorial",
           "--keys", json.dumps(TORUS_KEYS), "--seconds", str(max_seconds)]
    if steps is not None:
        cmd += ["--steps", str(steps)]
    r = subprocess.run(cmd, cwd=ROOT, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"CPU baseline failed: {r.stderr[-2000:]}")
    d = json.loads(r.stdout.strip().splitlines()[-1])
    return {"value": d["value"], "unit": "zone-updates/s", "cores": d["threads"], "kind": "port",
            "sample": f"{d['steps']} RK3 steps of the {d['grid']} torus ({d['seconds']:.1f} s)",
            "host": d["host"], "flags": d["flags"], "omp": d["omp"], "binary": d["binary"]}


def run_reference(args):
    rank, world, local = dist_env()
    if rank != 0:
        return
    pb = torus_problem()
    base = cpu_baseline(steps=args.steps)
    out = {"metric": METRIC, "value": base["value"], "unit": "zone-updates/s", "n_gpus": world,
           "steps": args.steps, "warmup": args.warmup, "ms_per_step": pb.n_cells / base["value"] * 1e3,
           "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
           "data": "synthetic (analytic torus initial data, seeded pressure noise)", "impl": "reference",
           "config": {"workload": WORKLOAD, "nx": pb.nx, "ny": pb.ny, "nz": pb.nz,
                      "note": "the reference is Fortran and no Fortran compiler exists on this host or "
                              "the build host; its C restatement (oracle/) is timed, built with the "
                              "reference's flags on this host, all physical cores"},
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
    ap.add_argument("--batch", type=int, default=32, help="torus grids per GPU stepped as one batch")
    ap.add_argument("--e2e-streams", type=int, default=8, help="sub-batches (streams) of the end-to-end pipeline")
    ap.add_argument("--serve-requests", type=int, default=256, help="serving sample size (0: skip)")
    ap.add_argument("--serve-rate", type=float, default=2000.0)
    ap.add_argument("--serve-michel-final-time", type=float, default=2.0)
    ap.add_argument("--serve-metric", choices=["host", "device"], default="host",
                    help="where the serving sample builds each request's metric tables")
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
