"""CPU baseline timings of the reference path (test and benchmark infrastructure only).

The reference (Fortran, gfortran + OpenMP) cannot be compiled here or on the GPU hosts:
neither has a Fortran compiler.  Its per-stage path is restated in oracle/grhd2_oracle.c;
this module times that restatement built as the reference builds itself (the reference's
Makefile:8 flags: -O3 -fopenmp -march=native -flto=auto -fno-math-errno
-fno-trapping-math, FMA contraction on), compiled on the host that runs it (`make -C
oracle stopwatch`), with OpenMP placed as the reference's campaign script places it
(inundaciones.sh:542-548: OMP_PROC_BIND=close, OMP_DYNAMIC=false).

Two measurements, each printed as one JSON line:

  run    one problem on all physical cores: zone-updates/s of the SSP-RK3 step loop
         (time loop only, after one warm-up step)
         python -m oracle.stopwatch run --problem fishbone_equatorial --keys '{...}' --seconds 15
  serve  a sample of the serving stream as concurrent single-thread processes, one per
         physical core and pinned to it (the campaign script's slots, each under its own
         taskset), each taking the next arrived request: p50/p99 time to solution and
         aggregate zone-updates/s
         python -m oracle.stopwatch serve --requests 256 --michel-final-time 2

Both run in a process of their own, so the OpenMP settings are in place before the
runtime starts.
"""
from __future__ import annotations

import argparse
import json
import multiprocessing as mp
import os
import subprocess
import sys
import time

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

FLAGS = "-O3 -fopenmp -march=native -flto=auto -fno-math-errno -fno-trapping-math (FMA contraction on)"


def host_info() -> dict:
    """Logical CPUs, model name and physical cores of this host (lscpu)."""
    info = {"nproc": os.cpu_count()}
    try:
        txt = subprocess.run(["lscpu"], capture_output=True, text=True, check=True).stdout
        kv = dict((a.strip(), b.strip()) for a, b in (ln.split(":", 1) for ln in txt.splitlines() if ":" in ln))
        info["model"] = kv.get("Model name")
        cores = int(kv.get("Core(s) per socket", "0")) * int(kv.get("Socket(s)", "1"))
        info["physical_cores"] = cores or os.cpu_count()
        info["threads_per_core"] = int(kv.get("Thread(s) per core", "1"))
    except (OSError, subprocess.CalledProcessError, ValueError):
        info["physical_cores"] = os.cpu_count()
    return info


def build() -> None:
    subprocess.run(["make", "-s", "-C", HERE, "stopwatch"], check=True)


def _omp_env(threads: int, bind: str = "close") -> None:
    os.environ["OMP_NUM_THREADS"] = str(threads)
    os.environ["OMP_PROC_BIND"] = bind
    os.environ["OMP_DYNAMIC"] = "false"


def time_run(problem: str, keys: dict, seconds: float, steps: int | None) -> dict:
    from grhd_b200.problem import Problem
    from oracle.binding import OracleRun, lib
    pb = Problem.from_keys(problem, **keys)
    p = pb.initial_prims()
    if pb.info.perturbation_type != 0 and pb.info.perturbation_time <= 0.0:
        pb.perturb(p)
    o = OracleRun(pb, p, stopwatch=True)
    o.prim_to_cons()
    o.set_boundary()
    dt = o.cfl()
    o.step(dt)  # warm-up
    n, t0 = 0, time.perf_counter()
    while True:
        o.step(dt)
        n += 1
        el = time.perf_counter() - t0
        if (steps is not None and n >= steps) or (steps is None and el >= seconds):
            break
    return {"value": pb.n_cells * n / el, "unit": "zone-updates/s", "steps": n, "seconds": el,
            "threads": int(lib(stopwatch=True).orc_num_threads()),
            "grid": f"{pb.nx}x{pb.ny}x{pb.nz}"}


# ---- serving sample -----------------------------------------------------------------
def _pin(counter, cpus):
    """Pool initializer: this worker runs on one CPU of its own (the campaign script runs
    each slot under `taskset -c`).  OpenMP binding stays off: with one thread per process
    and OMP_PROC_BIND set, every process would bind its thread to the same first place."""
    with counter.get_lock():
        k = counter.value
        counter.value += 1
    os.sched_setaffinity(0, {cpus[k % len(cpus)]})


def _solve(job):
    """One request on one thread: host set-up, then the reference time loop to its final
    time (what one single-thread reference process does for one .par file)."""
    rid, problem, keys, final_time = job
    from grhd_b200.problem import Problem
    from oracle.binding import OracleRun
    pb = Problem.from_keys(problem, **keys)
    o = OracleRun(pb, pb.initial_prims(), stopwatch=True)
    o.prim_to_cons()
    o.set_boundary()
    n, _ = o.run(0.0, final_time, -1)
    return rid, pb.n_cells * n, time.time()


def time_serve(nreq: int, seed: int, rate: float, michel_final_time: float, workers: int) -> dict:
    import numpy as np
    from grhd_b200.serve import make_stream
    reqs = make_stream(nreq, seed=seed, rate=rate, michel_final_time=michel_final_time)
    ctx = mp.get_context("spawn")
    cpus = sorted(os.sched_getaffinity(0))
    counter = ctx.Value("i", 0)
    with ctx.Pool(workers, initializer=_pin, initargs=(counter, cpus)) as pool:
        pool.map(int, range(workers))  # start the workers before the clock
        t0 = time.time()
        pending = []
        for r in reqs:
            wait = t0 + r.arrival - time.time()
            if wait > 0:
                time.sleep(wait)
            pending.append(pool.apply_async(_solve, ((r.id, r.problem, r.keys, r.final_time),)))
        done = [p.get() for p in pending]
    arr = {r.id: t0 + r.arrival for r in reqs}
    tts = np.array([d - arr[rid] for rid, _, d in done])
    zu = sum(z for _, z, _ in done)
    span = max(d for _, _, d in done) - t0
    return {"requests": nreq, "zone_updates": int(zu), "makespan_s": span, "zone_updates_per_s": zu / span,
            "tts_p50_s": float(np.percentile(tts, 50)), "tts_p99_s": float(np.percentile(tts, 99)),
            "tts_mean_s": float(tts.mean()), "processes": workers, "threads_per_process": 1,
            "pinning": "one CPU per process (sched_setaffinity)",
            "sample": f"{nreq} requests of the stream (seed {seed}), {rate:g} arrivals/s, "
                      f"Michel final time {michel_final_time:g} M"}


def main(argv=None):
    ap = argparse.ArgumentParser(description=__doc__.split("\n")[0])
    sub = ap.add_subparsers(dest="cmd", required=True)
    a = sub.add_parser("run")
    a.add_argument("--problem", required=True)
    a.add_argument("--keys", required=True, help="JSON object of .par keys")
    a.add_argument("--seconds", type=float, default=15.0)
    a.add_argument("--steps", type=int, default=None)
    a.add_argument("--threads", type=int, default=0, help="0: all physical cores")
    s = sub.add_parser("serve")
    s.add_argument("--requests", type=int, default=256)
    s.add_argument("--seed", type=int, default=20260901)
    s.add_argument("--rate", type=float, default=2000.0)
    s.add_argument("--michel-final-time", type=float, default=2.0)
    s.add_argument("--processes", type=int, default=0, help="0: one per physical core")
    for p in (a, s):
        p.add_argument("--no-build", action="store_true")
    args = ap.parse_args(argv)
    host = host_info()
    if not args.no_build:
        build()
    if args.cmd == "run":
        threads = args.threads or host["physical_cores"]
        _omp_env(threads)
        out = time_run(args.problem, json.loads(args.keys), args.seconds, args.steps)
    else:
        _omp_env(1, bind="false")
        out = time_serve(args.requests, args.seed, args.rate, args.michel_final_time,
                         args.processes or host["physical_cores"])
    out.update(host=host, flags=FLAGS, omp={k: os.environ[k] for k in ("OMP_NUM_THREADS", "OMP_PROC_BIND",
                                                                        "OMP_DYNAMIC")},
               binary="oracle restatement of the reference path (the reference is Fortran; no Fortran "
                      "compiler on this host)")
    print(json.dumps(out), flush=True)


if __name__ == "__main__":
    main()
