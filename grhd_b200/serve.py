"""Continuous-batching solve server: many independent 1D solves resident on one GPU.

Requests (shock-tube Riemann problems and Michel accretion runs of varying size) arrive
over time.  The server admits a waiting request as soon as its device memory fits in the
budget (first come, first served), prepares its grid on a private CUDA stream while the
resident grids keep stepping, and then moves it onto the batch stream.  Every round
enqueues K batched SSP-RK3 steps of all resident grids (one launch per kernel kind and
scheme group, replayed as a CUDA graph); each grid runs on its own device clock and stops
by itself at its final time.  After the round the server reads every clock in one
transfer, retires finished grids (result downloaded, memory released) and rebuilds the
batch if its membership changed.  State never leaves the device between steps.

The reference runs such sweeps as independent processes (one Fortran run per problem,
``inundaciones.sh``); a grid's result here is the result it has alone (FP64: bitwise).

    python -m grhd_b200.serve --requests 4096 --rate 2000 --michel-final-time 50
"""
from __future__ import annotations

import argparse
import collections
import concurrent.futures
import dataclasses
import json
import math
import sys
import time

import numpy as np

RIEMANN_FINAL_TIME = 0.4


@dataclasses.dataclass
class Request:
    id: int
    kind: str            # "riemann" or "michel"
    arrival: float       # seconds after the stream starts
    problem: str         # reference problem name
    keys: dict           # .par keys
    cells: int
    final_time: float


def make_stream(n: int = 4096, seed: int = 20260901, rate: float = 2000.0, michel_final_time: float = 50.0,
                riemann_final_time: float = RIEMANN_FINAL_TIME, riemann_cells=(128, 8192),
                michel_cells=(512, 4096)) -> list[Request]:
    """Seeded request stream: Poisson arrivals at `rate` per second; 70 % Minkowski
    Riemann problems (cells log-uniform in riemann_cells, rho_L, rho_R log-uniform in
    [0.1, 10], p log-uniform in [1e-3, 100], v uniform in [-0.9, 0.9], Gamma 4/3 or 5/3,
    WENO5 or MP5, HLLE or HLLC, x in [0, 1], to t = 0.4) and 30 % Michel accretion onto
    Schwarzschild (cells log-uniform in michel_cells, the Michel preset: ingoing EF,
    log r in [1.8, 20], Gamma 4/3, sonic radius 8, MP5 + HLLE)."""
    rng = np.random.default_rng(seed)
    out = []
    t = 0.0
    for i in range(n):
        t += rng.exponential(1.0 / rate)
        if rng.random() < 0.7:
            lo, hi = riemann_cells
            cells = int(round(math.exp(rng.uniform(math.log(lo), math.log(hi)))))
            lr = lambda a, b: float(math.exp(rng.uniform(math.log(a), math.log(b))))  # noqa: E731
            keys = dict(nx=cells, adiabatic_index=[1.3333333333333333, 1.6666666666666667][int(rng.integers(2))],
                        sod_interface=0.5, sod_density_left=lr(0.1, 10), sod_density_right=lr(0.1, 10),
                        sod_pressure_left=lr(1e-3, 100), sod_pressure_right=lr(1e-3, 100),
                        sod_velocity_left=float(rng.uniform(-0.9, 0.9)),
                        sod_velocity_right=float(rng.uniform(-0.9, 0.9)),
                        reconstruction=["weno5", "mp5"][int(rng.integers(2))],
                        riemann_solver=["hlle", "hllc"][int(rng.integers(2))], cfl=0.4,
                        final_time=riemann_final_time, shock_sensor=False)
            out.append(Request(i, "riemann", t, "sod", keys, cells, riemann_final_time))
        else:
            lo, hi = michel_cells
            cells = int(round(math.exp(rng.uniform(math.log(lo), math.log(hi)))))
            keys = dict(metric="eddington_finkelstein", geometry="spherical", logarithmic_r=True, bh_mass=1.0,
                        nx=cells, ny=1, nz=1, r_min=1.8, r_max=20.0, adiabatic_index=1.3333333333333333,
                        michel_critical_radius=8.0, reconstruction="mp5", riemann_solver="hlle",
                        final_time=michel_final_time, shock_sensor=False)
            out.append(Request(i, "michel", t, "michel", keys, cells, michel_final_time))
    return out


@dataclasses.dataclass
class Result:
    id: int
    kind: str
    cells: int
    arrival: float
    admitted: float
    done: float
    steps: int
    t: float
    up: np.ndarray | None = None

    @property
    def time_to_solution(self) -> float:
        return self.done - self.arrival


# ------------------------------------------------------------------------------------
class GpuEngine:
    """Grids and batches on the GPU through the C-ABI (grhd_b200.solver).

    The host-side set-up of a request (grid, metric tables, initial data: milliseconds of
    host work per request) runs on a pool of host threads from the moment the request
    arrives, so admission only waits for it when it has not finished yet."""

    def __init__(self, precision: str = "fp64", device: int = 0, host_workers: int = 8, metric: str = "host"):
        """metric: "host" builds each request's metric cache with its host set-up and
        uploads it; "device" leaves it out of the host set-up and builds the tables on the
        GPU (grhd2_gpu_set_metric_analytic)."""
        import torch
        torch.cuda.set_device(device)
        self.torch = torch
        self.precision = precision
        self.metric = metric
        self.stream = torch.cuda.Stream(device=device)
        self._problems = {}  # request id -> Future of its Problem
        self._pool = concurrent.futures.ThreadPoolExecutor(max_workers=host_workers)
        self.retire_stream = torch.cuda.Stream(device=device)
        # host seconds: waiting for a set-up, GPU grid creation (buffers, tables), initial
        # data (upload, prim_to_cons, first CFL), result + release, and the parts of a
        # batch rebuild
        self.host_s = dict(setup_wait=0.0, create=0.0, upload=0.0, retire=0.0, batch_close=0.0, batch_join=0.0,
                           batch_create=0.0, batch_clock=0.0)

    def close(self):
        self._pool.shutdown(wait=True)

    def free_bytes(self) -> int:
        return int(self.torch.cuda.mem_get_info()[0])

    def announce(self, req: Request):
        """Start the request's host-side set-up on the thread pool (ctypes releases the
        GIL while the host library builds it)."""
        from .problem import Problem
        if req.id not in self._problems:
            self._problems[req.id] = self._pool.submit(Problem.from_keys, req.problem,
                                                       metric_cache=self.metric == "host", **req.keys)

    def problem(self, req: Request):
        """The request's host-side set-up (metric tables, initial data), built once."""
        self.announce(req)
        ts = time.perf_counter()
        pb = self._problems[req.id].result()
        self.host_s["setup_wait"] += time.perf_counter() - ts
        return pb

    def bytes_needed(self, req: Request) -> int:
        from . import native as N
        from .solver import PRECISION
        cfg = self.problem(req).config(PRECISION[self.precision])
        return int(N.gpu_lib().grhd2_gpu_device_bytes(cfg)) + 64 * 1024  # + batch descriptors

    def prepare(self, req: Request):
        """Grid of the request on a private stream (overlaps the batch stream's work)."""
        from .solver import GpuGrid
        pb = self.problem(req)
        del self._problems[req.id]
        ts = time.perf_counter()
        g = GpuGrid(pb, precision=self.precision, upload_initial=False, metric=self.metric)
        tu = time.perf_counter()
        g.upload(p=pb.prims_view())
        g.prim_to_cons()
        g.cfl()
        te = time.perf_counter()
        self.host_s["create"] += tu - ts
        self.host_s["upload"] += te - tu
        return g

    def batch(self, grids, new_clocks):
        """Batch of the resident grids on the batch stream; new_clocks[k] = (t0, final) for
        grids that join now (None for grids keeping their running clock)."""
        from .solver import GpuBatch
        t = [time.perf_counter()]
        for g in grids:
            if g.stream_ptr != self.stream.cuda_stream:
                g.set_stream(self.stream.cuda_stream)
        t.append(time.perf_counter())
        b = GpuBatch(grids)
        t.append(time.perf_counter())
        for k, c in enumerate(new_clocks):
            if c is not None:
                b.set_clock(k, c[0], c[1], -1)
        t.append(time.perf_counter())
        for key, a, z in (("batch_join", 0, 1), ("batch_create", 1, 2), ("batch_clock", 2, 3)):
            self.host_s[key] += t[z] - t[a]
        return b

    def step(self, batch, nsteps: int):
        batch.step(nsteps, graph=True)

    def clocks(self, batch):
        return batch.clocks()

    def detach(self, grid):
        """Move a finished grid off the batch stream (which is idle after the round's clock
        read), so its result can be read while the next round runs."""
        grid.set_stream(self.retire_stream.cuda_stream)

    def finish(self, grid, keep: bool):
        ts = time.perf_counter()
        up = grid.download(want_p=False)[0] if keep else None
        grid.close()
        self.host_s["retire"] += time.perf_counter() - ts
        return up

    def close_batch(self, batch):
        ts = time.perf_counter()
        batch.close()
        self.host_s["batch_close"] += time.perf_counter() - ts


class SolveServer:
    """Admission by device memory, continuous batching, per-request time to solution."""

    def __init__(self, engine, budget_bytes: int | None = None, max_active: int = 1024, steps_per_round: int = 16,
                 keep_results: bool = False, clock=time.perf_counter, sleep=time.sleep):
        self.engine = engine
        self.budget = int(budget_bytes if budget_bytes is not None else 0.8 * engine.free_bytes())
        self.max_active = max_active
        self.k = steps_per_round
        self.keep = keep_results
        self.clock = clock
        self.sleep = sleep
        self.peak_bytes = 0
        self.peak_active = 0
        self.rounds = 0
        self.rebuilds = 0
        # host seconds per activity: where a round's wall clock goes
        self.host_s = dict(prepare=0.0, enqueue=0.0, wait=0.0, retire=0.0, rebuild=0.0)

    def run(self, requests: list[Request]) -> list[Result]:
        eng = self.engine
        pending = collections.deque(sorted(requests, key=lambda r: r.arrival))
        waiting = collections.deque()
        active = []        # [request, grid, bytes, admitted time]
        new_clock = []     # parallel to active: (t0, final) until the grid joins a batch
        retiring = []      # finished: [request, grid, bytes, admitted time, steps, t]
        results = []
        used = 0
        batch = None
        changed = False
        t0 = self.clock()
        while pending or waiting or active or retiring:
            if batch is not None:
                ts = self.clock()
                eng.step(batch, self.k)  # asynchronous: host work below overlaps it
                self.host_s["enqueue"] += self.clock() - ts
                self.rounds += 1
            # results of the grids that finished in the previous round, read while this
            # round runs; their memory returns to the budget here
            for req, g, need, adm, nsteps, tg in retiring:
                ts = self.clock()
                up = eng.finish(g, self.keep)
                self.host_s["retire"] += self.clock() - ts
                results.append(Result(req.id, req.kind, req.cells, req.arrival, adm, self.clock() - t0,
                                      nsteps, tg, up))
                used -= need
            retiring = []
            now = self.clock() - t0
            while pending and pending[0].arrival <= now:
                req = pending.popleft()
                if hasattr(eng, "announce"):
                    eng.announce(req)
                waiting.append(req)
            while waiting and len(active) < self.max_active:
                req = waiting[0]
                need = eng.bytes_needed(req)
                if need > self.budget:
                    raise ValueError(f"request {req.id} needs {need} bytes, more than the whole budget")
                if used + need > self.budget:
                    break  # first come, first served: wait for memory to free up
                waiting.popleft()
                ts = self.clock()
                g = eng.prepare(req)
                self.host_s["prepare"] += self.clock() - ts
                active.append([req, g, need, self.clock() - t0])
                new_clock.append((0.0, req.final_time))
                used += need
                changed = True
            self.peak_bytes = max(self.peak_bytes, used)
            self.peak_active = max(self.peak_active, len(active))
            if batch is not None:
                ts = self.clock()
                t, steps, act = eng.clocks(batch)  # waits for the round
                self.host_s["wait"] += self.clock() - ts
                keep_rows, keep_clock = [], []
                for k, row in enumerate(active):
                    if k < len(act) and not act[k]:
                        if hasattr(eng, "detach"):
                            eng.detach(row[1])
                        retiring.append(row + [int(steps[k]), float(t[k])])
                        changed = True
                    else:
                        keep_rows.append(row)
                        keep_clock.append(new_clock[k])
                active, new_clock = keep_rows, keep_clock
            if changed:
                ts = self.clock()
                if batch is not None:
                    eng.close_batch(batch)
                    batch = None
                if active:
                    batch = eng.batch([row[1] for row in active], new_clock)
                    new_clock = [None] * len(active)
                    self.rebuilds += 1
                changed = False
                self.host_s["rebuild"] += self.clock() - ts
            if not active and not retiring and pending and not waiting:
                wait = pending[0].arrival - (self.clock() - t0)
                if wait > 0:
                    self.sleep(wait)
        if batch is not None:
            eng.close_batch(batch)
        return sorted(results, key=lambda r: r.id)


def summarize(results: list[Result]) -> dict:
    tts = np.array([r.time_to_solution for r in results])
    zu = sum(r.cells * r.steps for r in results)
    span = max(r.done for r in results) - min(r.arrival for r in results)
    return {"requests": len(results), "zone_updates": int(zu), "makespan_s": span,
            "zone_updates_per_s": zu / span if span > 0 else None,
            "tts_p50_s": float(np.percentile(tts, 50)), "tts_p99_s": float(np.percentile(tts, 99)),
            "tts_mean_s": float(tts.mean())}


def main(argv=None):
    ap = argparse.ArgumentParser(description=__doc__.split("\n")[0])
    ap.add_argument("--requests", type=int, default=4096)
    ap.add_argument("--seed", type=int, default=20260901)
    ap.add_argument("--rate", type=float, default=2000.0, help="mean arrivals per second")
    ap.add_argument("--michel-final-time", type=float, default=50.0)
    ap.add_argument("--max-riemann-cells", type=int, default=8192)
    ap.add_argument("--max-michel-cells", type=int, default=4096)
    ap.add_argument("--steps-per-round", type=int, default=16)
    ap.add_argument("--precision", choices=["fp64", "mixed"], default="fp64")
    ap.add_argument("--metric", choices=["host", "device"], default="host",
                    help="build each request's metric tables on the host (uploaded) or on the device")
    args = ap.parse_args(argv)
    reqs = make_stream(args.requests, args.seed, args.rate, args.michel_final_time,
                       riemann_cells=(128, args.max_riemann_cells), michel_cells=(512, args.max_michel_cells))
    eng = GpuEngine(args.precision, metric=args.metric)
    srv = SolveServer(eng, steps_per_round=args.steps_per_round)
    res = srv.run(reqs)
    eng.close()
    out = summarize(res)
    out.update(peak_active=srv.peak_active, peak_bytes=srv.peak_bytes, rounds=srv.rounds, rebuilds=srv.rebuilds,
               budget_bytes=srv.budget, precision=args.precision, metric=args.metric, host_s=srv.host_s,
               engine_host_s=eng.host_s)
    print(json.dumps(out))


if __name__ == "__main__":
    sys.exit(main())
