"""Command-line runner: advance a problem on the GPU (the device-side counterpart of
``./grhd2 file.par`` without I/O) and report device time per SSP-RK3 step.

    python -m grhd_b200.run --par case.par [--steps N] [--precision fp64|mixed]
    python -m grhd_b200.run --workload torus3d --nx 128 --ny 64 --nz 64 --steps 4

Workloads name the benchmark configurations (shock tube, Michel, 2.5D and 3D Kerr-Schild
tori); extra ``--key value`` pairs override .par keys.
"""
from __future__ import annotations

import argparse
import json
import sys
import time

WORKLOADS = {
    "shock": ("sod", dict(nx=400, adiabatic_index=1.6666666666666667, sod_density_left=10,
                          sod_pressure_left=13.33, sod_density_right=1, sod_pressure_right=1e-6,
                          reconstruction="weno5", riemann_solver="hlle", cfl=0.4, final_time=0.4)),
    "michel": ("michel", dict(metric="eddington_finkelstein", geometry="spherical", logarithmic_r=True,
                              bh_mass=1.0, nx=1024, ny=1, nz=1, r_min=1.8, r_max=20.0,
                              adiabatic_index=1.3333333333333333, michel_critical_radius=8.0,
                              reconstruction="mp5", riemann_solver="hlle", final_time=500.0,
                              perturbation="density_noise", perturbation_amplitude=0.001,
                              perturbation_time=0.0, perturbation_seed=3435)),
    "torus2p5d": ("fishbone_equatorial", dict(
        metric="kerr_schild", geometry="spheroidal", logarithmic_r=True, spin=0.9, bh_mass=1.0, nx=400,
        ny=1, nz=200, r_min=1.2, r_max=40.0, theta_min=0, theta_max=1, phi_min=0, phi_max=2,
        fm_inner_radius=6.0, fm_pressure_max_radius=12.0, fm_polytropic_constant=0.0015,
        adiabatic_index=1.3333333333333333, reconstruction="weno5", riemann_solver="hlle",
        shock_sensor=False, cfl=0.4, perturbation="pressure_noise", perturbation_amplitude=0.01,
        perturbation_time=0.0, perturbation_seed=3435)),
    "torus3d": ("fishbone_3d", dict(
        metric="kerr_schild", geometry="spheroidal", logarithmic_r=True, spin=0.9, bh_mass=1.0, nx=256,
        ny=128, nz=128, r_min=1.2, r_max=40.0, theta_min=0, theta_max=1, phi_min=0, phi_max=2,
        fm_inner_radius=6.0, fm_pressure_max_radius=12.0, fm_polytropic_constant=0.0015,
        adiabatic_index=1.3333333333333333, reconstruction="mp5", riemann_solver="hllc",
        shock_sensor=True, cfl=0.4, perturbation="pressure_noise", perturbation_amplitude=0.01,
        perturbation_time=0.0, perturbation_seed=3435)),
}


def workload_text(name: str, **overrides) -> str:
    from .problem import par_text
    problem, keys = WORKLOADS[name]
    keys = dict(keys)
    keys.update(overrides)
    return par_text(problem, **keys)


def with_key(text: str, key: str, value) -> str:
    """.par text with every assignment of key replaced by key = value."""
    keep = [ln for ln in text.splitlines() if ln.split("=")[0].strip().lower() != key]
    return "\n".join(keep + [f"{key} = {value}"]) + "\n"


def _parse_overrides(rest):
    out = {}
    it = iter(rest)
    for k in it:
        if not k.startswith("--"):
            raise SystemExit(f"unexpected argument {k}")
        v = next(it)
        out[k[2:].replace("-", "_")] = v
    return out


def michel_l1(pb, p) -> float:
    """The reference's Michel error (output.f90:1189-1213): mean |rho - rho_exact| over
    cells i = int(0.10 nx) .. int(0.95 nx) (1-based), rho_exact the analytic steady
    profile the run starts from (before any perturbation)."""
    import numpy as np
    g, nx = pb.ng, pb.nx
    exact = pb.initial_prims()
    i0 = max(1, int(0.10 * nx))
    i1 = min(nx, max(i0, int(0.95 * nx)))
    rows = slice(g + i0, g + i1 + 1)  # array index of cell i is g + i
    j, k = g + 1, g + 1
    return float(np.abs(p[k, j, rows, 0] - exact[k, j, rows, 0]).mean())


def accuracy_run(pb, p0, final_time, max_steps):
    """FP64 and mixed runs of one problem from the same state (each on its own device
    clock: CFL dt clamped to final_time, or max_steps steps)."""
    import numpy as np
    from .solver import GpuBatch, GpuGrid
    tf = final_time if final_time is not None else 1e300
    ms = -1 if final_time is not None else max_steps
    out = {"cells": pb.n_cells, "final_time": final_time}
    ups, ps = {}, {}
    for prec in ("fp64", "mixed", "mixed_comp64", "mixed_comp32"):
        g = GpuGrid(pb, precision=prec, upload_initial=False)
        g.upload(p=p0)
        g.prim_to_cons()
        b = GpuBatch([g])
        b.set_clock(0, 0.0, tf, ms)
        t0 = time.perf_counter()
        while b.clock(0)[2]:
            b.step(2000, graph=True)
        el = time.perf_counter() - t0
        t, n, _ = b.clock(0)
        up, pp = g.download(p_template=p0)
        ups[prec], ps[prec] = up, pp
        out[prec] = {"steps": int(n), "t": t, "seconds": el, "zone_updates_per_s": pb.n_cells * n / el,
                     "counters": g.counters()}
        if pb.info.case_id == 7:
            out[prec]["michel_l1_vs_analytic"] = michel_l1(pb, pp)
        b.close()
        g.close()
    r = ups["fp64"].reshape(-1, 5)
    den = np.abs(r).sum(axis=0)
    out["l1_vs_fp64"] = {}
    for prec in ("mixed", "mixed_comp64", "mixed_comp32"):
        num = np.abs(ups[prec].reshape(-1, 5) - r).sum(axis=0)
        # relative L1 per conserved variable, each in its own norm (a variable that is zero
        # everywhere reports its absolute L1)
        out["l1_vs_fp64"][prec] = np.where(den > 0, num / np.where(den > 0, den, 1.0), num).tolist()
    out["l1_mixed_vs_fp64"] = out["l1_vs_fp64"]["mixed"]
    return out


def main(argv=None):
    ap = argparse.ArgumentParser(description=__doc__.split("\n")[0])
    ap.add_argument("--par", help=".par file")
    ap.add_argument("--workload", choices=sorted(WORKLOADS))
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=1)
    ap.add_argument("--precision", choices=["fp64", "mixed", "mixed_comp64", "mixed_comp32"], default="fp64")
    ap.add_argument("--batch", type=int, default=1, help="replicas stepped as one batch")
    ap.add_argument("--graph", type=int, default=1, help="replay each step as a CUDA graph")
    ap.add_argument("--flux", choices=["auto", "split", "fused", "split_var", "tune"], default="tune",
                    help="face-flux kernel variant ('tune': time variants and tiles on this batch)")
    ap.add_argument("--tile", type=int, default=0, help="face-kernel tile extent along i (0: automatic)")
    ap.add_argument("--stage", choices=["auto", "on", "off"], default="auto",
                    help="the stage kernel for 1D and 2D grids (one kernel per RK stage)")
    ap.add_argument("--step-mode", choices=["auto", "graph", "persistent"], default="auto",
                    help="stage kernels replayed as a graph, or whole steps in one persistent launch")
    ap.add_argument("--accuracy", action="store_true",
                    help="run the problem in FP64 and mixed from the same state to --final-time (or --steps) "
                         "and report the mixed-vs-FP64 L1 (and the Michel L1 against the analytic profile)")
    ap.add_argument("--final-time", type=float, default=None)
    ap.add_argument("--metric", choices=["host", "device"], default="host",
                    help="upload the host-built metric cache, or build it on the device")
    args, rest = ap.parse_known_args(argv)
    overrides = _parse_overrides(rest)
    from .problem import Problem
    from .solver import GpuBatch, GpuGrid
    if args.par:
        text = open(args.par).read()
        for k, v in overrides.items():
            text += f"{k} = {v}\n"
    elif args.workload:
        text = workload_text(args.workload, **overrides)
    else:
        raise SystemExit("give --par or --workload")
    pb = Problem(text)
    p = pb.initial_prims()
    if pb.info.perturbation_type and pb.info.perturbation_time <= 0.0:
        pb.perturb(p)
    if args.accuracy:
        print(json.dumps(accuracy_run(pb, p, args.final_time, args.steps)))
        return 0
    # replicas of the problem, each with its own perturbation seed, on one stream
    grids = []
    for r in range(max(1, args.batch)):
        pr = pb if r == 0 else Problem(with_key(text, "perturbation_seed", 3435 + r))
        q = p
        if r > 0:
            q = pr.initial_prims()
            if pr.info.perturbation_type and pr.info.perturbation_time <= 0.0:
                pr.perturb(q)
        gr = GpuGrid(pr, precision=args.precision, upload_initial=False,
                     stream=grids[0].stream_ptr if grids else None, metric=args.metric)
        gr.upload(p=q)
        gr.prim_to_cons()
        grids.append(gr)
    g = grids[0]
    batch = GpuBatch(grids)
    for k in range(len(grids)):
        batch.set_clock(k, 0.0, 1e300, -1)
    if args.flux == "tune":
        tuned = batch.autotune()
    else:
        tuned = None
        batch.set_flux_variant(args.flux)
        batch.set_tile(args.tile)
    batch.set_stage_kernel(args.stage)
    batch.set_step_mode(args.step_mode)
    batch.step(args.warmup, graph=args.graph)
    g.synchronize()
    t0 = time.perf_counter()
    batch.step(args.steps, graph=args.graph)
    g.synchronize()
    el = time.perf_counter() - t0
    prof = batch.profile_step()
    cells = pb.n_cells * len(grids)
    out = {"cells": cells, "grids": len(grids), "steps": args.steps, "dt": g.cfl(),
           "ms_per_step": el / args.steps * 1e3, "zone_updates_per_s": cells * args.steps / el,
           "kernels": prof, "counters": g.counters(), "flux_variant": tuned or args.flux,
           "stage_groups": batch.stage_groups, "metric": args.metric,
           "metric_ms": [round(gr.metric_seconds * 1e3, 3) for gr in grids]}
    batch.close()
    for gr in reversed(grids):
        gr.close()
    print(json.dumps(out))


if __name__ == "__main__":
    sys.exit(main())
