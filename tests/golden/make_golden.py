"""Generate tests/golden/golden_small.npz: outputs of the CPU oracle (the plain-C
restatement of GRHD2's per-stage path, oracle/grhd2_oracle.c) on small seeded cases.

The fixtures pin the oracle against drift (tests/test_golden.py re-runs it on the CPU)
and give the GPU kernels fixed vectors to match without the oracle.  Regenerate only on
purpose, after a reviewed change of the oracle:

    python tests/golden/make_golden.py
"""
from __future__ import annotations

import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

OUT = os.path.join(HERE, "golden_small.npz")


def cases():
    """(name, problem factory kwargs, kind, steps) of every fixture; kind 'run' stores the
    conserved state and counters after `steps` steps, 'rhs' the RHS of the initial state."""
    from tests.helpers import michel, shock_tube, torus_2p5d, torus_3d
    return [
        ("shock_weno5_hlle", shock_tube, dict(nx=64), "run", 40),
        ("shock_mp5_hllc_sensor", shock_tube, dict(nx=48, rec="mp5", rs="hllc", sensor=True,
                                                   sod_velocity_left=0.3, sod_velocity_right=-0.2), "run", 30),
        ("shock_tvd_superbee", shock_tube, dict(nx=40, rec="tvd", tvd_limiter="superbee"), "run", 25),
        ("michel_mp5_hlle", michel, dict(nx=64), "run", 20),
        ("torus2p5d_weno5_hlle", torus_2p5d, dict(nx=32, nz=16), "run", 6),
        ("torus2p5d_rhs_weno3_hllc", torus_2p5d, dict(nx=24, nz=12, rec="weno3", rs="hllc", sensor=True), "rhs", 0),
        ("torus3d_mp5_hllc", torus_3d, dict(nx=12, ny=8, nz=8), "run", 3),
    ]


def compute(name, maker, kw, kind, steps):
    from oracle.binding import OracleRun
    from tests.helpers import initial_state
    pb = maker(**kw)
    p0 = initial_state(pb)
    o = OracleRun(pb, p0)
    o.prim_to_cons()
    o.set_boundary()
    if kind == "rhs":
        return {f"{name}/rhs": o.calc_rhs()}
    n, t = o.run(0.0, 1e30, steps)
    c = o.counters.as_dict()
    return {f"{name}/up": o.up.copy(), f"{name}/t": np.array([t]), f"{name}/steps": np.array([n]),
            f"{name}/counters": np.array([c[k] for k in sorted(c)], dtype=np.int64)}


def main():
    data = {}
    for case in cases():
        data.update(compute(*case))
    np.savez_compressed(OUT, **data)
    print(f"wrote {OUT}: {len(data)} arrays, {os.path.getsize(OUT)} bytes")


if __name__ == "__main__":
    main()
