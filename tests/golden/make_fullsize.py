"""Oracle fixtures of whole runs at the configurations' full sizes and final times.

The oracle (oracle/, the plain-C restatement of the reference path) needs minutes to
hours of host time for these runs, far too long for a test, so its results are computed
once here and committed:

  fullsize_michel_1024_t500.npz   1D Michel accretion, 1024 log-r cells, MP5 + HLLE, to t = 500
                                  (about 2.4e5 steps): the whole final state
  fullsize_torus2p5d_400x1x200_2000.npz   2.5D Kerr-Schild torus 400 x 1 x 200, WENO5 + HLLE,
                                  2000 steps
  fullsize_torus3d_256x128x128_20.npz     3D Kerr-Schild torus 256 x 128 x 128, MP5 + HLLC +
                                  shock sensor, 20 steps
  fullsize_torus3d_128x64x64_500.npz      the 3D torus at 128 x 64 x 64, 500 steps
  fullsize_torus3d_256x128x128_500.npz    the 3D torus at its full size and final step count

For the tori each file holds the SHA-256 of the final conserved state (the bytes of up in
the reference layout, u(5, nx, ny, nz) with the variable fastest, little-endian float64),
the final state at 2048 seeded cell indices, the per-variable sums of |up|, the step
count, the final time and the con2prim / reconstruction / HLLC counters.  The GPU tests
compare the FP64 path's final state against these.

    python -m tests.golden.make_fullsize [name ...]
"""
from __future__ import annotations

import hashlib
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

from oracle.binding import OracleRun  # noqa: E402
from tests.helpers import initial_state, michel, torus_2p5d, torus_3d  # noqa: E402

SAMPLE = 2048
SAMPLE_SEED = 20261204

CASES = {
    "michel_1024_t500": (lambda: michel(nx=1024), dict(final_time=500.0), True),
    "torus2p5d_400x1x200_2000": (lambda: torus_2p5d(nx=400, nz=200), dict(nsteps=2000), False),
    "torus3d_256x128x128_20": (lambda: torus_3d(nx=256, ny=128, nz=128), dict(nsteps=20), False),
    "torus3d_128x64x64_500": (lambda: torus_3d(nx=128, ny=64, nz=64), dict(nsteps=500), False),
    "torus3d_256x128x128_500": (lambda: torus_3d(nx=256, ny=128, nz=128), dict(nsteps=500), False),
}


def state_digest(up: np.ndarray) -> str:
    """SHA-256 of a conserved state in the reference layout (little-endian float64)."""
    return hashlib.sha256(np.ascontiguousarray(up, dtype="<f8").tobytes()).hexdigest()


def sample_index(n_cells: int) -> np.ndarray:
    rng = np.random.default_rng(SAMPLE_SEED)
    return np.sort(rng.choice(n_cells, size=min(SAMPLE, n_cells), replace=False))


def path_of(name: str) -> str:
    return os.path.join(HERE, f"fullsize_{name}.npz")


def make(name: str) -> None:
    maker, run, whole = CASES[name]
    pb = maker()
    p0 = initial_state(pb)
    o = OracleRun(pb, p0)
    o.prim_to_cons()
    o.set_boundary()
    t0 = time.time()
    n, t = o.run(0.0, run.get("final_time", 1e30), run.get("nsteps", -1))
    el = time.time() - t0
    up = o.up
    flat = up.reshape(-1, 5)
    idx = sample_index(flat.shape[0])
    cnt = o.counters.as_dict()
    out = dict(steps=np.int64(n), t=np.float64(t), sha256=np.array(state_digest(up)),
               abs_sum=np.abs(flat).sum(axis=0), sample_index=idx, sample_up=flat[idx],
               counter_names=np.array(list(cnt.keys())), counters=np.array(list(cnt.values()), dtype=np.int64))
    if whole:
        out["up"] = up
    np.savez_compressed(path_of(name), **out)
    print(f"{name}: {n} steps to t = {t!r} in {el:.0f} s, counters {cnt}", flush=True)


if __name__ == "__main__":
    for nm in (sys.argv[1:] or list(CASES)):
        make(nm)
