"""A second, independent reading of update_adaptive_dt and prim_to_cons against the oracle's.

update_adaptive_dt (evolution.f90:198-275: the largest alpha sqrt(gamma^ii) + |beta^i| per
direction over the metric cache, summed as inverse time steps) and prim_to_cons
(equations.f90:30-88, the cell-metric twin of prim_to_cons_face) restated in plain Python
from the Fortran and compared bit for bit with the oracle's on the set-up's tables of every
metric family (the CFL) and on random states at random cells (prim_to_cons, superluminal
velocities included).  The reference's CFL tests pin three closed forms; this covers the
tables the runs use.
"""
import ctypes as C
import math

import numpy as np
import pytest

from grhd_b200.problem import Problem
from oracle.binding import OracleRun
from tests.helpers import michel, shock_tube, torus_2p5d, torus_3d


def fmax(a, b):
    return b if (b > a or a != a) else a


def prim_to_cons(prim, g, sqg, g1, v_max):
    """equations.f90:30-88 for one cell; g[row][col] the cell's 3-metric."""
    v = [prim[2], prim[3], prim[4]]
    v_sq = 0.0
    for ii in range(3):
        for jj in range(3):
            v_sq = v_sq + g[ii][jj] * v[ii] * v[jj]
    if v_sq >= v_max:
        v = [v[0] * math.sqrt(v_max / v_sq), v[1] * math.sqrt(v_max / v_sq), v[2] * math.sqrt(v_max / v_sq)]
        v_sq = v_max
    v_cov = [0.0, 0.0, 0.0]
    for ii in range(3):
        for jj in range(3):
            v_cov[ii] = v_cov[ii] + g[ii][jj] * v[jj]
    h = 1.0 + g1 * prim[1] / prim[0]
    W = 1.0 / math.sqrt(1.0 - v_sq)
    u = [prim[0] * W, prim[0] * h * (W * W) - prim[1] - prim[0] * W,
         prim[0] * h * (W * W) * v_cov[0], prim[0] * h * (W * W) * v_cov[1], prim[0] * h * (W * W) * v_cov[2]]
    return [x * sqg for x in u]


def update_adaptive_dt(pb):
    cfg, mv = pb.config(0), pb.metric_view()
    nx, ny, nz = pb.nx, pb.ny, pb.nz
    n = nx * ny
    alpha = np.ctypeslib.as_array(mv.alpha_c, (n,))
    beta = np.ctypeslib.as_array(mv.beta_c, (3 * n,)).reshape(n, 3)
    ginv = np.ctypeslib.as_array(mv.gamma_inv_c, (9 * n,)).reshape(n, 3, 3)  # [q][col][row], symmetric
    mx = my = mz = 0.0
    for k in range(nz):  # the cache is k-invariant; the reference loops over k all the same
        for q in range(n):
            a, b, gi = float(alpha[q]), beta[q].tolist(), ginv[q]
            mx = fmax(mx, a * math.sqrt(gi[0][0]) + abs(b[0]))
            if ny > 1:
                my = fmax(my, a * math.sqrt(gi[1][1]) + abs(b[1]))
            if nz > 1:
                mz = fmax(mz, a * math.sqrt(gi[2][2]) + abs(b[2]))
    inv = mx / cfg.dx
    if ny > 1:
        inv = inv + my / cfg.dy
    if nz > 1:
        inv = inv + mz / cfg.dz
    return cfg.cfl / inv


CASES = [
    ("sod", lambda: shock_tube(nx=64)),
    ("sod_xy", lambda: shock_tube(nx=32, ny=16)),
    ("cylindrical", lambda: shock_tube(nx=32, geometry="cylindrical", sod_interface=0.5)),
    ("michel", lambda: michel(nx=96)),
    ("torus_2p5d", lambda: torus_2p5d(nx=40, nz=20)),
    ("torus_3d", lambda: torus_3d(nx=16, ny=8, nz=8)),
    ("sagittal", lambda: Problem.from_keys("fishbone_sagittal", nx=24, ny=12, nz=1)),
    ("offaxis", lambda: Problem.from_keys("offaxis_blast", nx=16, ny=1, nz=8)),
]


@pytest.mark.parametrize("name,maker", CASES, ids=[c[0] for c in CASES])
def test_cfl_matches_an_independent_restatement(name, maker):
    pb = maker()
    o = OracleRun(pb)
    assert np.float64(o.cfl()).tobytes() == np.float64(update_adaptive_dt(pb)).tobytes()


@pytest.mark.parametrize("name,maker", CASES, ids=[c[0] for c in CASES])
def test_prim_to_cons_matches_an_independent_restatement(name, maker):
    pb = maker()
    mv = pb.metric_view()
    n = pb.nx * pb.ny
    gam = np.ctypeslib.as_array(mv.gamma_c, (9 * n,)).reshape(n, 3, 3)
    sqg = np.ctypeslib.as_array(mv.sqrt_gamma_c, (n,))
    o = OracleRun(pb)
    rng = np.random.default_rng(sum(map(ord, name)))
    dp = lambda a: a.ctypes.data_as(C.POINTER(C.c_double))
    for _ in range(200):
        i, j = int(rng.integers(1, pb.nx + 1)), int(rng.integers(1, pb.ny + 1))
        q = (i - 1) + pb.nx * (j - 1)
        g = gam[q].T  # Fortran (3,3) -> [row][col]
        d = rng.normal(size=3)
        d = d / math.sqrt(d @ g @ d)
        speed = rng.choice([0.0, rng.uniform(0.0, 0.99), rng.uniform(1.0, 1.5)])
        prim = np.array([10.0 ** rng.uniform(-8, 1), 10.0 ** rng.uniform(-10, 2), *(speed * d)])
        got = np.zeros(5)
        o.L.orc_prim_to_cons(C.byref(o.cfg), C.byref(o.met), dp(prim), dp(got), i, j)
        want = prim_to_cons(prim.tolist(), g.tolist(), float(sqg[q]), o.cfg.g1, o.cfg.v_max)
        assert got.tobytes() == np.array(want).tobytes(), (name, i, j, prim, got, want)
