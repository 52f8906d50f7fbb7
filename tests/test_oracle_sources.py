"""A second, independent reading of the reference's metric source terms against the oracle's.

calc_sources (equations.f90:509-552) with calculate_stress_energy_tensor
(metrics.f90:1251-1310) is restated here in plain Python from the Fortran, in its loop and
evaluation order, and compared bit for bit with the oracle's restatement on the metric
tables the host set-up builds (Kerr-Schild and Eddington-Finkelstein in logarithmic and
physical radius, Minkowski spherical and cylindrical; Minkowski Cartesian returns zero) at
random cells and states, superluminal velocities included (the tensor's velocity cap).
"""
import ctypes as C
import math
import zlib

import numpy as np
import pytest

from grhd_b200.problem import Problem
from oracle import binding as B
from oracle.binding import OracleRun
from tests.helpers import michel, shock_tube, torus_2p5d, torus_3d

DE, PR, VX = 0, 1, 2


def sources(prim, cell, g1, v_max, cartesian_minkowski):
    """calc_sources for one cell; `cell` holds its cache entries in Fortran index meaning."""
    src = [0.0] * 5
    if cartesian_minkowski:
        return src
    alpha, sqg = cell["alpha"], cell["sqg"]
    chris, dg, dlna = cell["chris"], cell["dg"], cell["dlna"]
    beta, g, gmunu = cell["beta"], cell["gamma"], cell["gmunu"]
    # calculate_stress_energy_tensor
    v = [prim[VX], prim[VX + 1], prim[VX + 2]]
    v_sq = 0.0
    for ii in range(3):
        for jj in range(3):
            v_sq = v_sq + g[ii][jj] * v[ii] * v[jj]
    if v_sq >= v_max:
        v = [v[0] * math.sqrt(v_max / v_sq), v[1] * math.sqrt(v_max / v_sq), v[2] * math.sqrt(v_max / v_sq)]
        v_sq = v_max
    h = 1.0 + g1 * prim[PR] / prim[DE]
    W = 1.0 / math.sqrt(1.0 - v_sq)
    u = [W / alpha, W * (v[0] - beta[0] / alpha), W * (v[1] - beta[1] / alpha), W * (v[2] - beta[2] / alpha)]
    T = [[0.0] * 4 for _ in range(4)]
    for mu in range(4):
        for nu in range(mu, 4):
            T[mu][nu] = (prim[DE] * h * u[mu] * u[nu]) + (prim[PR] * gmunu[mu][nu])
            if mu != nu:
                T[nu][mu] = T[mu][nu]
    # calc_sources
    for d in range(3):
        for mu in range(4):
            for nu in range(4):
                src[VX + d] = src[VX + d] + 0.5 * T[mu][nu] * dg[mu][nu][d]
    for mu in range(4):
        src[PR] = src[PR] + T[mu][0] * dlna[mu]
        for nu in range(4):
            src[PR] = src[PR] - T[mu][nu] * chris[0][mu][nu]
    src = [s * alpha * sqg for s in src]
    src[PR] = src[PR] * alpha
    return src


def cache_cell(mv, nx, q):
    """The cache entries of cell q (0-based (i-1) + nx (j-1)) from the host tables."""
    a = lambda ptr, n: np.ctypeslib.as_array(ptr, (n * (q + 1),))[n * q:n * (q + 1)]
    col = lambda x, shape: x.reshape(shape[::-1]).transpose(*range(len(shape) - 1, -1, -1))  # Fortran order
    return {"alpha": float(a(mv.alpha_c, 1)[0]), "sqg": float(a(mv.sqrt_gamma_c, 1)[0]),
            "beta": a(mv.beta_c, 3).tolist(), "gamma": col(a(mv.gamma_c, 9), (3, 3)).tolist(),
            "gmunu": col(a(mv.gmunu_c, 16), (4, 4)).tolist(), "chris": col(a(mv.chris_c, 64), (4, 4, 4)).tolist(),
            "dg": col(a(mv.dg_c, 48), (4, 4, 3)).tolist(), "dlna": a(mv.dlna_c, 4).tolist()}


CASES = [
    ("ks_log_3d", lambda: torus_3d(nx=16, ny=8, nz=8)),
    ("ks_log", lambda: torus_2p5d(nx=24, nz=12)),
    ("ks_phys", lambda: torus_2p5d(nx=24, nz=12, logarithmic_r=False, r_min=1.2, r_max=40.0)),
    ("ef_log", lambda: michel(nx=64)),
    ("ef_phys", lambda: michel(nx=64, logarithmic_r=False, r_min=1.8)),
    ("minkowski_spherical", lambda: Problem.from_keys("sod", nx=16, ny=8, geometry="spherical", r_min=1.0,
                                                      r_max=2.0, y_min=0.0, y_max=math.pi, sod_interface=1.5)),
    ("minkowski_cylindrical", lambda: shock_tube(nx=32, geometry="cylindrical", sod_interface=0.5)),
    ("minkowski_cartesian", lambda: shock_tube(nx=32)),
]


@pytest.mark.parametrize("name,maker", CASES, ids=[c[0] for c in CASES])
def test_sources_match_an_independent_restatement(name, maker):
    pb = maker()
    o = OracleRun(pb)
    cfg = pb.config(0)
    mv = pb.metric_view()
    rng = np.random.default_rng(zlib.crc32(name.encode()))
    dp = lambda a: a.ctypes.data_as(C.POINTER(C.c_double))
    capped = 0
    for _ in range(200):
        i, j = int(rng.integers(1, pb.nx + 1)), int(rng.integers(1, pb.ny + 1))
        q = (i - 1) + pb.nx * (j - 1)
        cell = cache_cell(mv, pb.nx, q)
        vdir = rng.normal(size=3)
        vdir = vdir / math.sqrt(vdir @ np.array(cell["gamma"]) @ vdir)
        speed = rng.choice([0.0, rng.uniform(0.0, 0.9), rng.uniform(0.9, 1.0), rng.uniform(1.0, 1.5)])
        prim = np.array([10.0 ** rng.uniform(-6, 1), 10.0 ** rng.uniform(-8, 2), *(speed * vdir)])
        got = np.zeros(5)
        B.lib().orc_sources(C.byref(o.cfg), C.byref(o.met), dp(prim), i, j, dp(got))
        want = sources(prim.tolist(), cell, cfg.g1, cfg.v_max, cfg.metric_kind == 0 and cfg.geom_kind == 0)
        assert got.tobytes() == np.array(want).tobytes(), (name, i, j, prim, got, want)
        capped += speed >= 1.0
    assert capped > 0
