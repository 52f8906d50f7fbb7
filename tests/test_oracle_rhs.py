"""The oracle's calc_rhs against the assembly of evolution.f90:30-191 written out here.

Per direction: extract each strip of primitives with its ghost cells, reconstruct it
(reconstruct_1d_core), solve the Riemann problem at every face with that face's metric
(index i of the strip -> cache entry i + 1), zero the flux on the cylindrical axis and on
polar faces instead of solving there, and accumulate -(F_i - F_{i-1}) / dx, the sources
added in the x sweep.  The reconstruction and sources come from the independent
restatements of test_oracle_reconstruction.py and test_oracle_sources.py, the Riemann
solver from the oracle (pinned by the reference's HLLE/HLLC known-answer tests); the check
is of the assembly -- strips, face-metric indexing, degenerate faces, accumulation order --
bit for bit.
"""
import ctypes as C
import math

import numpy as np
import pytest

from oracle.binding import OracleRun
from tests.helpers import initial_state, michel, shock_tube, shock_tube_xy, torus_2p5d, torus_3d
from tests.test_oracle_reconstruction import reconstruct
from tests.test_oracle_sources import cache_cell, sources

EPS64 = 64.0 * np.finfo(float).eps


def _p(a):
    return a.ctypes.data_as(C.POINTER(C.c_double))


def face_metric(mv, d, f):
    """(alpha, beta(3), gamma (Fortran order, 9), sqrt(gamma)) of face-table entry f."""
    name = "xyz"[d]
    a = np.ctypeslib.as_array(getattr(mv, "alpha_f_" + name), (f + 1,))[f]
    b = np.ctypeslib.as_array(getattr(mv, "beta_f_" + name), (3 * f + 3,))[3 * f:3 * f + 3].copy()
    g = np.ctypeslib.as_array(getattr(mv, "gamma_f_" + name), (9 * f + 9,))[9 * f:9 * f + 9].copy()
    s = np.ctypeslib.as_array(getattr(mv, "sqrt_gamma_f_" + name), (f + 1,))[f]
    return float(a), b, g, float(s)


def calc_rhs(o, pb):
    cfg, mv = pb.config(0), pb.metric_view()
    nx, ny, nz, g = pb.nx, pb.ny, pb.nz, pb.ng
    P = o.p  # [k + g, j + g, i + g, v]
    rhs = np.zeros((nz, ny, nx, 5))
    nonmink = cfg.metric_kind != 0
    polar = cfg.geom_kind in (2, 3)
    xf = np.ctypeslib.as_array(mv.x_face, (nx + 1,))
    cnt = o.counters

    def riemann(qL, qR, d, f):
        a, b, gm, s = face_metric(mv, d, f)
        out = np.zeros(5)
        o.L.orc_riemann(C.byref(o.cfg), _p(np.ascontiguousarray(qL)), _p(np.ascontiguousarray(qR)), d + 1, a,
                        _p(b), _p(gm), s, _p(out), C.byref(cnt))
        return out

    # x sweep, with the sources
    for k in range(1, nz + 1):
        for j in range(1, ny + 1):
            strip = P[k + g, j + g, :, :].tolist()
            qL, qR = reconstruct(strip, nx, cfg.rec_method, cfg.tvd_limiter, cfg.shock_sensor, nonmink, 1)
            F = np.zeros((nx + 1, 5))
            for i in range(nx + 1):
                if cfg.geom_kind == 1 and abs(xf[i]) <= EPS64:
                    continue
                F[i] = riemann(qL[i], qR[i], 0, i + (nx + 1) * (j - 1))
            for i in range(1, nx + 1):
                src = sources(P[k + g, j + g, i + g, :].tolist(), cache_cell(mv, nx, (i - 1) + nx * (j - 1)),
                              cfg.g1, cfg.v_max, cfg.metric_kind == 0 and cfg.geom_kind == 0)
                rhs[k - 1, j - 1, i - 1] = -(F[i] - F[i - 1]) / cfg.dx + np.array(src)
    if ny > 1:
        yf = np.ctypeslib.as_array(mv.y_face, (ny + 1,))
        for k in range(1, nz + 1):
            for i in range(1, nx + 1):
                strip = P[k + g, :, i + g, :].tolist()
                qL, qR = reconstruct(strip, ny, cfg.rec_method, cfg.tvd_limiter, cfg.shock_sensor, nonmink, 2)
                F = np.zeros((ny + 1, 5))
                for j in range(ny + 1):
                    if polar and abs(math.sin(yf[j])) <= EPS64:
                        continue
                    F[j] = riemann(qL[j], qR[j], 1, (i - 1) + nx * j)
                for j in range(1, ny + 1):
                    rhs[k - 1, j - 1, i - 1] = rhs[k - 1, j - 1, i - 1] - (F[j] - F[j - 1]) / cfg.dy
    if nz > 1:
        for j in range(1, ny + 1):
            for i in range(1, nx + 1):
                strip = P[:, j + g, i + g, :].tolist()
                qL, qR = reconstruct(strip, nz, cfg.rec_method, cfg.tvd_limiter, cfg.shock_sensor, nonmink, 3)
                F = np.zeros((nz + 1, 5))
                for k in range(nz + 1):
                    F[k] = riemann(qL[k], qR[k], 2, (i - 1) + nx * (j - 1))
                for k in range(1, nz + 1):
                    rhs[k - 1, j - 1, i - 1] = rhs[k - 1, j - 1, i - 1] - (F[k] - F[k - 1]) / cfg.dz
    return rhs


@pytest.mark.parametrize("maker,kw,steps", [
    (shock_tube, dict(nx=48, rec="weno5"), 3),
    (shock_tube, dict(nx=48, geometry="cylindrical", sod_interface=0.5, rec="tvd", tvd_limiter="superbee"), 3),
    (shock_tube_xy, dict(nx=24, ny=10), 2),
    (michel, dict(nx=48), 3),
    (torus_2p5d, dict(nx=20, nz=10), 2),
    (torus_3d, dict(nx=10, ny=6, nz=6), 1),
])
def test_oracle_rhs_is_the_reference_assembly(maker, kw, steps):
    pb = maker(**kw)
    o = OracleRun(pb, initial_state(pb), libm_exp=True)
    o.prim_to_cons()
    o.set_boundary()
    for _ in range(steps):  # an evolved state, not the initial one
        o.step(o.cfl())
    o.set_boundary()
    want = calc_rhs(o, pb)
    got = np.zeros(pb.cons_shape)
    o.L.orc_calc_rhs(C.byref(o.cfg), C.byref(o.met), _p(o.p), _p(got), C.byref(o.counters))
    assert got.tobytes() == want.tobytes(), np.argwhere(got != want)[:5]
