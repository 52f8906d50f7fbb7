"""The oracle's SSP-RK3 step against the stage loop of grhd2.f90:232-265 written out here.

u = up; set_boundary_conditions(p); then three times: calc_rhs(p, rhs), the stage
combination (up = u + rhs dt; up = 0.75 u + 0.25 (up + rhs dt); up = (u + 2 (up + rhs
dt)) / 3, in the reference's array-expression order), cons_to_prim over every cell, and
set_boundary_conditions(p).  The pieces are the oracle's, each cross-checked on its own
(reconstruction, sources, con2prim, the Riemann and boundary KATs); this checks their
order and the combination, bit for bit, on runs of several steps.
"""
import ctypes as C

import numpy as np
import pytest

from oracle.binding import OracleRun
from tests.helpers import initial_state, michel, shock_tube, torus_2p5d, torus_3d


def _p(a):
    return a.ctypes.data_as(C.POINTER(C.c_double))


def stage_loop(o, dt):
    """One step of grhd2.f90:232-265 from the oracle's calc_rhs, cons_to_prim and
    set_boundary_conditions."""
    L, c, m = o.L, C.byref(o.cfg), C.byref(o.met)
    u = o.up.copy()
    assert L.orc_set_boundary(c, m, _p(o.p)) == 0
    rhs = np.zeros_like(o.up)
    for rk in (1, 2, 3):
        L.orc_calc_rhs(c, m, _p(o.p), _p(rhs), C.byref(o.counters))
        if rk == 1:
            o.up[...] = u + rhs * dt
        elif rk == 2:
            o.up[...] = 0.75 * u + 0.25 * (o.up + rhs * dt)
        else:
            o.up[...] = (u + 2.0 * (o.up + rhs * dt)) / 3.0
        L.orc_cons_to_prim_all(c, m, _p(o.up), _p(o.p), C.byref(o.counters))
        assert L.orc_set_boundary(c, m, _p(o.p)) == 0


@pytest.mark.parametrize("maker,kw,steps", [
    (shock_tube, dict(nx=64), 6),
    (shock_tube, dict(nx=48, rec="mp5", rs="hllc", sensor=True), 6),
    (michel, dict(nx=64), 5),
    (torus_2p5d, dict(nx=24, nz=12), 3),
    (torus_3d, dict(nx=12, ny=6, nz=6), 2),
])
def test_oracle_step_is_the_reference_stage_loop(maker, kw, steps):
    pb = maker(**kw)
    p0 = initial_state(pb)
    a, b = OracleRun(pb, p0), OracleRun(pb, p0)
    for o in (a, b):
        o.prim_to_cons()
        o.set_boundary()
    for _ in range(steps):
        dt = a.cfl()
        a.step(dt)
        stage_loop(b, dt)
        assert a.up.tobytes() == b.up.tobytes()
        assert a.p.tobytes() == b.p.tobytes()
    assert a.counters.as_dict() == b.counters.as_dict()
