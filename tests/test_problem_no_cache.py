"""Host set-up without the metric cache (grhd2_problem_create_ex with
GRHD2_PROBLEM_NO_METRIC_CACHE), for grids whose tables are built on the device.

The initial state must not depend on where the tables come from: the Fishbone-Moncrief
initial data reads the centre metric from the cache when there is one and evaluates the
same function at the same point when there is none."""
import ctypes as C

import numpy as np
import pytest

from grhd_b200 import native as N
from grhd_b200.problem import Problem
from tests.helpers import michel, shock_tube, torus_2p5d, torus_3d

ERR_ARG, ERR_STATE = -1, -4


@pytest.mark.parametrize("maker,kw", [(torus_3d, dict(nx=32, ny=16, nz=16)), (torus_2p5d, dict(nx=48, nz=24)),
                                      (michel, dict(nx=128)), (shock_tube, dict(nx=64))])
def test_initial_state_is_the_same_without_the_cache(maker, kw):
    pb = maker(**kw)
    nc = Problem(pb.text, metric_cache=False)
    assert pb.initial_prims().tobytes() == nc.initial_prims().tobytes()
    assert pb.accretion_probe() == nc.accretion_probe()
    assert nc.config(0).nx == pb.config(0).nx
    bp, np_ = pb.bc_view(), nc.bc_view()
    if bp.michel_injector:
        n = 5 * pb.ng * pb.ny * pb.nz
        assert (np.ctypeslib.as_array(bp.michel_injector, (n,)).tobytes() ==
                np.ctypeslib.as_array(np_.michel_injector, (n,)).tobytes())


def test_metric_view_without_the_cache():
    pb = Problem(michel(nx=64).text, metric_cache=False)
    with pytest.raises(RuntimeError):
        pb.metric_view()
    m = N.MetricView()
    assert N.host_lib().grhd2_problem_metric(pb._h, C.byref(m)) == ERR_STATE
    assert not m.alpha_c and not m.alpha_f_x
    xf = np.ctypeslib.as_array(m.x_face, (65,))
    info = pb.info
    assert xf[0] == info.x_min and np.all(np.diff(xf) > 0)


def test_unknown_problem_flags_are_refused():
    h = C.c_void_p()
    err = C.create_string_buffer(256)
    rc = N.host_lib().grhd2_problem_create_ex(michel(nx=64).text.encode(), 6, C.byref(h), err, 256)
    assert rc == ERR_ARG and not h.value
    assert b"flags" in err.value
