"""The metric cache built on the device (grhd2_gpu_set_metric_analytic) against the cache the
host builds and uploads (grhd2_gpu_set_metric).

Both evaluate the same functions (grhd_b200/csrc/gpu/metric_eval.h) in the same operation
order without FMA contraction; only the device's sin, cos and exp differ from the C
library's, by a few ulps.  So: bit-identical tables where no transcendental is taken
(Minkowski Cartesian and cylindrical), tables within 1e-13 of the largest entry of fields with the same units
elsewhere with identical flags (frame validity, axis and pole faces), and runs that stay
within round-off of the host-table runs.  The host tables are themselves pinned by the
reference's set-up tests (tests/test_host_kats.py) and the full-size fixtures.
"""
import ctypes as C
import math

import numpy as np
import pytest

from grhd_b200 import native as N
from grhd_b200.problem import Problem
from grhd_b200.solver import GpuGrid
from tests.helpers import initial_state, michel, rel_l1, shock_tube, torus_2p5d, torus_3d

pytestmark = pytest.mark.gpu

PI = math.pi
ERR_ARG, ERR_STATE = -1, -4  # GRHD2_ERR_ARG, GRHD2_ERR_STATE
SPH = dict(nx=32, ny=16, geometry="spherical", r_min=1.0, r_max=2.0, y_min=0.0, y_max=PI, sod_interface=1.5)


def _cases():
    # (id, problem, bitwise): every metric x geometry x radial-coordinate branch of the
    # set_metric_type dispatch (metrics.f90:94-201)
    return [
        ("minkowski_cartesian", lambda: shock_tube(nx=64), True),
        ("minkowski_cartesian_xy", lambda: shock_tube(nx=40, ny=12), True),
        ("minkowski_cylindrical", lambda: shock_tube(nx=64, geometry="cylindrical", sod_interface=0.5), True),
        ("minkowski_spherical", lambda: Problem.from_keys("sod", **SPH), False),
        ("minkowski_spherical_log", lambda: Problem.from_keys("sod", logarithmic_r=True, **SPH), False),
        ("ef_spherical", lambda: michel(nx=96, logarithmic_r=False, r_min=1.8), False),
        ("ef_spherical_log", lambda: michel(nx=96), False),
        ("ks_spheroidal", lambda: torus_2p5d(nx=48, nz=24, logarithmic_r=False, r_min=1.2, r_max=40.0), False),
        ("ks_spheroidal_log", lambda: torus_2p5d(nx=48, nz=24), False),
        ("ks_spheroidal_log_3d", lambda: torus_3d(nx=24, ny=12, nz=12), False),
    ]


CASES = _cases()


def _grids(pb):
    host = GpuGrid(pb, upload_initial=False, metric="host")
    dev = GpuGrid(pb, upload_initial=False, metric="device")
    return host, dev


def _flag_fields(which):
    # face tables: the frame-validity and axis/pole flags are exact
    return [] if which == 0 else [19, 20]


# fields that share units, compared against the group's largest entry (an entry that is
# zero analytically -- the normal's own covector components, most Christoffel symbols --
# holds only round-off in both tables)
CENTRE_GROUPS = [[0], [1, 2, 3], list(range(4, 10)), list(range(10, 16)), [16], list(range(17, 27)),
                 list(range(27, 37)), list(range(37, 67)), list(range(67, 71)), [71, 72, 73]]
FACE_GROUPS = [[0], [1], list(range(2, 8)), [8], [9], list(range(10, 19)), [19], [20]]


def _max_rel_err(a, b, which):
    """Largest |a - b| over the finite entries, relative to the largest |a| of the field's
    group; also the (field, entry) where it occurs."""
    fin = np.isfinite(a)
    a, b = np.where(fin, a, 0.0), np.where(fin, b, 0.0)
    err = np.zeros_like(a)
    for grp in (CENTRE_GROUPS if which == 0 else FACE_GROUPS):
        scale = np.abs(a[grp]).max()
        err[grp] = np.abs(a[grp] - b[grp]) / (scale if scale > 0 else 1.0)
    worst = np.unravel_index(np.argmax(err), err.shape)
    return err.max(), worst


@pytest.mark.parametrize("name,maker,bitwise", CASES, ids=[c[0] for c in CASES])
def test_device_tables_match_host_tables(name, maker, bitwise):
    pb = maker()
    host, dev = _grids(pb)
    for which in range(4):
        a, b = host.metric_table(which), dev.metric_table(which)
        assert a.shape == b.shape, (which, a.shape, b.shape)
        if a.size == 0:
            continue
        if bitwise:
            assert a.tobytes() == b.tobytes(), f"table {which} differs"
            continue
        # degenerate faces (the cylindrical axis, the poles) have non-finite frame
        # cofactors and a zero frame flag in both
        assert np.array_equal(np.isfinite(a), np.isfinite(b)), f"table {which}: non-finite pattern"
        for f in _flag_fields(which):
            assert np.array_equal(a[f], b[f]), f"table {which} flag field {f}"
        err, worst = _max_rel_err(a, b, which)
        assert err <= 1e-13, f"table {which}: field {worst[0]} entry {worst[1]} off by {err:.3g}"
        if which == 2:  # the pole faces' sqrt(gamma) is exactly zero in both
            assert np.array_equal(a[8] == 0.0, b[8] == 0.0)


RUN_CASES = [c for c in CASES if c[0] in ("minkowski_cylindrical", "ef_spherical_log", "ks_spheroidal_log",
                                          "ks_spheroidal_log_3d")]


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
@pytest.mark.parametrize("name,maker,bitwise", RUN_CASES, ids=[c[0] for c in RUN_CASES])
def test_runs_on_device_tables_match_host_tables(name, maker, bitwise, precision):
    """Ten SSP-RK3 steps on each set of tables: identical where the tables are, within
    round-off of the metric elsewhere (FP64 1e-11 relative L1; the mixed policy, whose
    tables are rounded to FP32, 1e-6)."""
    pb = maker()
    p0 = initial_state(pb)
    out = []
    for metric in ("host", "device"):
        # the device-table grid comes from a host set-up that built no metric cache
        src = pb if metric == "host" else Problem(pb.text, metric_cache=False)
        g = GpuGrid(src, precision=precision, upload_initial=False, metric=metric)
        g.upload(p=p0)
        g.prim_to_cons()
        g.set_boundary()
        n, _ = g.run(0.0, 1e30, 10)
        assert n == 10
        up, _ = g.download()
        out.append(up)
        g.close()
    if bitwise:
        assert out[0].tobytes() == out[1].tobytes()
    else:
        tol = 1e-11 if precision == "fp64" else 1e-6
        err = rel_l1(out[1], out[0])
        assert np.all(err <= tol), err


def test_metric_build_argument_and_state_errors():
    pb = michel(nx=64)
    g = GpuGrid(pb, upload_initial=False, metric="device")
    lib, h = g.lib, g._h
    n = C.c_size_t()
    assert lib.grhd2_gpu_metric_table(h, 4, None, 0, C.byref(n)) == ERR_ARG
    assert lib.grhd2_gpu_metric_table(h, 2, None, 0, C.byref(n)) == 0 and n.value == 0  # ny = 1: no y faces
    assert lib.grhd2_gpu_metric_table(h, 0, None, 0, C.byref(n)) == 0 and n.value == 74 * 64
    small = np.empty(10)
    assert lib.grhd2_gpu_metric_table(h, 0, N.dptr(small), small.size, None) == ERR_ARG
    bad = pb.metric_params()
    bad.bh_mass = float("nan")
    assert lib.grhd2_gpu_set_metric_analytic(h, C.byref(bad)) == ERR_ARG
    # a logarithmic radial grid on a Cartesian configuration is refused before any launch
    c = shock_tube(nx=64).config(0)
    c.use_log_r = 1
    h2 = C.c_void_p()
    assert lib.grhd2_gpu_create(C.byref(c), C.byref(h2)) == 0
    try:
        assert lib.grhd2_gpu_set_metric_analytic(h2, C.byref(pb.metric_params())) == ERR_ARG
        assert lib.grhd2_gpu_metric_table(h2, 0, None, 0, C.byref(n)) == ERR_STATE
        assert lib.grhd2_gpu_cfl(h2, C.byref(C.c_double())) == ERR_STATE
    finally:
        lib.grhd2_gpu_destroy(h2)
    with pytest.raises(ValueError):
        GpuGrid(pb, upload_initial=False, metric="disk")
    g.close()


def test_device_tables_replace_host_tables_in_place():
    """Building the tables on the device over a handle that already holds host tables
    leaves the same tables (to the tolerance above) and a usable handle."""
    pb = torus_2p5d(nx=48, nz=24)
    g = GpuGrid(pb, upload_initial=False, metric="host")
    before = [g.metric_table(w) for w in range(4)]
    assert g.lib.grhd2_gpu_set_metric_analytic(g._h, C.byref(pb.metric_params())) == 0
    for w in range(4):
        a, b = before[w], g.metric_table(w)
        if a.size:
            assert np.array_equal(np.isfinite(a), np.isfinite(b))
            assert _max_rel_err(a, b, w)[0] <= 1e-13
    g.upload(p=initial_state(pb))
    g.prim_to_cons()
    assert g.cfl() > 0.0
    g.close()
