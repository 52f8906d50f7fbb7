"""The C-ABI libraries load without a GPU and export every entry point their headers declare."""
import ctypes as C
import os
import re

import pytest

from grhd_b200 import native as N

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared(header):
    txt = open(os.path.join(ROOT, "include", header)).read()
    txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
    return sorted(set(re.findall(r"\b(grhd2_[a-z0-9_]+)\s*\(", txt)))


@pytest.mark.parametrize("header,loader", [("grhd2_gpu.h", N.gpu_lib), ("grhd2_host.h", N.host_lib)])
def test_every_declared_symbol_is_exported(header, loader):
    names = declared(header)
    assert len(names) >= 10
    lib = loader()
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing


def test_abi_version():
    assert N.gpu_lib().grhd2_gpu_abi_version() == 1


def test_create_rejects_bad_configs_without_touching_the_device():
    """Argument checks run before any CUDA call (so this also runs without a GPU)."""
    lib = N.gpu_lib()
    c = N.GpuConfig()
    c.nx, c.ny, c.nz, c.nghost, c.neq = 400, 1, 1, 3, 4
    c.rec_method, c.riemann, c.case_id = 5, 1, 1
    c.dx = 0.0025
    h = C.c_void_p()
    rc = lib.grhd2_gpu_create(C.byref(c), C.byref(h))
    assert rc == -1 and b"neq must be 5" in lib.grhd2_gpu_last_error(h)
    lib.grhd2_gpu_destroy(h)
    c.neq = 5
    c.nghost = 2
    rc = lib.grhd2_gpu_create(C.byref(c), C.byref(h))
    assert rc == -1 and b"nghost" in lib.grhd2_gpu_last_error(h)
    lib.grhd2_gpu_destroy(h)
    c.nghost, c.case_id, c.nz, c.ny = 3, 12, 5, 8
    rc = lib.grhd2_gpu_create(C.byref(c), C.byref(h))
    assert rc == -6 and b"nz must be even" in lib.grhd2_gpu_last_error(h)
    lib.grhd2_gpu_destroy(h)


def test_metric_entries_reject_missing_arguments_without_touching_the_device():
    """The device metric build and the table read-back check their arguments first."""
    lib = N.gpu_lib()
    mp = N.MetricParams(bh_mass=1.0, a_spin=0.0, x_min=0.0, y_min=0.0)
    assert lib.grhd2_gpu_set_metric_analytic(None, C.byref(mp)) == -1
    assert lib.grhd2_gpu_set_metric_analytic(None, None) == -1
    n = C.c_size_t(7)
    assert lib.grhd2_gpu_metric_table(None, 0, None, 0, C.byref(n)) == -1
    assert n.value == 7  # untouched on an argument error
