"""ctypes view of the two native libraries of the package.

``libgrhd2gpu.so`` is the drop-in boundary (``include/grhd2_gpu.h``): hand-written sm_100a
kernels for GRHD2's per-stage RHS and update path behind a C-ABI.  ``libgrhd2host.so``
(``include/grhd2_host.h``) is the host-side problem setup that stands in for the Fortran
driver's init-time routines.  Both are built in-tree by ``grhd_b200.build``.

Loading fails loudly when a library is missing: there is no Python or CPU fallback for
the GPU path.
"""
from __future__ import annotations

import ctypes as C
import os

LIB_DIR = os.path.join(os.path.dirname(os.path.abspath(__file__)), "lib")

c_double_p = C.POINTER(C.c_double)


class GpuConfig(C.Structure):
    """grhd2_gpu_config (include/grhd2_gpu.h)."""
    _fields_ = [(n, C.c_int32) for n in (
        "nx", "ny", "nz", "nghost", "neq", "rec_method", "tvd_limiter", "riemann",
        "shock_sensor", "metric_kind", "geom_kind", "use_log_r", "case_id",
        "precision_policy", "reserved")] + [(n, C.c_double) for n in (
        "dx", "dy", "dz", "adb_idx", "g1", "cfl", "rho_floor", "p_floor", "v_max")]


class MetricView(C.Structure):
    """grhd2_gpu_metric_view (include/grhd2_gpu.h)."""
    _fields_ = [(n, c_double_p) for n in (
        "alpha_c", "beta_c", "gamma_c", "gamma_inv_c", "gmunu_c", "sqrt_gamma_c",
        "chris_c", "dg_c", "dlna_c",
        "alpha_f_x", "beta_f_x", "gamma_f_x", "sqrt_gamma_f_x",
        "alpha_f_y", "beta_f_y", "gamma_f_y", "sqrt_gamma_f_y",
        "alpha_f_z", "beta_f_z", "gamma_f_z", "sqrt_gamma_f_z",
        "x_face", "y_face")]


class MetricParams(C.Structure):
    """grhd2_gpu_metric_params (include/grhd2_gpu.h)."""
    _fields_ = [(n, C.c_double) for n in ("bh_mass", "a_spin", "x_min", "y_min")]


class BcView(C.Structure):
    """grhd2_gpu_bc_view (include/grhd2_gpu.h)."""
    _fields_ = [("michel_injector", c_double_p), ("dust_outer", c_double_p),
                ("x_c", c_double_p), ("jet", C.c_double * 7)]


COUNTER_NAMES = ("c2p_floor_pre", "c2p_causal_rescale", "c2p_brent_used", "c2p_root_fail",
                 "c2p_bad_V", "c2p_final_sanitise", "recon_floor_clamps", "hllc_fallbacks")


class Counters(C.Structure):
    """grhd2_gpu_counters (include/grhd2_gpu.h)."""
    _fields_ = [(n, C.c_int64) for n in COUNTER_NAMES]

    def as_dict(self):
        return {n: int(getattr(self, n)) for n in COUNTER_NAMES}


class Diagnostics(C.Structure):
    """grhd2_gpu_diagnostics (include/grhd2_gpu.h)."""
    _fields_ = [(n, C.c_double) for n in ("mass_total", "disk_mass", "angular_momentum", "rho_min", "p_min",
                                         "rho_max", "p_max", "max_v_sq")] + \
        [(n, C.c_int64) for n in ("atmosphere_cells", "invalid_cells")]

    def as_dict(self):
        return {n: getattr(self, n) for n, _ in self._fields_}


class ProblemInfo(C.Structure):
    """grhd2_problem_info (include/grhd2_host.h)."""
    _fields_ = [(n, C.c_int32) for n in ("case_id", "nx", "ny", "nz", "nghost",
                                          "perturbation_type")] + \
        [("perturbation_seed", C.c_int64)] + [(n, C.c_double) for n in (
            "final_time", "cfl", "perturbation_time", "perturbation_amplitude",
            "perturbation_mode", "x_min", "x_max", "y_min", "y_max", "z_min", "z_max",
            "bh_mass", "a_spin", "fm_l", "fm_w_in")]


# symbol table: name -> (restype, argtypes)
_VP = C.c_void_p
GPU_SYMBOLS = {
    "grhd2_gpu_create": (C.c_int, [C.POINTER(GpuConfig), C.POINTER(_VP)]),
    "grhd2_gpu_set_metric": (C.c_int, [_VP, C.POINTER(MetricView)]),
    "grhd2_gpu_set_metric_analytic": (C.c_int, [_VP, C.POINTER(MetricParams)]),
    "grhd2_gpu_metric_table": (C.c_int, [_VP, C.c_int32, c_double_p, C.c_size_t, C.POINTER(C.c_size_t)]),
    "grhd2_gpu_set_bc_data": (C.c_int, [_VP, C.POINTER(BcView)]),
    "grhd2_gpu_upload": (C.c_int, [_VP, c_double_p, c_double_p]),
    "grhd2_gpu_prim_to_cons_all": (C.c_int, [_VP]),
    "grhd2_gpu_cfl": (C.c_int, [_VP, c_double_p]),
    "grhd2_gpu_step": (C.c_int, [_VP, C.c_double]),
    "grhd2_gpu_run": (C.c_int, [_VP, C.c_double, C.c_double, C.c_int64, c_double_p,
                                C.POINTER(C.c_int64)]),
    "grhd2_gpu_calc_rhs": (C.c_int, [_VP, c_double_p]),
    "grhd2_gpu_cons_to_prim_all": (C.c_int, [_VP]),
    "grhd2_gpu_set_boundary": (C.c_int, [_VP]),
    "grhd2_gpu_download": (C.c_int, [_VP, c_double_p, c_double_p]),
    "grhd2_gpu_upload_async": (C.c_int, [_VP, c_double_p, c_double_p]),
    "grhd2_gpu_global_diagnostics": (C.c_int, [_VP, C.POINTER(Diagnostics)]),
    "grhd2_gpu_snapshot_begin": (C.c_int, [_VP, c_double_p]),
    "grhd2_gpu_gw_strain": (C.c_int, [_VP, c_double_p, c_double_p, c_double_p, C.c_int, C.c_double, C.c_double,
                                      c_double_p]),
    "grhd2_gpu_vtk_cell_data": (C.c_int, [_VP, c_double_p, _VP]),
    "grhd2_gpu_snapshot_wait": (C.c_int, [_VP]),
    "grhd2_gpu_total_mass": (C.c_int, [_VP, c_double_p]),
    "grhd2_gpu_mdot": (C.c_int, [_VP, C.c_int, c_double_p]),
    "grhd2_gpu_ppi_modes": (C.c_int, [_VP, c_double_p, c_double_p]),
    "grhd2_gpu_download_async": (C.c_int, [_VP, c_double_p, c_double_p]),
    "grhd2_gpu_get_counters": (C.c_int, [_VP, C.POINTER(Counters)]),
    "grhd2_gpu_reset_counters": (C.c_int, [_VP]),
    "grhd2_gpu_riemann_faces": (C.c_int, [_VP, C.c_int, C.c_int, c_double_p, c_double_p,
                                          c_double_p, c_double_p, c_double_p, c_double_p,
                                          c_double_p]),
    "grhd2_gpu_riemann_faces_noalloc": (C.c_int, [_VP, C.c_int, C.c_int, c_double_p, c_double_p,
                                                  c_double_p, c_double_p, c_double_p, c_double_p,
                                                  c_double_p]),
    "grhd2_gpu_physical_flux": (C.c_int, [_VP, C.c_int, C.c_int, c_double_p, c_double_p,
                                          c_double_p, c_double_p, c_double_p, c_double_p]),
    "grhd2_gpu_synchronize": (C.c_int, [_VP]),
    "grhd2_gpu_get_stream": (C.c_int, [_VP, C.POINTER(_VP)]),
    "grhd2_gpu_profile_step": (C.c_int, [_VP, C.c_double, C.POINTER(C.c_float), C.POINTER(C.c_char_p),
                                         C.c_int, C.POINTER(C.c_int)]),
    "grhd2_gpu_last_error": (C.c_char_p, [_VP]),
    "grhd2_gpu_destroy": (None, [_VP]),
    "grhd2_gpu_abi_version": (C.c_int, []),
    "grhd2_gpu_create_on_stream": (C.c_int, [C.POINTER(GpuConfig), _VP, C.POINTER(_VP)]),
    "grhd2_gpu_batch_create": (C.c_int, [C.POINTER(_VP), C.c_int, C.POINTER(_VP)]),
    "grhd2_gpu_batch_set_clock": (C.c_int, [_VP, C.c_int, C.c_double, C.c_double, C.c_int64]),
    "grhd2_gpu_batch_step": (C.c_int, [_VP, C.c_int, C.c_int]),
    "grhd2_gpu_batch_cons_to_prim": (C.c_int, [_VP]),
    "grhd2_gpu_batch_get_clock": (C.c_int, [_VP, C.c_int, c_double_p, C.POINTER(C.c_int64),
                                            C.POINTER(C.c_int)]),
    "grhd2_gpu_batch_profile_step": (C.c_int, [_VP, C.POINTER(C.c_float), C.POINTER(C.c_char_p),
                                               C.c_int, C.POINTER(C.c_int)]),
    "grhd2_gpu_batch_set_flux_variant": (C.c_int, [_VP, C.c_int]),
    "grhd2_gpu_batch_set_stage_kernel": (C.c_int, [_VP, C.c_int]),
    "grhd2_gpu_batch_stage_kernel": (C.c_int, [_VP]),
    "grhd2_gpu_batch_clocks": (C.c_int, [_VP, c_double_p, C.POINTER(C.c_int64), C.POINTER(C.c_int)]),
    "grhd2_gpu_set_stream": (C.c_int, [_VP, _VP]),
    "grhd2_gpu_device_bytes": (C.c_int64, [C.POINTER(GpuConfig)]),
    "grhd2_gpu_batch_set_tile": (C.c_int, [_VP, C.c_int]),
    "grhd2_gpu_batch_set_step_mode": (C.c_int, [_VP, C.c_int]),
    "grhd2_gpu_batch_step_mode": (C.c_int, [_VP]),
    "grhd2_gpu_batch_autotune": (C.c_int, [_VP, C.c_int, C.POINTER(C.c_int), C.POINTER(C.c_int), C.c_int,
                                           C.POINTER(C.c_int)]),
    "grhd2_gpu_batch_last_error": (C.c_char_p, [_VP]),
    "grhd2_gpu_batch_destroy": (None, [_VP]),
}

HOST_SYMBOLS = {
    "grhd2_problem_create": (C.c_int, [C.c_char_p, C.POINTER(_VP), C.c_char_p, C.c_int]),
    "grhd2_problem_create_ex": (C.c_int, [C.c_char_p, C.c_uint32, C.POINTER(_VP), C.c_char_p, C.c_int]),
    "grhd2_problem_destroy": (None, [_VP]),
    "grhd2_problem_config": (C.c_int, [_VP, C.c_int32, C.POINTER(GpuConfig)]),
    "grhd2_problem_metric": (C.c_int, [_VP, C.POINTER(MetricView)]),
    "grhd2_problem_bc": (C.c_int, [_VP, C.POINTER(BcView)]),
    "grhd2_problem_info_get": (C.c_int, [_VP, C.POINTER(ProblemInfo)]),
    "grhd2_problem_prims": (c_double_p, [_VP]),
    "grhd2_problem_prim_size": (C.c_int64, [_VP]),
    "grhd2_problem_cons_size": (C.c_int64, [_VP]),
    "grhd2_problem_perturb": (C.c_int, [_VP, c_double_p]),
    "grhd2_problem_x": (c_double_p, [_VP]),
    "grhd2_problem_y": (c_double_p, [_VP]),
    "grhd2_problem_z": (c_double_p, [_VP]),
    "grhd2_problem_eval_metric": (C.c_int, [_VP, C.c_double, C.c_double] + [c_double_p] * 8),
    "grhd2_host_metric_at": (C.c_int, [C.c_int32] * 3 + [C.c_double] * 2 + [C.c_int32] + [C.c_double] * 2
                             + [c_double_p] * 8),
    "grhd2_host_dust_state": (C.c_int, [C.c_int32, C.c_double, C.c_double, C.c_double, C.c_double, c_double_p]),
    "grhd2_host_fm_prepare": (C.c_int, [C.c_int32] * 3 + [C.c_double] * 4 + [c_double_p] * 2
                              + [C.POINTER(C.c_int32)]),
    "grhd2_host_fm_state": (C.c_int, [C.c_int32] * 3 + [C.c_double] * 11 + [c_double_p, C.POINTER(C.c_int32)]),
}

_cache = {}


def _load(name: str, symbols: dict):
    if name in _cache:
        return _cache[name]
    path = os.path.join(LIB_DIR, name)
    if not os.path.exists(path):
        raise RuntimeError(
            f"{path} is missing: build the native libraries first "
            "(python -c 'import __graft_entry__ as g; g.build()' or python -m grhd_b200.build)")
    lib = C.CDLL(path, mode=C.RTLD_GLOBAL)
    for sym, (res, args) in symbols.items():
        fn = getattr(lib, sym)
        fn.restype = res
        fn.argtypes = args
    _cache[name] = lib
    return lib


def gpu_lib():
    """The CUDA C-ABI library (raises if it has not been built)."""
    return _load("libgrhd2gpu.so", GPU_SYMBOLS)


def host_lib():
    """The host-side problem setup library (raises if it has not been built)."""
    return _load("libgrhd2host.so", HOST_SYMBOLS)


def dptr(arr):
    """double* of a contiguous float64 numpy array (None passes NULL)."""
    if arr is None:
        return None
    assert arr.dtype.name == "float64" and arr.flags["C_CONTIGUOUS"]
    return arr.ctypes.data_as(c_double_p)
