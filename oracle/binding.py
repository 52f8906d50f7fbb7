"""ctypes binding of the parity oracle (test infrastructure only).

Loads ``oracle/lib/libgrhd2_oracle.so``, the plain-C restatement of GRHD2's per-stage
path (``grhd2_oracle.c``).  Only the tests, the smoke check and the benchmark's CPU
baseline use it; it is never on the product path.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "lib", "libgrhd2_oracle.so")
# the same oracle calling the C library's exp (as the reference build does) in WENO3
LIB_LIBM = os.path.join(HERE, "lib", "libgrhd2_oracle_libm.so")
# the CPU baseline: the same source with the reference's optimisation flags, built on the
# host that times it (oracle/stopwatch.py); never used to check results
LIB_STOPWATCH = os.path.join(HERE, "lib", "libgrhd2_oracle_stopwatch.so")
_dp = C.POINTER(C.c_double)


class OrcConfig(C.Structure):
    _fields_ = [(n, C.c_int32) for n in (
        "nx", "ny", "nz", "nghost", "rec_method", "tvd_limiter", "riemann", "shock_sensor",
        "metric_kind", "geom_kind", "case_id", "pad0")] + [(n, C.c_double) for n in (
        "dx", "dy", "dz", "adb_idx", "g1", "cfl", "rho_floor", "p_floor", "v_max")]


class OrcMetric(C.Structure):
    _fields_ = [(n, _dp) for n in (
        "alpha_c", "beta_c", "gamma_c", "gamma_inv_c", "gmunu_c", "sqrt_gamma_c", "chris_c",
        "dg_c", "dlna_c", "alpha_fx", "beta_fx", "gamma_fx", "sqg_fx", "alpha_fy", "beta_fy",
        "gamma_fy", "sqg_fy", "alpha_fz", "beta_fz", "gamma_fz", "sqg_fz", "x_face", "y_face",
        "x_c", "michel_injector", "dust_outer")] + [("jet", C.c_double * 7)]


class OrcCounters(C.Structure):
    _fields_ = [(n, C.c_int64) for n in (
        "c2p_floor_pre", "c2p_causal_rescale", "c2p_brent_used", "c2p_root_fail", "c2p_bad_V",
        "c2p_final_sanitise", "recon_floor_clamps", "hllc_fallbacks")]

    def as_dict(self):
        return {n: int(getattr(self, n)) for n, _ in self._fields_}


_libs = {}


def build():
    """Compile the oracle with its own Makefile (gcc, no FMA contraction)."""
    subprocess.run(["make", "-s", "-C", HERE], check=True)


def lib(libm_exp: bool = False, stopwatch: bool = False):
    path = LIB_STOPWATCH if stopwatch else (LIB_LIBM if libm_exp else LIB)
    if path not in _libs:
        if stopwatch and not os.path.exists(path):
            raise RuntimeError("the stopwatch build is made on the timing host: python -m oracle.stopwatch")
        if not os.path.exists(path):
            build()
        L = C.CDLL(path)
        P, M, K = C.POINTER(OrcConfig), C.POINTER(OrcMetric), C.POINTER(OrcCounters)
        sig = {
            "orc_calc_rhs": (None, [P, M, _dp, _dp, K]),
            "orc_cfl": (C.c_int, [P, M, _dp]),
            "orc_cons_to_prim": (None, [P, M, _dp, _dp, C.c_int, C.c_int, K]),
            "orc_cons_to_prim_all": (None, [P, M, _dp, _dp, K]),
            "orc_prim_to_cons": (None, [P, M, _dp, _dp, C.c_int, C.c_int]),
            "orc_prim_to_cons_all": (None, [P, M, _dp, _dp]),
            "orc_set_boundary": (C.c_int, [P, M, _dp]),
            "orc_riemann": (None, [P, _dp, _dp, C.c_int, C.c_double, _dp, _dp, C.c_double, _dp, K]),
            "orc_physical_flux": (None, [P, _dp, C.c_int, C.c_double, _dp, _dp, C.c_double, _dp]),
            "orc_reconstruct": (None, [P, _dp, C.c_int, C.c_int, _dp, _dp, K]),
            "orc_step": (C.c_int, [P, M, _dp, _dp, _dp, _dp, C.c_double, K]),
            "orc_run": (C.c_int64, [P, M, _dp, _dp, C.c_double, C.c_double, C.c_int64, _dp, K]),
            "orc_num_threads": (C.c_int, []),
            "orc_exp": (C.c_double, [C.c_double]),
            "orc_total_mass": (C.c_double, [P, _dp]),
            "orc_gw_strain": (C.c_int, [P, M, _dp, _dp, _dp, _dp, C.c_int, C.c_double, C.c_double, _dp]),
            "orc_mdot": (C.c_int, [P, M, _dp, _dp, C.c_int, _dp]),
            "orc_horizon_radius": (C.c_int, [C.c_double, C.c_double, _dp]),
            "orc_root_brent": (C.c_double, [P, _dp, _dp]),
            "orc_sources": (None, [P, M, _dp, C.c_int, C.c_int, _dp]),
            "orc_ks_spheroidal_position": (None, [C.c_double] * 4 + [_dp]),
            "orc_gw_kinematics": (None, [C.c_double] * 5 + [_dp, _dp, C.c_int, _dp, _dp, _dp]),
            "orc_finn_evans_stress": (None, [C.c_double] * 3 + [_dp, _dp, C.c_double, _dp, _dp, _dp]),
            "orc_ppi_modes": (None, [P, _dp, _dp, _dp, _dp]),
            "orc_global_diagnostics": (None, [P, M, _dp, _dp, _dp, C.POINTER(C.c_int64)]),
        }
        for name, (res, args) in sig.items():
            f = getattr(L, name)
            f.restype, f.argtypes = res, args
        _libs[path] = L
    return _libs[path]


def _p(a):
    return None if a is None else a.ctypes.data_as(_dp)


def config_from(gcfg) -> OrcConfig:
    """orc_config from a grhd2_gpu_config (same field meanings)."""
    c = OrcConfig()
    for n in ("nx", "ny", "nz", "nghost", "rec_method", "tvd_limiter", "riemann",
              "shock_sensor", "metric_kind", "geom_kind", "case_id", "dx", "dy", "dz",
              "adb_idx", "g1", "cfl", "rho_floor", "p_floor", "v_max"):
        setattr(c, n, getattr(gcfg, n))
    return c


def metric_from(mv, bv) -> OrcMetric:
    """orc_metric from grhd2_gpu_metric_view + grhd2_gpu_bc_view (pointers are shared)."""
    m = OrcMetric()
    names = {"alpha_c": "alpha_c", "beta_c": "beta_c", "gamma_c": "gamma_c",
             "gamma_inv_c": "gamma_inv_c", "gmunu_c": "gmunu_c", "sqrt_gamma_c": "sqrt_gamma_c",
             "chris_c": "chris_c", "dg_c": "dg_c", "dlna_c": "dlna_c",
             "alpha_fx": "alpha_f_x", "beta_fx": "beta_f_x", "gamma_fx": "gamma_f_x",
             "sqg_fx": "sqrt_gamma_f_x", "alpha_fy": "alpha_f_y", "beta_fy": "beta_f_y",
             "gamma_fy": "gamma_f_y", "sqg_fy": "sqrt_gamma_f_y", "alpha_fz": "alpha_f_z",
             "beta_fz": "beta_f_z", "gamma_fz": "gamma_f_z", "sqg_fz": "sqrt_gamma_f_z",
             "x_face": "x_face", "y_face": "y_face"}
    for o, g in names.items():
        setattr(m, o, getattr(mv, g))
    m.x_c = bv.x_c
    m.michel_injector = bv.michel_injector
    m.dust_outer = bv.dust_outer
    for i in range(7):
        m.jet[i] = bv.jet[i]
    return m


class OracleRun:
    """Oracle state for one problem: p (ghosted) and up (interior), reference layout."""

    def __init__(self, problem, p=None, libm_exp: bool = False, stopwatch: bool = False):
        self.problem = problem
        self.cfg = config_from(problem.config(0))
        self._mv = problem.metric_view()
        self._bv = problem.bc_view()
        self.met = metric_from(self._mv, self._bv)
        self.p = (problem.initial_prims() if p is None else p.copy())
        self.up = np.zeros(problem.cons_shape)
        self.counters = OrcCounters()
        self.L = lib(libm_exp, stopwatch)

    def prim_to_cons(self):
        self.L.orc_prim_to_cons_all(C.byref(self.cfg), C.byref(self.met), _p(self.p), _p(self.up))

    def cons_to_prim(self):
        self.L.orc_cons_to_prim_all(C.byref(self.cfg), C.byref(self.met), _p(self.up), _p(self.p),
                                    C.byref(self.counters))

    def set_boundary(self):
        rc = self.L.orc_set_boundary(C.byref(self.cfg), C.byref(self.met), _p(self.p))
        if rc != 0:
            raise RuntimeError(f"oracle boundary error {rc}")

    def cfl(self) -> float:
        dt = C.c_double()
        rc = self.L.orc_cfl(C.byref(self.cfg), C.byref(self.met), C.byref(dt))
        if rc != 0:
            raise RuntimeError(f"oracle CFL error {rc}")
        return dt.value

    def calc_rhs(self) -> np.ndarray:
        rhs = np.zeros(self.problem.cons_shape)
        self.L.orc_calc_rhs(C.byref(self.cfg), C.byref(self.met), _p(self.p), _p(rhs),
                            C.byref(self.counters))
        return rhs

    def step(self, dt: float):
        u = np.zeros(self.problem.cons_shape)
        rhs = np.zeros(self.problem.cons_shape)
        rc = self.L.orc_step(C.byref(self.cfg), C.byref(self.met), _p(u), _p(self.up), _p(self.p),
                             _p(rhs), dt, C.byref(self.counters))
        if rc != 0:
            raise RuntimeError(f"oracle step error {rc}")

    # diagnostics: grhd2.f90:283-301, output.f90:951-1125 (serial loops)
    def total_mass(self, u: np.ndarray) -> float:
        return float(self.L.orc_total_mass(C.byref(self.cfg), _p(np.ascontiguousarray(u))))

    def mdot(self, idx_probe: int) -> float:
        out = C.c_double()
        rc = self.L.orc_mdot(C.byref(self.cfg), C.byref(self.met), _p(self.up), _p(self.p), idx_probe, C.byref(out))
        if rc != 0:
            raise ValueError("invalid accretion-probe index")
        return out.value

    def ppi_modes(self, z: np.ndarray) -> np.ndarray:
        out = np.zeros(17)
        self.L.orc_ppi_modes(C.byref(self.cfg), _p(self.up), _p(self.p), _p(np.ascontiguousarray(z)), _p(out))
        return out

    def gw_strain(self, use_log_r: bool, bh_mass: float, spin: float) -> np.ndarray:
        pb = self.problem
        x, y, z = (np.ascontiguousarray(a[pb.ng + 1:pb.ng + 1 + n]) for a, n in zip(pb.coords(), (pb.nx, pb.ny, pb.nz)))
        out = np.zeros(5)
        rc = self.L.orc_gw_strain(C.byref(self.cfg), C.byref(self.met), _p(self.p), _p(x), _p(y), _p(z),
                                  int(use_log_r), bh_mass, spin, _p(out))
        if rc < 0:
            raise ValueError("undefined horizon radius")
        return out

    def global_diagnostics(self) -> dict:
        f = np.zeros(8)
        n = np.zeros(2, dtype=np.int64)
        self.L.orc_global_diagnostics(C.byref(self.cfg), C.byref(self.met), _p(self.up), _p(self.p), _p(f),
                                      n.ctypes.data_as(C.POINTER(C.c_int64)))
        keys = ("mass_total", "disk_mass", "angular_momentum", "rho_min", "p_min", "rho_max", "p_max", "max_v_sq")
        out = dict(zip(keys, f.tolist()))
        out.update(atmosphere_cells=int(n[0]), invalid_cells=int(n[1]))
        return out

    def run(self, t0: float, final_time: float, max_steps: int = -1):
        t = C.c_double()
        n = self.L.orc_run(C.byref(self.cfg), C.byref(self.met), _p(self.up), _p(self.p), t0,
                           final_time, max_steps, C.byref(t), C.byref(self.counters))
        if n < 0:
            raise RuntimeError(f"oracle run error {n}")
        return int(n), t.value
