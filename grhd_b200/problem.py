"""Problem setup: the host side that feeds the GPU path (include/grhd2_host.h).

A :class:`Problem` is built from .par text with the reference's keys
(parameters.f90:147-349).  It owns the grid, the k-invariant metric tables
(initialization.f90:265-391), the per-case boundary data and the initial primitives
(conditions.f90:26-214) in the reference's Fortran layout.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import native as N

PROBLEM_NAMES = {
    1: "sod", 2: "strong_shock", 3: "shu_osher", 4: "kelvin_helmholtz", 5: "axisymmetric_jet",
    6: "convergence", 7: "michel", 8: "dust", 9: "offaxis_blast", 10: "fishbone_equatorial",
    11: "fishbone_sagittal", 12: "fishbone_3d"}


def par_text(problem: str, **keys) -> str:
    """Compose .par text: par_text('sod', nx=400, reconstruction='weno5')."""
    lines = [f"problem = {problem}"]
    for k, v in keys.items():
        if isinstance(v, bool):
            v = "true" if v else "false"
        lines.append(f"{k} = {v}")
    return "\n".join(lines) + "\n"


class Problem:
    """Host-side problem: grid, metric tables, boundary data, initial primitives."""

    def __init__(self, text: str, metric_cache: bool = True):
        """metric_cache=False builds no host metric cache (grhd2_problem_create_ex with
        GRHD2_PROBLEM_NO_METRIC_CACHE): for grids whose tables are built on the device."""
        lib = N.host_lib()
        h = C.c_void_p()
        err = C.create_string_buffer(512)
        rc = lib.grhd2_problem_create_ex(text.encode(), 0 if metric_cache else 1, C.byref(h), err, 512)
        if rc != 0:
            raise ValueError(f"invalid problem ({rc}): {err.value.decode()}")
        self._lib = lib
        self._h = h
        self.text = text
        self.metric_cache = metric_cache
        info = N.ProblemInfo()
        lib.grhd2_problem_info_get(h, C.byref(info))
        self.info = info
        self.nx, self.ny, self.nz, self.ng = info.nx, info.ny, info.nz, info.nghost

    @classmethod
    def from_keys(cls, problem: str, metric_cache: bool = True, **keys) -> "Problem":
        return cls(par_text(problem, **keys), metric_cache=metric_cache)

    def __del__(self):
        h = getattr(self, "_h", None)
        if h is not None and h.value:
            self._lib.grhd2_problem_destroy(h)
            self._h = None

    # ---- views -----------------------------------------------------------------
    def config(self, precision_policy: int = 0) -> N.GpuConfig:
        c = N.GpuConfig()
        self._lib.grhd2_problem_config(self._h, precision_policy, C.byref(c))
        return c

    def metric_view(self) -> N.MetricView:
        if not self.metric_cache:
            raise RuntimeError("this problem was built without a host metric cache (metric_cache=False)")
        m = N.MetricView()
        self._lib.grhd2_problem_metric(self._h, C.byref(m))
        return m

    def metric_params(self) -> N.MetricParams:
        """What grhd2_gpu_set_metric_analytic needs beyond the configuration."""
        i = self.info
        return N.MetricParams(bh_mass=i.bh_mass, a_spin=i.a_spin, x_min=i.x_min, y_min=i.y_min)

    def bc_view(self) -> N.BcView:
        b = N.BcView()
        self._lib.grhd2_problem_bc(self._h, C.byref(b))
        return b

    @property
    def prim_shape(self):
        """numpy shape (C order) of the Fortran array p(5,-g:nx+g,-g:ny+g,-g:nz+g)."""
        g = self.ng
        return (self.nz + 2 * g + 1, self.ny + 2 * g + 1, self.nx + 2 * g + 1, 5)

    @property
    def cons_shape(self):
        """numpy shape (C order) of the Fortran array u(5,nx,ny,nz)."""
        return (self.nz, self.ny, self.nx, 5)

    @property
    def n_cells(self) -> int:
        return self.nx * self.ny * self.nz

    def initial_prims(self) -> np.ndarray:
        """A fresh copy of the initial ghosted primitives (Fortran order as a C array)."""
        n = self._lib.grhd2_problem_prim_size(self._h)
        ptr = self._lib.grhd2_problem_prims(self._h)
        return np.ctypeslib.as_array(ptr, shape=(n,)).copy().reshape(self.prim_shape)

    def prims_view(self) -> np.ndarray:
        """The initial ghosted primitives in the problem's own buffer (no copy; valid while
        the problem lives and only to be read)."""
        n = self._lib.grhd2_problem_prim_size(self._h)
        ptr = self._lib.grhd2_problem_prims(self._h)
        v = np.ctypeslib.as_array(ptr, shape=(n,)).reshape(self.prim_shape)
        v.flags.writeable = False
        return v

    def perturb(self, p: np.ndarray) -> np.ndarray:
        """Apply the configured perturbation to a ghosted primitive array in place."""
        assert p.shape == self.prim_shape and p.dtype == np.float64
        rc = self._lib.grhd2_problem_perturb(self._h, N.dptr(p))
        if rc != 0:
            raise ValueError("invalid perturbation parameters")
        return p

    def coords(self):
        g = self.ng
        lib = self._lib
        x = np.ctypeslib.as_array(lib.grhd2_problem_x(self._h), shape=(self.nx + 2 * g + 1,)).copy()
        y = np.ctypeslib.as_array(lib.grhd2_problem_y(self._h), shape=(self.ny + 2 * g + 1,)).copy()
        z = np.ctypeslib.as_array(lib.grhd2_problem_z(self._h), shape=(self.nz + 2 * g + 1,)).copy()
        return x, y, z

    def accretion_probe(self) -> int:
        """Index of the accretion probe (initialization.f90:146-161): the first cell whose
        centre lies outside the horizon r_+ = M + sqrt(M^2 - a^2) (log r coordinate when the
        grid is logarithmic); 1 when the horizon is below the grid, 0 when above it."""
        import math
        info = self.info
        m, a = info.bh_mass, info.a_spin
        r_h = m + math.sqrt(max(0.0, m * m - a * a))
        if self.config(0).use_log_r:
            r_h = math.log(r_h)
        x, _, _ = self.coords()
        g = self.ng
        xc = x[g + 1:g + 1 + self.nx]
        m = N.MetricView()
        self._lib.grhd2_problem_metric(self._h, C.byref(m))  # x_face is set with or without the cache
        xf = np.ctypeslib.as_array(m.x_face, shape=(self.nx + 1,))
        if r_h < xf[0]:
            return 1
        if r_h > xf[self.nx]:
            return 0
        for i, xi in enumerate(xc, start=1):
            if xi >= r_h:
                return i
        return 0

    def eval_metric(self, x: float, y: float) -> dict:
        out = {k: np.zeros(n) for k, n in (("beta", 3), ("gamma", 9), ("gmunu", 16),
                                            ("dlnalpha", 4), ("chris", 64), ("dg", 48))}
        a = C.c_double()
        d = C.c_double()
        self._lib.grhd2_problem_eval_metric(
            self._h, x, y, C.byref(a), N.dptr(out["beta"]), N.dptr(out["gamma"]),
            N.dptr(out["gmunu"]), C.byref(d), N.dptr(out["dlnalpha"]), N.dptr(out["chris"]),
            N.dptr(out["dg"]))
        out["alpha"] = a.value
        out["det"] = d.value
        # Fortran-order views
        out["gamma"] = out["gamma"].reshape(3, 3).T.copy()
        out["gmunu"] = out["gmunu"].reshape(4, 4).T.copy()
        out["chris"] = out["chris"].reshape(4, 4, 4).transpose(2, 1, 0).copy()
        out["dg"] = out["dg"].reshape(3, 4, 4).transpose(2, 1, 0).copy()
        return out
