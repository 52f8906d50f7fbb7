"""Python front end of the drop-in boundary (include/grhd2_gpu.h).

:class:`GpuGrid` owns one ``grhd2_gpu`` handle: the device-resident state of one grid and
the per-stage kernels.  It mirrors the module-level surface of the reference that the
C-ABI replaces -- ``calc_rhs``, ``update_adaptive_dt``, ``cons_to_prim``, ``prim_to_cons``,
``set_boundary_conditions`` and the SSP-RK3 step of grhd2.f90 -- with the same argument
meaning, layouts and error behaviour (a nonzero status raises :class:`GpuError` carrying
the library's message).  There is no CPU fallback: a missing library or device raises.
"""
from __future__ import annotations

import ctypes as C
import math
import time

import numpy as np

from . import native as N
from .problem import Problem

PRECISION = {"fp64": 0, "mixed": 1, "mixed_comp64": 2, "mixed_comp32": 3}
"""Precision policies (include/grhd2_gpu.h GRHD2_PREC_*): the FP64 parity path; the mixed
policy (FP32 reconstruction, Riemann fluxes and metric contraction, FP64 lapse and
sqrt(gamma) factors, con2prim and RK state); the mixed policy with the RK3 accumulation
compensated by an FP64 or an FP32 carry."""


class GpuError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"grhd2_gpu error {code}: {msg}")
        self.code = code


class GpuGrid:
    """One grid on the GPU, built from a :class:`Problem` (or explicit config/tables)."""

    def __init__(self, problem: Problem, precision: str = "fp64", upload_initial: bool = True,
                 stream: int | None = None, metric: str | None = None):
        """stream: a cudaStream_t (integer) the handle launches on; None creates a private
        one.  Grids that will step together in a :class:`GpuBatch` share one stream.
        metric: "host" uploads the problem's metric cache (grhd2_gpu_set_metric); "device"
        builds the same tables from the analytic metric on the GPU
        (grhd2_gpu_set_metric_analytic); None picks "host" when the problem has a host
        cache and "device" when it was built without one."""
        if metric is None:
            metric = "host" if problem.metric_cache else "device"
        if metric not in ("host", "device"):
            raise ValueError(f"metric must be 'host' or 'device', not {metric!r}")
        self.lib = N.gpu_lib()
        self.problem = problem
        self.precision = precision
        self.cfg = problem.config(PRECISION[precision])
        self._mv = problem.metric_view() if metric == "host" else None
        self._bv = problem.bc_view()
        h = C.c_void_p()
        if stream is None:
            rc = self.lib.grhd2_gpu_create(C.byref(self.cfg), C.byref(h))
        else:
            rc = self.lib.grhd2_gpu_create_on_stream(C.byref(self.cfg), C.c_void_p(stream), C.byref(h))
        self._h = h
        self._check(rc)
        t0 = time.perf_counter()
        if metric == "host":
            self._check(self.lib.grhd2_gpu_set_metric(self._h, C.byref(self._mv)))
        else:
            self._check(self.lib.grhd2_gpu_set_metric_analytic(self._h, C.byref(problem.metric_params())))
        # wall time of the metric-table call (both return with the tables on the device)
        self.metric_seconds = time.perf_counter() - t0
        self._check(self.lib.grhd2_gpu_set_bc_data(self._h, C.byref(self._bv)))
        if upload_initial:
            p0 = problem.initial_prims()
            self.upload(p=p0)
            self.prim_to_cons()

    # ---- plumbing ------------------------------------------------------------------
    def _check(self, rc: int):
        if rc != 0:
            msg = self.lib.grhd2_gpu_last_error(self._h) if self._h else b"create failed"
            raise GpuError(rc, (msg or b"").decode())

    def close(self):
        if getattr(self, "_h", None) is not None and self._h.value:
            self.lib.grhd2_gpu_destroy(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def metric_table(self, which: int) -> np.ndarray:
        """The device metric table `which` (0 centre, 1-3 the x, y, z faces) as a
        (fields, entries) array; empty for a direction without faces."""
        n = C.c_size_t()
        self._check(self.lib.grhd2_gpu_metric_table(self._h, which, None, 0, C.byref(n)))
        out = np.empty(n.value, dtype=np.float64)
        if n.value:
            self._check(self.lib.grhd2_gpu_metric_table(self._h, which, N.dptr(out), out.size, None))
        nfield = 74 if which == 0 else 21
        return out.reshape(nfield, -1)

    # ---- the reference surface -------------------------------------------------------
    def upload(self, up: np.ndarray | None = None, p: np.ndarray | None = None):
        if up is not None:
            up = np.ascontiguousarray(up, dtype=np.float64)
            assert up.size == 5 * self.problem.n_cells
        if p is not None:
            p = np.ascontiguousarray(p, dtype=np.float64)
            assert p.shape == self.problem.prim_shape
        self._check(self.lib.grhd2_gpu_upload(self._h, N.dptr(up), N.dptr(p)))

    def prim_to_cons(self):
        """up = prim_to_cons(p) over interior cells (grhd2.f90:126-134)."""
        self._check(self.lib.grhd2_gpu_prim_to_cons_all(self._h))

    def cons_to_prim(self):
        """p = cons_to_prim(up), up floored in place (grhd2.f90:252-260)."""
        self._check(self.lib.grhd2_gpu_cons_to_prim_all(self._h))

    def set_boundary(self):
        self._check(self.lib.grhd2_gpu_set_boundary(self._h))

    def cfl(self) -> float:
        """dt of update_adaptive_dt (evolution.f90:198)."""
        dt = C.c_double()
        self._check(self.lib.grhd2_gpu_cfl(self._h, C.byref(dt)))
        return dt.value

    def step(self, dt: float):
        """One SSP-RK3 step (grhd2.f90:232-265), asynchronous on the handle's stream."""
        self._check(self.lib.grhd2_gpu_step(self._h, dt))

    def run(self, t0: float, final_time: float, max_steps: int = -1):
        """Time loop of grhd2.f90:179-265 without I/O; returns (steps, t)."""
        t = C.c_double()
        n = C.c_int64()
        self._check(self.lib.grhd2_gpu_run(self._h, t0, final_time, max_steps, C.byref(t), C.byref(n)))
        return n.value, t.value

    def calc_rhs(self) -> np.ndarray:
        """calc_rhs(p) of the resident primitives (evolution.f90:30), (5,nx,ny,nz) layout."""
        rhs = np.empty(self.problem.cons_shape)
        self._check(self.lib.grhd2_gpu_calc_rhs(self._h, N.dptr(rhs)))
        return rhs

    def download(self, p_template: np.ndarray | None = None, want_up: bool = True, want_p: bool = True):
        """(up, p): p holds interior cells and single-direction ghosts; the remaining
        ghost entries keep the values of p_template (zeros by default)."""
        up = np.empty(self.problem.cons_shape) if want_up else None
        p = None
        if want_p:
            p = np.zeros(self.problem.prim_shape) if p_template is None else np.array(p_template, dtype=np.float64)
        self._check(self.lib.grhd2_gpu_download(self._h, N.dptr(up), N.dptr(p)))
        return up, p

    # ---- diagnostics (device reductions) -------------------------------------------
    def global_diagnostics(self) -> dict:
        """calc_global_diagnostics (output.f90:1052) of the resident state."""
        d = N.Diagnostics()
        self._check(self.lib.grhd2_gpu_global_diagnostics(self._h, C.byref(d)))
        return d.as_dict()

    def total_mass(self) -> float:
        """The time loop's mass monitor (grhd2.f90:283-301): sum u(D) dx dy dz."""
        out = C.c_double()
        self._check(self.lib.grhd2_gpu_total_mass(self._h, C.byref(out)))
        return out.value

    def mdot(self, idx_probe: int | None = None) -> float:
        """calc_m_dot (output.f90:951) at the probe cell (default: the problem's)."""
        idx = self.problem.accretion_probe() if idx_probe is None else idx_probe
        out = C.c_double()
        self._check(self.lib.grhd2_gpu_mdot(self._h, int(idx), C.byref(out)))
        return out.value

    def ppi_modes(self) -> np.ndarray:
        """calc_ppi_modes (output.f90:995) values without the time column (17 numbers)."""
        z = np.ascontiguousarray(self.problem.coords()[2][self.problem.ng + 1:self.problem.ng + 1 + self.problem.nz])
        out = np.zeros(17)
        self._check(self.lib.grhd2_gpu_ppi_modes(self._h, N.dptr(z), N.dptr(out)))
        return out

    def gw_strain(self) -> np.ndarray:
        """calc_gw_strain (output.f90:852): h_plus, h_cross, Ixx, Iyy, Ixy of the resident state."""
        pb = self.problem
        x, y, z = (np.ascontiguousarray(a[pb.ng + 1:pb.ng + 1 + n]) for a, n in zip(pb.coords(), (pb.nx, pb.ny, pb.nz)))
        spin = pb.info.a_spin if self.cfg.metric_kind == 2 else 0.0
        out = np.zeros(5)
        self._check(self.lib.grhd2_gpu_gw_strain(self._h, N.dptr(x), N.dptr(y), N.dptr(z), int(self.cfg.use_log_r),
                                                 pb.info.bh_mass, spin, N.dptr(out)))
        return out

    def vtk_cell_data(self) -> np.ndarray:
        """The 7 big-endian cell fields of a VTK frame (output.f90:398-453), shape
        (7, nz, ny, nx), dtype '>f8'; v^r and beta^r scaled by exp(x) on log-r grids."""
        pb = self.problem
        r_scale = None
        if self.cfg.use_log_r:
            x = pb.coords()[0][pb.ng + 1:pb.ng + 1 + pb.nx]
            r_scale = np.array([math.exp(v) for v in x])  # the C library's exp, as the reference's writer
        out = np.empty((7, pb.nz, pb.ny, pb.nx), dtype=">f8")
        self._check(self.lib.grhd2_gpu_vtk_cell_data(self._h, N.dptr(r_scale), out.ctypes.data_as(C.c_void_p)))
        return out

    def counters(self) -> dict:
        c = N.Counters()
        self._check(self.lib.grhd2_gpu_get_counters(self._h, C.byref(c)))
        return c.as_dict()

    def reset_counters(self):
        self._check(self.lib.grhd2_gpu_reset_counters(self._h))

    def synchronize(self):
        self._check(self.lib.grhd2_gpu_synchronize(self._h))

    def set_stream(self, stream: int | None):
        """Move the handle to another cudaStream_t (None: a new private stream)."""
        self._check(self.lib.grhd2_gpu_set_stream(self._h, C.c_void_p(stream) if stream else None))

    @property
    def device_bytes(self) -> int:
        """Device bytes the handle allocated (the admission estimate of its config)."""
        return int(self.lib.grhd2_gpu_device_bytes(C.byref(self.cfg)))

    @property
    def stream_ptr(self) -> int:
        """The handle's cudaStream_t as an integer (for torch.cuda.ExternalStream)."""
        s = C.c_void_p()
        self._check(self.lib.grhd2_gpu_get_stream(self._h, C.byref(s)))
        return s.value or 0

    def profile_step(self, dt: float):
        """[(kernel name, ms)] for every launch of one step."""
        cap = 64
        ms = (C.c_float * cap)()
        names = (C.c_char_p * cap)()
        n = C.c_int()
        self._check(self.lib.grhd2_gpu_profile_step(self._h, dt, ms, names, cap, C.byref(n)))
        return [(names[k].decode(), float(ms[k])) for k in range(min(n.value, cap))]

    # ---- single-face entry points ------------------------------------------------------
    def riemann_faces(self, dir: int, qL, qR, alpha, beta, gamma, sqg) -> np.ndarray:
        """resolve_riemann_problem (fluxes.f90:56) for n independent faces.
        qL, qR: (n,5); alpha, sqg: (n,); beta: (n,3); gamma: (n,3,3) (symmetric)."""
        qL, qR = (np.ascontiguousarray(a, dtype=np.float64) for a in (qL, qR))
        n = qL.shape[0]
        alpha, sqg = (np.ascontiguousarray(np.broadcast_to(a, (n,)), dtype=np.float64) for a in (alpha, sqg))
        beta = np.ascontiguousarray(np.broadcast_to(beta, (n, 3)), dtype=np.float64)
        # Fortran (3,3) order per face: g[(a-1)+3(b-1)] -> transpose of a C (3,3)
        gamma = np.ascontiguousarray(np.broadcast_to(gamma, (n, 3, 3)).transpose(0, 2, 1), dtype=np.float64)
        flux = np.empty((n, 5))
        self._check(self.lib.grhd2_gpu_riemann_faces(self._h, n, dir, N.dptr(qL), N.dptr(qR), N.dptr(alpha),
                                                     N.dptr(beta), N.dptr(gamma), N.dptr(sqg), N.dptr(flux)))
        return flux

    def riemann_faces_noalloc(self, dir: int, qL, qR, alpha, beta, gamma, sqg) -> np.ndarray:
        """riemann_faces through the allocation-free entry point: the library allocates
        nothing (fixed device scratch of GRHD2_GPU_NOALLOC_MAX_FACES faces; more raises)."""
        qL, qR = (np.ascontiguousarray(a, dtype=np.float64) for a in (qL, qR))
        n = qL.shape[0]
        alpha, sqg = (np.ascontiguousarray(np.broadcast_to(a, (n,)), dtype=np.float64) for a in (alpha, sqg))
        beta = np.ascontiguousarray(np.broadcast_to(beta, (n, 3)), dtype=np.float64)
        gamma = np.ascontiguousarray(np.broadcast_to(gamma, (n, 3, 3)).transpose(0, 2, 1), dtype=np.float64)
        flux = np.empty((n, 5))
        self._check(self.lib.grhd2_gpu_riemann_faces_noalloc(
            self._h, n, dir, N.dptr(qL), N.dptr(qR), N.dptr(alpha), N.dptr(beta), N.dptr(gamma), N.dptr(sqg),
            N.dptr(flux)))
        return flux

    def physical_flux(self, dir: int, q, alpha, beta, gamma, sqg) -> np.ndarray:
        """calc_fluxes (equations.f90:434) for n states."""
        q = np.ascontiguousarray(q, dtype=np.float64)
        n = q.shape[0]
        alpha, sqg = (np.ascontiguousarray(np.broadcast_to(a, (n,)), dtype=np.float64) for a in (alpha, sqg))
        beta = np.ascontiguousarray(np.broadcast_to(beta, (n, 3)), dtype=np.float64)
        gamma = np.ascontiguousarray(np.broadcast_to(gamma, (n, 3, 3)).transpose(0, 2, 1), dtype=np.float64)
        flux = np.empty((n, 5))
        self._check(self.lib.grhd2_gpu_physical_flux(self._h, n, dir, N.dptr(q), N.dptr(alpha), N.dptr(beta),
                                                     N.dptr(gamma), N.dptr(sqg), N.dptr(flux)))
        return flux


class GpuBatch:
    """Many grids stepped together: one launch per kernel kind and scheme group, so grids
    of uneven sizes fill the GPU together; a step can replay as one CUDA graph.  Each grid
    keeps its own clock (t, final time, CFL dt) on the device and stops by itself when it
    reaches its final time or step limit."""

    def __init__(self, grids: list[GpuGrid]):
        self.lib = N.gpu_lib()
        self.grids = list(grids)
        arr = (C.c_void_p * len(self.grids))(*[g._h.value for g in self.grids])
        b = C.c_void_p()
        rc = self.lib.grhd2_gpu_batch_create(arr, len(self.grids), C.byref(b))
        self._b = b
        self._check(rc)

    def _check(self, rc: int):
        if rc != 0:
            msg = self.lib.grhd2_gpu_batch_last_error(self._b) if self._b else b"batch create failed"
            raise GpuError(rc, (msg or b"").decode())

    def close(self):
        if getattr(self, "_b", None) is not None and self._b.value:
            self.lib.grhd2_gpu_batch_destroy(self._b)
            self._b = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def set_clock(self, k: int, t0: float, final_time: float, max_steps: int = -1):
        """Grid k runs from t0 to final_time (at most max_steps steps, -1 unlimited) with its
        CFL dt clamped to the final time, as the time loop of grhd2.f90:179-230."""
        self._check(self.lib.grhd2_gpu_batch_set_clock(self._b, k, t0, final_time, max_steps))

    def step(self, nsteps: int = 1, graph: bool = True):
        """Enqueue nsteps batched steps (asynchronous)."""
        self._check(self.lib.grhd2_gpu_batch_step(self._b, nsteps, 1 if graph else 0))

    def cons_to_prim(self):
        """cons_to_prim of every grid's uploaded conserved state, one launch per scheme
        group (asynchronous; the results of GpuGrid.cons_to_prim on each grid)."""
        self._check(self.lib.grhd2_gpu_batch_cons_to_prim(self._b))

    def clocks(self):
        """(t, steps, active) arrays of every grid in one device read (synchronises)."""
        n = len(self.grids)
        t = np.empty(n)
        st = np.empty(n, dtype=np.int64)
        ac = np.empty(n, dtype=np.int32)
        self._check(self.lib.grhd2_gpu_batch_clocks(
            self._b, N.dptr(t), st.ctypes.data_as(C.POINTER(C.c_int64)), ac.ctypes.data_as(C.POINTER(C.c_int))))
        return t, st, ac.astype(bool)

    def clock(self, k: int):
        """(t, steps, active) of grid k (synchronises the stream)."""
        t, n, a = C.c_double(), C.c_int64(), C.c_int()
        self._check(self.lib.grhd2_gpu_batch_get_clock(self._b, k, C.byref(t), C.byref(n), C.byref(a)))
        return t.value, n.value, bool(a.value)

    FLUX_VARIANTS = {"auto": -1, "split": 0, "fused": 1, "split_var": 2}

    def set_flux_variant(self, variant: str):
        """'split' (recon + Riemann kernels), 'fused' (one kernel) or 'auto' (tuned/cached)."""
        self._check(self.lib.grhd2_gpu_batch_set_flux_variant(self._b, self.FLUX_VARIANTS[variant]))

    STAGE_MODES = {"auto": -1, "off": 0, "on": 1}

    def set_stage_kernel(self, mode: str):
        """'on' (one stage kernel per RK stage for the batch's 1D and 2D grids: every face
        of a tile and its cell update through shared memory), 'off' (face and cell
        kernels) or 'auto' (the library's choice)."""
        self._check(self.lib.grhd2_gpu_batch_set_stage_kernel(self._b, self.STAGE_MODES[mode]))

    @property
    def stage_groups(self) -> int:
        """Scheme groups of the batch that step with the stage kernel."""
        rc = self.lib.grhd2_gpu_batch_stage_kernel(self._b)
        if rc < 0:
            self._check(rc)
        return rc

    STEP_MODES = {"auto": -1, "graph": 0, "persistent": 1}

    def set_step_mode(self, mode: str):
        """'graph' (stage kernels replayed as a CUDA graph), 'persistent' (one cooperative
        launch per scheme group runs whole steps) or 'auto' (the library's choice: graph)."""
        self._check(self.lib.grhd2_gpu_batch_set_step_mode(self._b, self.STEP_MODES[mode]))

    @property
    def step_mode(self) -> str:
        rc = self.lib.grhd2_gpu_batch_step_mode(self._b)
        if rc < 0:
            self._check(rc)
        return "persistent" if rc == 1 else "graph"

    def set_tile(self, tx: int):
        """Face-kernel block tile extent along i (32, 64, 128, 256; 0 = automatic)."""
        self._check(self.lib.grhd2_gpu_batch_set_tile(self._b, tx))

    def autotune(self, reps: int = 5):
        """Time every (flux variant, tile) pair per scheme group and direction; returns the
        choices (group order, x before y before z) as (variant name, tile extent)."""
        cap = 64
        var = (C.c_int * cap)()
        til = (C.c_int * cap)()
        n = C.c_int()
        self._check(self.lib.grhd2_gpu_batch_autotune(self._b, reps, var, til, cap, C.byref(n)))
        names = {v: k for k, v in self.FLUX_VARIANTS.items()}
        return [(names[var[k]], int(til[k])) for k in range(min(n.value, cap))]

    def profile_step(self):
        """[(kernel name, ms)] for every launch of one batched step."""
        cap = 256
        ms = (C.c_float * cap)()
        names = (C.c_char_p * cap)()
        n = C.c_int()
        self._check(self.lib.grhd2_gpu_batch_profile_step(self._b, ms, names, cap, C.byref(n)))
        return [(names[k].decode(), float(ms[k])) for k in range(min(n.value, cap))]


def l1_relative(a: np.ndarray, b: np.ndarray) -> np.ndarray:
    """Per-variable sum|a-b| / sum|b| over interior cells; arrays in (…,5) layout."""
    a = a.reshape(-1, 5)
    b = b.reshape(-1, 5)
    den = np.abs(b).sum(axis=0)
    num = np.abs(a - b).sum(axis=0)
    return np.where(den > 0, num / np.where(den > 0, den, 1.0), num)
