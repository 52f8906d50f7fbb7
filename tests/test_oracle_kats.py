"""Pins the CPU oracle against the known-answer tests of the reference's own test programs.

Each case restates one check of tests/test_hllc_fluxes.f90, tests/test_multidimensional_cfl.f90,
tests/test_polar_boundaries.f90, tests/test_case_corrections.f90, tests/test_gw_geometry.f90
or tests/test_gw_stress.f90 (file:line in the docstrings) with the same inputs and
tolerances, run through the oracle.  The same flux, CFL and boundary KATs run through the
GPU C-ABI in test_gpu_kats.py; the device's GW strain equals the oracle's
(test_diagnostics.py).
"""
import ctypes as C
import math

import numpy as np
import pytest

from oracle import binding as B

ADB = 4.0 / 3.0
G1 = ADB / (ADB - 1.0)
V_MAX = 1.0 - 1.0e-5
EPS = np.finfo(float).eps


def cfg(metric=0, geom=0, rs=2, **kw):
    c = B.OrcConfig()
    c.nx, c.ny, c.nz, c.nghost = 4, 1, 1, 3
    c.rec_method, c.tvd_limiter, c.riemann, c.shock_sensor = 5, 3, rs, 0
    c.metric_kind, c.geom_kind, c.case_id = metric, geom, 1
    c.dx = c.dy = c.dz = 1.0
    c.adb_idx, c.g1, c.cfl = ADB, G1, 0.4
    c.rho_floor, c.p_floor, c.v_max = 1e-10, 1e-13, V_MAX
    for k, v in kw.items():
        setattr(c, k, v)
    return c


def _p(a):
    return np.ascontiguousarray(a, dtype=np.float64).ctypes.data_as(C.POINTER(C.c_double))


def riemann(c, qL, qR, d, alpha, beta, g, sqg):
    out = np.zeros(5)
    gF = np.ascontiguousarray(np.asarray(g, dtype=float).T)  # Fortran (3,3)
    qL, qR, beta = (np.ascontiguousarray(x, dtype=float) for x in (qL, qR, beta))
    B.lib().orc_riemann(C.byref(c), _p(qL), _p(qR), d, alpha, _p(beta), _p(gF), sqg, _p(out), None)
    return out


def phys_flux(c, q, d, alpha, beta, g, sqg):
    out = np.zeros(5)
    gF = np.ascontiguousarray(np.asarray(g, dtype=float).T)
    q, beta = (np.ascontiguousarray(x, dtype=float) for x in (q, beta))
    B.lib().orc_physical_flux(C.byref(c), _p(q), d, alpha, _p(beta), _p(gF), sqg, _p(out))
    return out


def close(actual, expected, tol):
    """assert_close of test_hllc_fluxes.f90:62-78."""
    scale = max(1.0, np.max(np.abs(expected)))
    err = np.max(np.abs(actual - expected)) / scale
    assert np.all(np.isfinite(actual)) and err <= tol, (err, actual, expected)


I3 = np.eye(3)
G_GEN = np.array([[2.0, 0.08, -0.35], [0.08, 1.5, 0.10], [-0.35, 0.10, 3.0]])


def test_hllc_uniform_cartesian():
    """test_hllc_fluxes.f90:95-110: uniform state -> physical flux, every direction."""
    c = cfg()
    q = [1.2, 0.25, 0.12, -0.07, 0.05]
    for d in (1, 2, 3):
        close(riemann(c, q, q, d, 1.0, np.zeros(3), I3, 1.0), phys_flux(c, q, d, 1.0, np.zeros(3), I3, 1.0), 2e-12)


def test_hllc_uniform_general_metric():
    """test_hllc_fluxes.f90:113-133 (Kerr-Schild-like metric with g13 != 0 and shift)."""
    c = cfg(metric=2, geom=3)
    sqg = np.sqrt(np.linalg.det(G_GEN))
    beta = np.array([0.18, -0.05, 0.09])
    q = [0.9, 0.12, 0.08, -0.04, 0.06]
    for d in (1, 2, 3):
        close(riemann(c, q, q, d, 0.73, beta, G_GEN, sqg), phys_flux(c, q, d, 0.73, beta, G_GEN, sqg), 5e-12)


def test_hllc_stationary_contact():
    """test_hllc_fluxes.f90:136-149."""
    c = cfg()
    qL, qR = [1.0, 0.4, 0, 0, 0], [0.125, 0.4, 0, 0, 0]
    close(riemann(c, qL, qR, 1, 1.0, np.zeros(3), I3, 1.0), phys_flux(c, qL, 1, 1.0, np.zeros(3), I3, 1.0), 2e-12)


def test_hllc_moving_contact():
    """test_hllc_fluxes.f90:152-165: right-moving contact selects the left state."""
    c = cfg()
    qL, qR = [1.0, 0.1, 0.2, 0.03, -0.02], [0.2, 0.1, 0.2, 0.03, -0.02]
    close(riemann(c, qL, qR, 1, 1.0, np.zeros(3), I3, 1.0), phys_flux(c, qL, 1, 1.0, np.zeros(3), I3, 1.0), 3e-12)


def test_hllc_shifted_contact():
    """test_hllc_fluxes.f90:168-181: shift 0.3, lapse 0.8: selects the right state."""
    c = cfg(metric=2, geom=3)
    beta = np.array([0.3, 0, 0])
    qL, qR = [1.0, 0.1, 0.2, 0.03, -0.02], [0.2, 0.1, 0.2, 0.03, -0.02]
    close(riemann(c, qL, qR, 1, 0.8, beta, I3, 1.0), phys_flux(c, qR, 1, 0.8, beta, I3, 1.0), 3e-12)


def test_hllc_tangential_contact():
    """test_hllc_fluxes.f90:184-197: exact flux (0, 0, p, 0, 0)."""
    c = cfg()
    qL, qR = [1.0, 0.2, 0.0, 0.30, -0.10], [0.4, 0.2, 0.0, -0.20, 0.15]
    close(riemann(c, qL, qR, 1, 1.0, np.zeros(3), I3, 1.0), np.array([0, 0, 0.2, 0, 0]), 3e-12)


def test_hllc_general_metric_contact():
    """test_hllc_fluxes.f90:200-219."""
    c = cfg(metric=2, geom=3)
    g = np.diag([2.2, 1.4, 3.1])
    g[0, 2] = g[2, 0] = -0.45
    sqg = np.sqrt(np.linalg.det(g))
    qL, qR = [1.0, 0.15, 0.0, 0.04, 0.08], [0.3, 0.15, 0.0, -0.03, -0.05]
    close(riemann(c, qL, qR, 1, 0.75, np.zeros(3), g, sqg), phys_flux(c, qL, 1, 0.75, np.zeros(3), g, sqg), 5e-12)


def test_hllc_general_metric_moving_contact():
    """test_hllc_fluxes.f90:222-238."""
    c = cfg(metric=2, geom=3)
    beta = np.array([0.02, -0.01, 0.03])
    sqg = np.sqrt(np.linalg.det(G_GEN))
    qL, qR = [1.1, 0.12, 0.08, -0.04, 0.06], [0.25, 0.12, 0.08, -0.04, 0.06]
    close(riemann(c, qL, qR, 1, 0.8, beta, G_GEN, sqg), phys_flux(c, qL, 1, 0.8, beta, G_GEN, sqg), 8e-12)


def test_hllc_atmosphere_scale_contact():
    """test_hllc_fluxes.f90:241-254 (absolute 1e-18)."""
    c = cfg()
    qL, qR = [4e-10, 2e-13, 0.12, 0, 0], [1.2e-10, 2e-13, 0.12, 0, 0]
    close(riemann(c, qL, qR, 1, 1.0, np.zeros(3), I3, 1.0), phys_flux(c, qL, 1, 1.0, np.zeros(3), I3, 1.0), 1e-18)


def test_hllc_scale_invariance():
    """test_hllc_fluxes.f90:257-277: density and pressure scaled by 1e-10."""
    c = cfg()
    qL, qR = np.array([1.0, 1.0, 0.30, 0.10, 0.0]), np.array([0.125, 0.10, -0.10, -0.05, 0.02])
    sL, sR = qL.copy(), qR.copy()
    sL[:2] *= 1e-10
    sR[:2] *= 1e-10
    ref = riemann(c, qL, qR, 1, 1.0, np.zeros(3), I3, 1.0)
    small = riemann(c, sL, sR, 1, 1.0, np.zeros(3), I3, 1.0)
    close(small / 1e-10, ref, 2e-11)


def test_hllc_strong_relativistic_jump():
    """test_hllc_fluxes.f90:280-292: 1e3 : 1e-2 pressure jump gives a finite flux."""
    c = cfg()
    out = riemann(c, [1.0, 1e3, 0, 0, 0], [1.0, 1e-2, 0, 0, 0], 1, 1.0, np.zeros(3), I3, 1.0)
    assert np.all(np.isfinite(out))


def test_hlle_uniform_states_give_physical_flux():
    """The uniform-state HLLC cases also pin HLLE (its star region collapses)."""
    for metric, geom, g, alpha, beta in ((0, 0, I3, 1.0, np.zeros(3)),
                                         (2, 3, G_GEN, 0.73, np.array([0.18, -0.05, 0.09]))):
        c = cfg(metric=metric, geom=geom, rs=1)
        sqg = np.sqrt(np.linalg.det(g))
        q = [0.9, 0.12, 0.08, -0.04, 0.06]
        for d in (1, 2, 3):
            close(riemann(c, q, q, d, alpha, beta, g, sqg), phys_flux(c, q, d, alpha, beta, g, sqg), 5e-12)


# ---------------------------------------------------------------------------------------
class MetricArrays:
    """Fake metric caches as in the reference tests (constant lapse/shift/inverse metric)."""

    def __init__(self, nx, ny, lapse=1.0, shift=(0, 0, 0), inv_diag=(1, 1, 1)):
        n = nx * ny
        self.alpha = np.full(n, lapse)
        self.beta = np.tile(np.asarray(shift, float), n)
        gi = np.zeros((n, 3, 3))
        for d in range(3):
            gi[:, d, d] = inv_diag[d]
        self.ginv = gi.reshape(-1).copy()
        self.m = B.OrcMetric()
        self.m.alpha_c = _p(self.alpha)
        self.m.beta_c = _p(self.beta)
        self.m.gamma_inv_c = _p(self.ginv)


@pytest.mark.parametrize("nx,ny,nz,dx,dy,dz,lapse,shift,inv,expected", [
    (4, 1, 1, 0.5, 1.0, 1.0, 1.0, (0, 0, 0), (1, 1, 1), 0.4 / (1.0 / 0.5)),
    (4, 3, 1, 0.5, 0.25, 1.0, 1.0, (0, 0, 0), (1, 4, 1), 0.4 / (1.0 / 0.5 + 2.0 / 0.25)),
    (4, 3, 2, 0.5, 0.25, 0.125, 0.8, (0.1, -0.2, 0.05), (1, 4, 9), 0.4 / (0.9 / 0.5 + 1.8 / 0.25 + 2.45 / 0.125)),
])
def test_multidimensional_cfl(nx, ny, nz, dx, dy, dz, lapse, shift, inv, expected):
    """test_multidimensional_cfl.f90:12-25: additive CFL within 64 eps."""
    c = cfg(nx=nx, ny=ny, nz=nz, dx=dx, dy=dy, dz=dz, cfl=0.4)
    M = MetricArrays(nx, ny, lapse, shift, inv)
    dt = C.c_double()
    assert B.lib().orc_cfl(C.byref(c), C.byref(M.m), C.byref(dt)) == 0
    assert abs(dt.value - expected) <= 64 * EPS * max(1.0, abs(expected))


# ---------------------------------------------------------------------------------------
def fortran_state(nx, ny, nz, g, fill):
    return np.full((nz + 2 * g + 1, ny + 2 * g + 1, nx + 2 * g + 1, 5), fill)


def at(q, g, i, j, k):
    return q[k + g, j + g, i + g]


def fill_interior(q, nx, ny, nz, g):
    """test_polar_boundaries.f90:117-131."""
    for k in range(1, nz + 1):
        for j in range(1, ny + 1):
            for i in range(1, nx + 1):
                for comp in range(1, 6):
                    q[k + g, j + g, i + g, comp - 1] = 1.0e5 * comp + 1.0e3 * i + 10.0 * j + k


def set_bc(c, M, q):
    return B.lib().orc_set_boundary(C.byref(c), C.byref(M.m), _p(q)) if q.flags["C_CONTIGUOUS"] else None


def test_polar_boundaries_3d():
    """test_polar_boundaries.f90:80-95, 134-161: trans-polar ghost map and phi periodicity."""
    nx, ny, nz, g = 3, 4, 6, 2
    c = cfg(nx=nx, ny=ny, nz=nz, nghost=g, case_id=12)
    M = MetricArrays(nx, ny)
    q = fortran_state(nx, ny, nz, g, -np.finfo(float).max)
    fill_interior(q, nx, ny, nz, g)
    assert B.lib().orc_set_boundary(C.byref(c), C.byref(M.m), _p(q)) == 0
    for k in range(1, nz + 1):
        ks = (k - 1 + nz // 2) % nz + 1
        for gg in range(1, g + 1):
            exp = at(q, g, 1, gg, ks).copy()
            exp[3] = -exp[3]
            assert np.array_equal(at(q, g, 1, 1 - gg, k), exp)
            exp = at(q, g, 1, ny + 1 - gg, ks).copy()
            exp[3] = -exp[3]
            assert np.array_equal(at(q, g, 1, ny + gg, k), exp)
    for gg in range(1, g + 1):
        assert np.array_equal(at(q, g, 1, 2, 1 - gg), at(q, g, 1, 2, nz + 1 - gg))
        assert np.array_equal(at(q, g, 1, 2, nz + gg), at(q, g, 1, 2, gg))


def test_polar_boundaries_sagittal():
    """test_polar_boundaries.f90:97-107, 164-181: reflecting poles of the sagittal case."""
    nx, ny, nz, g = 3, 4, 1, 2
    c = cfg(nx=nx, ny=ny, nz=nz, nghost=g, case_id=11)
    M = MetricArrays(nx, ny)
    q = fortran_state(nx, ny, nz, g, -np.finfo(float).max)
    fill_interior(q, nx, ny, nz, g)
    assert B.lib().orc_set_boundary(C.byref(c), C.byref(M.m), _p(q)) == 0
    for gg in range(1, g + 1):
        exp = at(q, g, 1, gg, 1).copy()
        exp[3] = -exp[3]
        assert np.array_equal(at(q, g, 1, 1 - gg, 1), exp)
        exp = at(q, g, 1, ny + 1 - gg, 1).copy()
        exp[3] = -exp[3]
        assert np.array_equal(at(q, g, 1, ny + gg, 1), exp)


def test_shift_aware_outflow():
    """test_case_corrections.f90:266-294: v^x clamped to beta/alpha = 0.25 on both sides."""
    nx, ny, nz, g = 2, 1, 1, 1
    c = cfg(nx=nx, ny=ny, nz=nz, nghost=g, case_id=9, metric=1, geom=2)
    M = MetricArrays(nx, ny, lapse=0.8, shift=(0.2, 0, 0))
    q = fortran_state(nx, ny, nz, g, 0.0)
    q[..., 0] = 1.0
    q[..., 1] = 1.0
    q[g + 1, g + 1, g + 1, 2] = 0.40
    q[g + 1, g + 1, g + 2, 2] = 0.00
    assert B.lib().orc_set_boundary(C.byref(c), C.byref(M.m), _p(q)) == 0
    assert abs(at(q, g, 0, 1, 1)[2] - 0.25) <= 2e-13
    assert abs(at(q, g, nx + 1, 1, 1)[2] - 0.25) <= 2e-13


def test_dust_boundaries():
    """test_case_corrections.f90:234-261: inner outflow clip, analytic outer injection,
    transverse periodicity (outer states from the host problem setup)."""
    nx, ny, nz, g = 3, 2, 2, 2
    c = cfg(nx=nx, ny=ny, nz=nz, nghost=g, case_id=8, metric=1, geom=2)
    M = MetricArrays(nx, ny)
    outer = np.arange(1, 11, dtype=float).reshape(2, 5) * 1e-3
    M.dust = outer.reshape(-1).copy()
    M.m.dust_outer = _p(M.dust)
    q = fortran_state(nx, ny, nz, g, -np.finfo(float).max)
    q[g + 1:g + 1 + nz, g + 1:g + 1 + ny, g + 1:g + 1 + nx, :] = 0.0
    q[g + 1:g + 1 + nz, g + 1:g + 1 + ny, g + 1:g + 1 + nx, 0] = 0.2
    q[g + 1:g + 1 + nz, g + 1:g + 1 + ny, g + 1:g + 1 + nx, 1] = 0.3
    q[g + 1:g + 1 + nz, g + 1:g + 1 + ny, g + 1:g + 1 + nx, 2] = 0.1
    assert B.lib().orc_set_boundary(C.byref(c), C.byref(M.m), _p(q)) == 0
    assert at(q, g, 0, 1, 1)[2] == 0.0
    assert at(q, g, 0, 1, 1)[0] == at(q, g, 1, 1, 1)[0]
    assert np.array_equal(at(q, g, nx + 1, 1, 1), outer[0])
    assert np.array_equal(at(q, g, 2, 0, 1), at(q, g, 2, ny, 1))


def test_weno3_exp_accuracy():
    """The exp shared by the oracle and the kernels (Cody-Waite + Taylor) stays within
    one ulp of the C library's exp over the WENO3 argument range and beyond."""
    L = B.lib()
    xs = np.concatenate([np.linspace(-10.0, 0.0, 20001), np.linspace(-700.0, 700.0, 20001),
                         np.random.default_rng(3).uniform(-12, 1, 20000)])
    for x in xs:
        a, b = L.orc_exp(float(x)), float(np.exp(x))
        assert abs(a - b) <= np.spacing(b), (x, a, b)
    assert L.orc_exp(0.0) == 1.0


# ---- tests/test_gw_geometry.f90, tests/test_gw_stress.f90 (calc_gw_strain's pieces) ----
def _gw(r, th, ph, spin, alpha, beta, v, log_r):
    pos, vel, jac = np.zeros(3), np.zeros(3), C.c_double()
    B.lib().orc_gw_kinematics(r, th, ph, spin, alpha, _p(np.asarray(beta, dtype=float)),
                              _p(np.asarray(v, dtype=float)), int(log_r), _p(pos), _p(vel), C.byref(jac))
    return pos, vel, jac.value


def _ks_position(r, th, ph, spin):
    pos = np.zeros(3)
    B.lib().orc_ks_spheroidal_position(r, th, ph, spin, _p(pos))
    return pos


def test_gw_horizon_radius():
    """test_gw_geometry.f90:17-22: Schwarzschild, Kerr a = 0.9 and extremal horizons."""
    L, r = B.lib(), C.c_double()
    for spin, want in [(0.0, 2.0), (0.9, 1.0 + math.sqrt(0.19)), (1.0, 1.0)]:
        assert L.orc_horizon_radius(1.0, spin, C.byref(r)) == 0
        assert abs(r.value - want) <= 1e-14
    assert L.orc_horizon_radius(1.0, 1.1, C.byref(r)) == -1  # beyond extremal: undefined


def test_gw_cartesian_kinematics():
    """test_gw_geometry.f90:24-104: a fluid at rest with the shift has no transport
    velocity; the logarithmic grid's components give the same position and velocity; the
    position equals the spheroidal VTK map; the flat Jacobian; the velocity is the chain
    rule of the position (central differences, 2e-9); a = 0 is the spherical map; the
    poles collapse exactly onto the axis."""
    r, th, ph, spin, alpha = 7.0, 1.1, 0.7, 0.8, 0.8
    beta = np.array([0.04, -0.02, 0.01])
    _, vel, _ = _gw(r, th, ph, spin, alpha, beta, beta / alpha, False)
    assert np.max(np.abs(vel)) <= 1e-14
    v = np.array([0.03, -0.04, 0.05])
    pos, vel, _ = _gw(r, th, ph, spin, alpha, beta, v, False)
    bl, vl = beta.copy(), v.copy()
    bl[0] /= r
    vl[0] /= r
    pos_l, vel_l, _ = _gw(r, th, ph, spin, alpha, bl, vl, True)
    assert np.max(np.abs(pos_l - pos)) <= 1e-14
    assert np.max(np.abs(vel_l - vel)) <= 1e-14

    r, rates = 4.3, np.array([0.12, -0.03, 0.21])
    zero = np.zeros(3)
    pos, vel, jac = _gw(r, th, ph, spin, 1.0, zero, rates, False)
    assert np.max(np.abs(_ks_position(r, th, ph, spin) - pos)) <= 1e-14
    assert abs(jac - (r ** 2 + spin ** 2 * math.cos(th) ** 2) * math.sin(th)) <= 1e-13
    eps = 1e-6
    pp = _gw(r + eps * rates[0], th + eps * rates[1], ph + eps * rates[2], spin, 1.0, zero, zero, False)[0]
    pm = _gw(r - eps * rates[0], th - eps * rates[1], ph - eps * rates[2], spin, 1.0, zero, zero, False)[0]
    assert np.max(np.abs(vel - (pp - pm) / (2.0 * eps))) <= 2e-9
    pos, _, jac = _gw(r, th, ph, 0.0, 1.0, zero, zero, False)
    sph = [r * math.sin(th) * math.cos(ph), r * math.sin(th) * math.sin(ph), r * math.cos(th)]
    assert np.max(np.abs(pos - sph)) <= 1e-13
    assert abs(jac - r ** 2 * math.sin(th)) <= 1e-13
    assert np.array_equal(_ks_position(r, 0.0, ph, spin), [0.0, 0.0, r])
    assert np.array_equal(_ks_position(r, math.acos(-1.0), ph, spin), [0.0, 0.0, -r])


def test_finn_evans_circular_orbit():
    """test_gw_stress.f90: a point mass on a circular Keplerian orbit has the analytic
    second derivative of its trace-free quadrupole (1e-13)."""
    M, m, R, phase = 1.0, 0.2, 5.0, 0.37
    om = math.sqrt(M / R ** 3)
    pos = np.array([R * math.cos(phase), R * math.sin(phase), 0.0])
    vel = np.array([-R * om * math.sin(phase), R * om * math.cos(phase), 0.0])
    ixx, iyy, ixy = C.c_double(), C.c_double(), C.c_double()
    B.lib().orc_finn_evans_stress(m, 0.0, M / R ** 3, _p(pos), _p(vel), 1.0, C.byref(ixx), C.byref(iyy),
                                  C.byref(ixy))
    amp = 2.0 * m * R ** 2 * om ** 2
    assert abs(ixx.value - (-amp * math.cos(2 * phase))) <= 1e-13
    assert abs(iyy.value - (amp * math.cos(2 * phase))) <= 1e-13
    assert abs(ixy.value - (-amp * math.sin(2 * phase))) <= 1e-13
