"""The reference's known-answer tests of the initial data and metrics, against the host
set-up (grhd_b200/csrc/host/problem.cpp, include/grhd2_host.h).

The host set-up builds the metric tables and the initial state that both the oracle and
the GPU path start from, so an error there would be common to both and pass every parity
test; these tests pin it to the reference's own checks:

* tests/test_fm_initial.f90:29-89 -- Fishbone-Moncrief tori in Eddington-Finkelstein
  (a = 0, r_in 6, r_max 12, K 0.015) and Kerr-Schild (a = 0.9, r_in 6.25, r_max 9.25,
  K 0.0015): the centre belongs to the torus with finite, positive thermodynamics and the
  constant specific angular momentum l (2e-12), the pressure maximum sits at r_max, the
  state is symmetric about the equator (2e-12), points inside r_in and sub-floor cells are
  the exact floor atmosphere at rest;
* tests/test_minkowski_spherical.f90:19-87 -- Minkowski in physical and logarithmic
  spherical coordinates has its closed forms (2e-13), Eddington-Finkelstein at M = 0 is
  the same metric (2e-13), and the Riemann tensor of both charts vanishes to 2e-8 by
  central differences of the Christoffel symbols.
"""
import ctypes as C
import math

import numpy as np
import pytest

from grhd_b200 import native as N

MINK, EF, KS = 0, 1, 2
CART, CYL, SPH, SPHEROID = 0, 1, 2, 3
NEQ = 5
EQ_DE, EQ_PR = 0, 1


def _p(a):
    return a.ctypes.data_as(C.POINTER(C.c_double))


def metric_at(kind, geom, log_r, mass, spin, ny, x, y):
    """(alpha, beta(3), gamma(3,3), gmunu(4,4), det, dlnalpha(4), chris[l,m,n], dg[m,n,d-1])
    with Fortran index meaning: chris[l, m, n] = Gamma^l_{mn}, dg[m, n, d-1] = d_d g_{mn}."""
    a, det = C.c_double(), C.c_double()
    beta, gamma, gmunu = np.zeros(3), np.zeros(9), np.zeros(16)
    dlna, ch, dg = np.zeros(4), np.zeros(64), np.zeros(48)
    rc = N.host_lib().grhd2_host_metric_at(kind, geom, int(log_r), mass, spin, ny, x, y, C.byref(a), _p(beta),
                                           _p(gamma), _p(gmunu), C.byref(det), _p(dlna), _p(ch), _p(dg))
    assert rc == 0
    # column-major (Fortran) arrays -> [first, second, ...] index order
    return (a.value, beta, gamma.reshape(3, 3).T, gmunu.reshape(4, 4).T, det.value, dlna,
            ch.reshape(4, 4, 4).transpose(2, 1, 0), dg.reshape(3, 4, 4).transpose(2, 1, 0))


# ---- tests/test_minkowski_spherical.f90 ------------------------------------------------
TOL = 2.0e-13
CURV_TOL = 2.0e-8
R, TH = 3.7, 0.91


def close(value, expected, tol=TOL):
    value, expected = np.asarray(value, dtype=float), np.asarray(expected, dtype=float)
    return np.max(np.abs(value - expected)) <= tol * max(1.0, np.max(np.abs(expected)))


def physical_form(r, th):
    s, c = math.sin(th), math.cos(th)
    g3 = np.zeros((3, 3)); g3[0, 0] = 1.0; g3[1, 1] = r ** 2; g3[2, 2] = r ** 2 * s ** 2
    g4 = np.zeros((4, 4)); g4[0, 0] = -1.0; g4[1, 1] = 1.0; g4[2, 2] = 1.0 / r ** 2; g4[3, 3] = 1.0 / (r ** 2 * s ** 2)
    ch = np.zeros((4, 4, 4))
    ch[1, 2, 2] = -r; ch[1, 3, 3] = -r * s ** 2
    ch[2, 1, 2] = ch[2, 2, 1] = 1.0 / r; ch[2, 3, 3] = -s * c
    ch[3, 1, 3] = ch[3, 3, 1] = 1.0 / r; ch[3, 2, 3] = ch[3, 3, 2] = c / s
    dg = np.zeros((4, 4, 3))
    dg[2, 2, 0] = 2.0 * r; dg[3, 3, 0] = 2.0 * r * s ** 2; dg[3, 3, 1] = 2.0 * r ** 2 * s * c
    return g3, g4, r ** 4 * s ** 2, ch, dg


def log_form(r, th):
    s, c = math.sin(th), math.cos(th)
    g3 = np.zeros((3, 3)); g3[0, 0] = r ** 2; g3[1, 1] = r ** 2; g3[2, 2] = r ** 2 * s ** 2
    g4 = np.zeros((4, 4)); g4[0, 0] = -1.0; g4[1, 1] = 1.0 / r ** 2; g4[2, 2] = 1.0 / r ** 2
    g4[3, 3] = 1.0 / (r ** 2 * s ** 2)
    ch = np.zeros((4, 4, 4))
    ch[1, 1, 1] = 1.0; ch[1, 2, 2] = -1.0; ch[1, 3, 3] = -s ** 2
    ch[2, 1, 2] = ch[2, 2, 1] = 1.0; ch[2, 3, 3] = -s * c
    ch[3, 1, 3] = ch[3, 3, 1] = 1.0; ch[3, 2, 3] = ch[3, 3, 2] = c / s
    dg = np.zeros((4, 4, 3))
    dg[1, 1, 0] = 2.0 * r ** 2; dg[2, 2, 0] = 2.0 * r ** 2; dg[3, 3, 0] = 2.0 * r ** 2 * s ** 2
    dg[3, 3, 1] = 2.0 * r ** 2 * s * c
    return g3, g4, r ** 6 * s ** 2, ch, dg


def max_riemann(kind, log_r, x1, x2, mass=0.0):
    """max |R^rho_{sigma mu nu}| from central differences (step 1e-5) of the Christoffel
    symbols in x1 and x2 (check_flat_riemann, test_minkowski_spherical.f90:204-241)."""
    eps = 1.0e-5
    ch = lambda a, b: metric_at(kind, SPH, log_r, mass, 0.0, 8, a, b)[6]
    c0 = ch(x1, x2)
    dc = np.zeros((4, 4, 4, 4))  # dc[l, m, n, d] = d_d Gamma^l_{mn}
    dc[..., 1] = (ch(x1 + eps, x2) - ch(x1 - eps, x2)) / (2.0 * eps)
    dc[..., 2] = (ch(x1, x2 + eps) - ch(x1, x2 - eps)) / (2.0 * eps)
    worst = 0.0
    for rho in range(4):
        for sig in range(4):
            for mu in range(4):
                for nu in range(4):
                    v = dc[rho, nu, sig, mu] - dc[rho, mu, sig, nu]
                    for lam in range(4):
                        v += c0[rho, mu, lam] * c0[lam, nu, sig] - c0[rho, nu, lam] * c0[lam, mu, sig]
                    worst = max(worst, abs(v))
    return worst


@pytest.mark.parametrize("log_r", [False, True])
def test_minkowski_spherical_closed_forms(log_r):
    x = math.log(R) if log_r else R
    alpha, beta, g3, g4, det, dlna, ch, dg = metric_at(MINK, SPH, log_r, 0.0, 0.0, 8, x, TH)
    e3, e4, edet, ech, edg = (log_form if log_r else physical_form)(R, TH)
    assert close(alpha, 1.0) and close(beta, np.zeros(3)) and close(dlna, np.zeros(4))
    assert close(g3, e3), "spatial metric"
    assert close(g4, e4), "inverse metric"
    assert close(det, edet), "determinant"
    assert close(ch, ech), "Christoffel symbols"
    assert close(dg, edg), "metric derivatives"
    assert max_riemann(MINK, log_r, x, TH) <= CURV_TOL


@pytest.mark.parametrize("log_r", [False, True])
def test_eddington_finkelstein_at_zero_mass_is_minkowski(log_r):
    x = math.log(R) if log_r else R
    mink = metric_at(MINK, SPH, log_r, 0.0, 0.0, 8, x, TH)
    ef = metric_at(EF, SPH, log_r, 0.0, 0.0, 8, x, TH)
    for name, a, b in zip(("lapse", "shift", "spatial metric", "inverse metric", "determinant",
                           "lapse derivative", "Christoffel", "metric derivatives"), ef, mink):
        assert close(a, b), f"M=0 EF {name}"
    assert max_riemann(EF, log_r, x, TH) <= CURV_TOL


# ---- tests/test_fm_initial.f90 ---------------------------------------------------------
ADB = 4.0 / 3.0
RHO_FLOOR, P_FLOOR = 1.0e-10, 1.0e-13


def fm_prepare(kind, geom, spin, r_in, r_c):
    l, w, ok = C.c_double(), C.c_double(), C.c_int32()
    assert N.host_lib().grhd2_host_fm_prepare(kind, geom, 0, 1.0, spin, r_in, r_c, C.byref(l), C.byref(w),
                                              C.byref(ok)) == 0
    return l.value, w.value, bool(ok.value)


def fm_state(kind, geom, spin, r, th, r_in, K, l, w):
    st = np.zeros(NEQ)
    inside = C.c_int32()
    assert N.host_lib().grhd2_host_fm_state(kind, geom, 0, 1.0, spin, ADB, RHO_FLOOR, P_FLOOR, r, th, r_in, K, l, w,
                                            _p(st), C.byref(inside)) == 0
    return st, bool(inside.value)


FM_MODELS = [("Eddington-Finkelstein", EF, SPH, 0.0, 6.0, 12.0, 0.015),
             ("Kerr-Schild", KS, SPHEROID, 0.9, 6.25, 9.25, 0.0015)]


@pytest.mark.parametrize("label,kind,geom,spin,r_in,r_c,K", FM_MODELS)
def test_fishbone_moncrief_initial_data(label, kind, geom, spin, r_in, r_c, K):
    l_ang, w_in, ok = fm_prepare(kind, geom, spin, r_in, r_c)
    assert ok, f"{label} preparation"
    half_pi = math.pi / 2.0
    centre, inside = fm_state(kind, geom, spin, r_c, half_pi, r_in, K, l_ang, w_in)
    assert inside, "centre belongs to torus"
    assert np.all(np.isfinite(centre)), "centre is finite"
    assert centre[EQ_DE] > RHO_FLOOR and centre[EQ_PR] > P_FLOOR, "positive thermodynamics"

    # constant specific angular momentum -u_phi / u_t (check_specific_angular_momentum)
    alpha, beta, g, *_ = metric_at(kind, geom, False, 1.0, spin, 1, r_c, half_pi)
    v = centre[2:5]
    W = 1.0 / math.sqrt(1.0 - v @ g @ v)
    shift_cov = g @ beta
    g_tt = -alpha ** 2 + beta @ shift_cov
    u0 = W / alpha
    ui = W * (v - beta / alpha)
    u_t = g_tt * u0 + shift_cov @ ui
    u_phi = shift_cov[2] * u0 + g[2, :] @ ui
    actual = -u_phi / u_t
    assert abs(actual - l_ang) <= 2.0e-12 * max(1.0, abs(l_ang)), f"constant angular momentum {actual} vs {l_ang}"

    # sub-floor cells are the exact floor atmosphere at rest (check_atmosphere_projection)
    h_c = 1.0 + K * ADB / (ADB - 1.0) * centre[EQ_DE] ** (ADB - 1.0)
    for target in (0.5 * RHO_FLOOR, 10.0 * RHO_FLOOR):
        p_t = K * target ** ADB
        assert target < RHO_FLOOR or p_t < P_FLOOR, "projection test setup"
        h_t = 1.0 + K * ADB / (ADB - 1.0) * target ** (ADB - 1.0)
        w_proj = w_in - math.log(h_c) + math.log(h_t)
        st, inside = fm_state(kind, geom, spin, r_c, half_pi, r_in, K, l_ang, w_proj)
        assert not inside, "subfloor cell is atmosphere"
        assert st[EQ_DE] == RHO_FLOOR and st[EQ_PR] == P_FLOOR, "subfloor cell uses exact floors"
        assert np.all(st[2:5] == 0.0), "subfloor atmosphere has zero velocity"

    # the pressure maximum at r_max
    off = 1.0e-3 * r_c
    left, in_l = fm_state(kind, geom, spin, r_c - off, half_pi, r_in, K, l_ang, w_in)
    right, in_r = fm_state(kind, geom, spin, r_c + off, half_pi, r_in, K, l_ang, w_in)
    assert in_l and in_r, "neighbours belong to torus"
    assert centre[EQ_PR] >= left[EQ_PR] and centre[EQ_PR] >= right[EQ_PR], "pressure maximum radius"

    # equatorial symmetry
    north, in_n = fm_state(kind, geom, spin, r_c, half_pi - 0.2, r_in, K, l_ang, w_in)
    south, in_s = fm_state(kind, geom, spin, r_c, half_pi + 0.2, r_in, K, l_ang, w_in)
    assert in_n and in_s, "north and south points belong to torus"
    assert np.all(np.isfinite(north))
    assert np.max(np.abs(north - south)) <= 2.0e-12 * max(1.0, np.max(np.abs(south))), "equatorial symmetry"

    # inside r_in: the exact floors
    atm, inside = fm_state(kind, geom, spin, 0.9 * r_in, half_pi, r_in, K, l_ang, w_in)
    assert not inside, "inner atmosphere classification"
    assert atm[EQ_DE] == RHO_FLOOR and atm[EQ_PR] == P_FLOOR, "inner atmosphere floors"


def test_torus_initial_data_uses_the_prepared_state():
    """The 2.5D torus preset's initial primitives at a torus cell equal the state evaluated
    at that cell's centre with the problem's own l and W_in (the set-up path that feeds the
    oracle and the GPU is the one pinned above)."""
    from tests.helpers import torus_2p5d
    pb = torus_2p5d(nx=64, nz=8)
    info = pb.info
    p = pb.initial_prims()
    g = pb.ng
    x = pb.coords()[0]
    rho = p[g + 1, g + 1, g + 1:g + 1 + pb.nx, EQ_DE]
    i = int(np.argmax(rho))
    l2, w2, ok = fm_prepare(KS, SPHEROID, info.a_spin, 6.0, 12.0)
    st_r = math.exp(x[g + 1 + i])
    # the problem's constants, evaluated through the log-r chart the grid uses
    l_p, w_p = info.fm_l, info.fm_w_in
    assert ok and l2 == l_p
    st = np.zeros(NEQ)
    inside = C.c_int32()
    assert N.host_lib().grhd2_host_fm_state(KS, SPHEROID, 1, 1.0, info.a_spin, ADB, RHO_FLOOR, P_FLOOR, st_r,
                                            pb.coords()[1][g + 1], 6.0, 0.0015, l_p, w_p, _p(st),
                                            C.byref(inside)) == 0
    assert inside
    assert np.allclose(st, p[g + 1, g + 1, g + 1 + i, :], rtol=1e-12, atol=0.0)
