"""A second, independent reading of the reference's HLLE face flux against the oracle's.

calc_hlle_fluxes (fluxes.f90:125-156) with calc_fluxes (equations.f90:434-502),
prim_to_cons_face (fluxes.f90:76-121) and both wavespeed routines (calc_wavespeeds_srhd
:669-720 for Minkowski Cartesian, calc_wavespeeds_grhd :724-803 otherwise, as
init_wavespeed_solver :43-49 selects) restated in plain Python from the Fortran, compared
bit for bit with the oracle's on random states (superluminal ones included: the velocity
cap of each routine) and random face metrics (lapse, shift, a general positive-definite
3-metric), every sweep direction.  The reference's HLLE known-answer tests cover uniform
states only; this covers the general case.
"""
import ctypes as C
import math

import numpy as np
import pytest

from oracle import binding as B

ADB, G1, V_MAX = 4.0 / 3.0, 4.0, 1.0 - 1.0e-5
DE, PR, VX = 0, 1, 2


def fmax(a, b):
    return b if (b > a or a != a) else a


def fmin(a, b):
    return b if (b < a or a != a) else a


def capped(prim, g):
    v = [prim[VX], prim[VX + 1], prim[VX + 2]]
    v_sq = 0.0
    for ii in range(3):
        for jj in range(3):
            v_sq = v_sq + g[ii][jj] * v[ii] * v[jj]
    if v_sq >= V_MAX:
        v = [v[0] * math.sqrt(V_MAX / v_sq), v[1] * math.sqrt(V_MAX / v_sq), v[2] * math.sqrt(V_MAX / v_sq)]
        v_sq = V_MAX
    return v, v_sq


def lower(g, v):
    out = [0.0, 0.0, 0.0]
    for ii in range(3):
        for jj in range(3):
            out[ii] = out[ii] + g[ii][jj] * v[jj]
    return out


def calc_fluxes(prim, d, alpha, beta, g, sqg):
    v, v_sq = capped(prim, g)
    v_cov = lower(g, v)
    vn, bn = v[d], beta[d]
    h = 1.0 + G1 * prim[PR] / prim[DE]
    W = 1.0 / math.sqrt(1.0 - v_sq)
    v_eff = alpha * vn - bn
    f = [0.0] * 5
    f[DE] = prim[DE] * W * v_eff
    f[PR] = prim[DE] * h * (W * W) * v_eff + prim[PR] * bn - f[DE]
    for a in range(3):
        f[VX + a] = prim[DE] * h * (W * W) * v_cov[a] * v_eff + (alpha * prim[PR] if d == a else 0.0)
    return [x * sqg for x in f]


def prim_to_cons_face(prim, g, sqg):
    v, v_sq = capped(prim, g)
    v_cov = lower(g, v)
    h = 1.0 + G1 * prim[PR] / prim[DE]
    W = 1.0 / math.sqrt(1.0 - v_sq)
    u = [0.0] * 5
    u[DE] = prim[DE] * W
    u[PR] = prim[DE] * h * (W * W) - prim[PR] - prim[DE] * W
    for a in range(3):
        u[VX + a] = prim[DE] * h * (W * W) * v_cov[a]
    return [x * sqg for x in u]


def wavespeeds_srhd(prim, d, g):
    v, v_sq = capped(prim, g)
    enth = 1.0 + G1 * prim[PR] / prim[DE]
    cs_sq = ADB * prim[PR] / (prim[DE] * enth)
    cs = math.sqrt(cs_sq)
    vn = v[d]
    term1 = 1.0 / (1.0 - v_sq * cs_sq)
    term2 = cs * math.sqrt((1.0 - v_sq) * (1.0 / term1 - (vn * vn) * (1.0 - cs_sq)))
    e1 = vn
    e2 = term1 * (vn * (1.0 - cs_sq) + term2)
    e3 = term1 * (vn * (1.0 - cs_sq) - term2)
    return fmin(fmin(fmin(0.0, e1), e2), e3), fmax(fmax(fmax(0.0, e1), e2), e3)


def wavespeeds_grhd(prim, d, alpha, beta, g):
    v, v_sq = capped(prim, g)
    enth = 1.0 + G1 * prim[PR] / prim[DE]
    cs_sq = ADB * prim[PR] / (prim[DE] * enth)
    cs = math.sqrt(cs_sq)
    det = (g[0][0] * (g[1][1] * g[2][2] - g[1][2] * g[2][1])
           - g[0][1] * (g[1][0] * g[2][2] - g[1][2] * g[2][0])
           + g[0][2] * (g[1][0] * g[2][1] - g[1][1] * g[2][0]))
    if d == 0:
        gup = (g[1][1] * g[2][2] - g[1][2] * g[2][1]) / det
    elif d == 1:
        gup = (g[0][0] * g[2][2] - g[0][2] * g[2][0]) / det
    else:
        gup = (g[0][0] * g[1][1] - g[0][1] * g[1][0]) / det
    vn, bn = v[d], beta[d]
    term1 = alpha / (1.0 - v_sq * cs_sq)
    term2 = cs * math.sqrt(fmax(0.0, (1.0 - v_sq) * (gup * (1.0 - v_sq * cs_sq) - (vn * vn) * (1.0 - cs_sq))))
    e1 = alpha * vn - bn
    e2 = term1 * (vn * (1.0 - cs_sq) + term2) - bn
    e3 = term1 * (vn * (1.0 - cs_sq) - term2) - bn
    return fmin(fmin(fmin(0.0, e1), e2), e3), fmax(fmax(fmax(0.0, e1), e2), e3)


def hlle(qL, qR, d, alpha, beta, g, sqg, flat):
    fL, fR = calc_fluxes(qL, d, alpha, beta, g, sqg), calc_fluxes(qR, d, alpha, beta, g, sqg)
    uL, uR = prim_to_cons_face(qL, g, sqg), prim_to_cons_face(qR, g, sqg)
    if flat:
        lLmin, lLmax = wavespeeds_srhd(qL, d, g)
        lRmin, lRmax = wavespeeds_srhd(qR, d, g)
    else:
        lLmin, lLmax = wavespeeds_grhd(qL, d, alpha, beta, g)
        lRmin, lRmax = wavespeeds_grhd(qR, d, alpha, beta, g)
    a_plus = fmax(fmax(0.0, lLmax), lRmax)
    a_minus = fmin(fmin(0.0, lLmin), lRmin)
    if abs(a_plus - a_minus) < 1.0e-14:
        return [0.0] * 5
    return [(a_plus * fL[n] - a_minus * fR[n] + a_plus * a_minus * (uR[n] - uL[n])) / (a_plus - a_minus)
            for n in range(5)]


def _cfg(flat):
    c = B.OrcConfig()
    c.nx, c.ny, c.nz, c.nghost = 4, 4, 4, 3
    c.rec_method, c.tvd_limiter, c.riemann, c.shock_sensor = 5, 3, 1, 0
    c.metric_kind, c.geom_kind, c.case_id = (0, 0, 1) if flat else (2, 3, 10)
    c.dx = c.dy = c.dz = 1.0
    c.adb_idx, c.g1, c.cfl = ADB, G1, 0.4
    c.rho_floor, c.p_floor, c.v_max = 1e-10, 1e-13, V_MAX
    return c


def _state(rng, g):
    d = rng.normal(size=3)
    d = d / math.sqrt(d @ g @ d)
    speed = rng.choice([0.0, rng.uniform(0, 0.9), rng.uniform(0.9, 0.99999), rng.uniform(1.0, 1.3)])
    return [10.0 ** rng.uniform(-6, 1), 10.0 ** rng.uniform(-8, 2), *(speed * d)]


@pytest.mark.parametrize("flat", [True, False])
def test_hlle_matches_an_independent_restatement(flat):
    rng = np.random.default_rng(31 + int(flat))
    c = _cfg(flat)
    dp = lambda a: a.ctypes.data_as(C.POINTER(C.c_double))
    for n in range(600):
        if flat:
            g, alpha, beta = np.eye(3), 1.0, np.zeros(3)
        else:
            A = rng.normal(size=(3, 3)) * 0.3
            g = A @ A.T + np.eye(3) * rng.uniform(0.5, 3.0)
            alpha, beta = rng.uniform(0.2, 1.5), rng.normal(size=3) * 0.3
        sqg = math.sqrt(np.linalg.det(g))
        qL, qR = _state(rng, g), _state(rng, g)
        if n % 10 == 0:
            qR = list(qL)  # a uniform state: the physical flux
        d = n % 3
        got = np.zeros(5)
        gf = np.ascontiguousarray(g.T).reshape(-1)  # Fortran order
        B.lib().orc_riemann(C.byref(c), dp(np.array(qL)), dp(np.array(qR)), d + 1, alpha,
                            dp(np.ascontiguousarray(beta)), dp(gf), sqg, dp(got), None)
        want = hlle(qL, qR, d, alpha, beta.tolist(), g.tolist(), sqg, flat)
        assert got.tobytes() == np.array(want).tobytes(), (n, qL, qR, got, want)
