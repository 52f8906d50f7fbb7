"""A second, independent reading of the reference's HLLC face flux against the oracle's.

calc_hllc_fluxes (fluxes.f90:174-397) with build_face_orthonormal_frame (:402-473),
metric_dot, primitives_to_local_frame, calc_srhd_local_state,
conservative_state_is_admissible and local_flux_to_coordinate (:474-624), restated in plain
Python from the Fortran -- every fallback to HLLE included -- and compared bit for bit
(flux and fallback counter) with the oracle's on random states and face metrics.  The
reference's eleven HLLC known-answer tests pin particular states; this covers the rest.
"""
import ctypes as C
import math
import sys

import numpy as np
import pytest

from oracle import binding as B
from tests.test_oracle_hlle import ADB, G1, V_MAX, _state, fmax, fmin, hlle

DE, PR, VX = 0, 1, 2
TINY = sys.float_info.min
EPS = sys.float_info.epsilon


def finite(*xs):
    return all(math.isfinite(x) for x in xs)


def metric_dot(a, b, g):
    s = 0.0
    for i in range(3):
        for j in range(3):
            s = s + g[i][j] * a[i] * b[j]
    return s


def face_frame(g, d):
    """(frame[j][a] = frame(j+1, a+1), coframe[a][i], gamma^dd, ok)"""
    frame = [[0.0] * 3 for _ in range(3)]
    cof = [[0.0] * 3 for _ in range(3)]
    if not finite(*[x for row in g for x in row]):
        return frame, cof, 0.0, False
    det = (g[0][0] * (g[1][1] * g[2][2] - g[1][2] * g[2][1])
           - g[0][1] * (g[1][0] * g[2][2] - g[1][2] * g[2][0])
           + g[0][2] * (g[1][0] * g[2][1] - g[1][1] * g[2][0]))
    if not finite(det) or det <= 1.0e-30:
        return frame, cof, 0.0, False
    gi = [[(g[1][1] * g[2][2] - g[1][2] * g[2][1]) / det, (g[0][2] * g[2][1] - g[0][1] * g[2][2]) / det,
           (g[0][1] * g[1][2] - g[0][2] * g[1][1]) / det],
          [(g[1][2] * g[2][0] - g[1][0] * g[2][2]) / det, (g[0][0] * g[2][2] - g[0][2] * g[2][0]) / det,
           (g[0][2] * g[1][0] - g[0][0] * g[1][2]) / det],
          [(g[1][0] * g[2][1] - g[1][1] * g[2][0]) / det, (g[0][1] * g[2][0] - g[0][0] * g[2][1]) / det,
           (g[0][0] * g[1][1] - g[0][1] * g[1][0]) / det]]
    if not finite(*[x for row in gi for x in row]):
        return frame, cof, 0.0, False
    gup = gi[d][d]
    if gup <= 1.0e-30 or not finite(gup):
        return frame, cof, gup, False
    for i in range(3):
        frame[i][0] = gi[i][d] / math.sqrt(gup)
    tangents = {0: (1, 2), 1: (2, 0), 2: (0, 1)}[d]
    for b in (1, 2):
        seed = [0.0, 0.0, 0.0]
        seed[tangents[b - 1]] = 1.0
        for a in range(b):
            col = [frame[j][a] for j in range(3)]
            proj = metric_dot(seed, col, g)
            seed = [seed[j] - proj * col[j] for j in range(3)]
        nsq = metric_dot(seed, seed, g)
        if not finite(nsq) or nsq <= 1.0e-28:
            return frame, cof, gup, False
        for j in range(3):
            frame[j][b] = seed[j] / math.sqrt(nsq)
    for a in range(3):
        for i in range(3):
            for j in range(3):
                cof[a][i] = cof[a][i] + g[i][j] * frame[j][a]
    if not finite(*[x for row in frame for x in row], *[x for row in cof for x in row]):
        return frame, cof, gup, False
    return frame, cof, gup, True


def to_local(prim, cof):
    out = list(prim)
    for a in range(3):
        out[VX + a] = 0.0
        for i in range(3):
            out[VX + a] = out[VX + a] + cof[a][i] * prim[VX + i]
    return out


def srhd_local_state(p):
    """(cons, flux, wave_min, wave_max, ok) in the face's orthonormal frame"""
    rho, pres, vel = p[DE], p[PR], p[VX:VX + 3]
    bad = ([0.0] * 5, [0.0] * 5, 0.0, 0.0, False)
    if not finite(rho, pres, *vel) or rho <= 0.0 or pres < 0.0:
        return bad
    v_sq = vel[0] * vel[0] + vel[1] * vel[1] + vel[2] * vel[2]
    if not finite(v_sq) or v_sq < 0.0 or v_sq >= V_MAX:
        return bad
    h = 1.0 + G1 * pres / rho
    if not finite(h) or h <= 0.0:
        return bad
    cs_sq = ADB * pres / (rho * h)
    if not finite(cs_sq) or cs_sq < 0.0 or cs_sq >= 1.0:
        return bad
    W = 1.0 / math.sqrt(1.0 - v_sq)
    D = rho * W
    tau = rho * h * (W * W) - pres - D
    mom = [rho * h * (W * W) * v for v in vel]
    u = [D, tau, *mom]
    f = [D * vel[0], mom[0] - D * vel[0], mom[0] * vel[0] + pres, mom[1] * vel[0], mom[2] * vel[0]]
    denom = 1.0 - v_sq * cs_sq
    rad = (1.0 - v_sq) * (1.0 - v_sq * cs_sq - (vel[0] * vel[0]) * (1.0 - cs_sq))
    if denom <= 1.0e-14 or rad < -1.0e-12:
        return bad
    ac = math.sqrt(cs_sq) * math.sqrt(fmax(0.0, rad))
    wmin = (vel[0] * (1.0 - cs_sq) - ac) / denom
    wmax = (vel[0] * (1.0 - cs_sq) + ac) / denom
    if not finite(*u, *f, wmin, wmax):
        return bad
    return u, f, wmin, wmax, True


def admissible(u):
    if not finite(*u) or u[DE] <= 0.0:
        return False
    E = u[PR] + u[DE]
    msq = u[VX] * u[VX] + u[VX + 1] * u[VX + 1] + u[VX + 2] * u[VX + 2]
    scale = fmax(fmax(TINY, E * E), u[DE] * u[DE] + msq)
    if E <= 0.0:
        return False
    return not (E * E - u[DE] * u[DE] - msq <= 1.0e-13 * scale)


def to_coordinate(u, f, fs, alpha, sqg, gup, cof):
    moving = [f[n] - fs * u[n] for n in range(5)]
    factor = sqg * alpha * math.sqrt(gup)
    if not finite(factor, *moving):
        return None
    out = [factor * moving[DE], factor * moving[PR], 0.0, 0.0, 0.0]
    for i in range(3):
        for a in range(3):
            out[VX + i] = out[VX + i] + factor * cof[a][i] * moving[VX + a]
    return out if finite(*out) else None


def hllc(qL, qR, d, alpha, beta, g, sqg):
    """(flux, fell back to HLLE)"""
    fallback = lambda: (hlle(qL, qR, d, alpha, beta, g, sqg, False), True)
    if alpha <= 0.0 or sqg <= 0.0 or not finite(alpha, sqg):
        return fallback()
    frame, cof, gup, ok = face_frame(g, d)
    if not ok:
        return fallback()
    qLh, qRh = to_local(qL, cof), to_local(qR, cof)
    uL, fL, lLmin, lLmax, ok = srhd_local_state(qLh)
    if not ok:
        return fallback()
    uR, fR, lRmin, lRmax, ok = srhd_local_state(qRh)
    if not ok:
        return fallback()
    ll, lr = fmin(lLmin, lRmin), fmax(lLmax, lRmax)
    fs = beta[d] / (alpha * math.sqrt(gup))
    if not finite(fs) or lr - ll <= 1.0e-13:
        return fallback()
    if fs <= ll or fs >= lr:
        out = to_coordinate(uL if fs <= ll else uR, fL if fs <= ll else fR, fs, alpha, sqg, gup, cof)
        return (out, False) if out is not None else fallback()
    den = lr - ll
    u_hll = [(lr * uR[n] - ll * uL[n] + fL[n] - fR[n]) / den for n in range(5)]
    f_hll = [(lr * fL[n] - ll * fR[n] + lr * ll * (uR[n] - uL[n])) / den for n in range(5)]
    if not finite(*u_hll, *f_hll):
        return fallback()
    E_hll, FE_hll = u_hll[PR] + u_hll[DE], f_hll[PR] + f_hll[DE]
    M_hll, FM_hll = u_hll[VX], f_hll[VX]
    A, Bq, Cq = FE_hll, -(E_hll + FM_hll), M_hll
    disc = Bq * Bq - 4.0 * A * Cq
    disc_scale = fmax(fmax(TINY, Bq * Bq), abs(4.0 * A * Cq))
    if not finite(disc) or disc < -1.0e-12 * disc_scale:
        return fallback()
    disc = fmax(0.0, disc)
    coef_scale = fmax(fmax(TINY, abs(Bq)), abs(Cq))
    quad = abs(A) > 1.0e-13 * coef_scale
    if not quad:
        if abs(Bq) <= 1.0e-14 * fmax(TINY, abs(Cq)):
            return fallback()
        ls = -Cq / Bq
    else:
        den = -Bq - math.sqrt(disc)
        if abs(den) > 1.0e-14 * fmax(fmax(TINY, abs(Bq)), math.sqrt(disc)):
            ls = den / (2.0 * A)
        else:
            den = -Bq + math.sqrt(disc)
            if abs(den) <= 1.0e-14 * fmax(fmax(TINY, abs(Bq)), math.sqrt(disc)):
                return fallback()
            ls = (2.0 * Cq) / den
    tol = 1.0e-10 * fmax(fmax(1.0, abs(ll)), abs(lr))
    valid = finite(ls) and ls >= ll - tol and ls <= lr + tol and abs(ls) <= 1.0 + tol
    if not valid and quad:
        alt = (-Bq + math.sqrt(disc)) / (2.0 * A)
        if finite(alt) and alt >= ll - tol and alt <= lr + tol and abs(alt) <= 1.0 + tol:
            ls, valid = alt, True
    if not valid:
        return fallback()
    ls = fmin(lr, fmax(ll, ls))
    A_l = ll * (uL[PR] + uL[DE]) - uL[VX]
    B_l = uL[VX] * (ll - qLh[VX]) - qLh[PR]
    A_r = lr * (uR[PR] + uR[DE]) - uR[VX]
    B_r = uR[VX] * (lr - qRh[VX]) - qRh[PR]
    den = 1.0 - ll * ls
    if abs(den) <= 1.0e-13:
        return fallback()
    ps_l = (A_l * ls - B_l) / den
    den = 1.0 - lr * ls
    if abs(den) <= 1.0e-13:
        return fallback()
    ps_r = (A_r * ls - B_r) / den
    state_scale = fmax(fmax(fmax(fmax(TINY, abs(uL[PR] + uL[DE])), abs(uR[PR] + uR[DE])), abs(uL[VX])), abs(uR[VX]))
    p_tol = (1.0e-8 * fmax(fmax(fmax(fmax(TINY, abs(qLh[PR])), abs(qRh[PR])), abs(ps_l)), abs(ps_r))
             + 1.0e2 * EPS * state_scale)
    if not finite(ps_l, ps_r) or abs(ps_l - ps_r) > p_tol:
        return fallback()
    ps = 0.5 * (ps_l + ps_r)
    if not finite(ps) or abs(ll - ls) <= 1.0e-13 or abs(lr - ls) <= 1.0e-13:
        return fallback()
    pv = [0.0, ls, 1.0, 0.0, 0.0]
    usL = [(ll * uL[n] - fL[n] + ps * pv[n]) / (ll - ls) for n in range(5)]
    usR = [(lr * uR[n] - fR[n] + ps * pv[n]) / (lr - ls) for n in range(5)]
    fsL = [fL[n] + ll * (usL[n] - uL[n]) for n in range(5)]
    fsR = [fR[n] + lr * (usR[n] - uR[n]) for n in range(5)]
    if not admissible(usL) or not admissible(usR) or not finite(*fsL, *fsR):
        return fallback()
    u_sel, f_sel = (usL, fsL) if fs <= ls else (usR, fsR)
    out = to_coordinate(u_sel, f_sel, fs, alpha, sqg, gup, cof)
    return (out, False) if out is not None else fallback()


@pytest.mark.parametrize("seed", [41, 42, 43])
def test_hllc_matches_an_independent_restatement(seed):
    rng = np.random.default_rng(seed)
    c = B.OrcConfig()
    c.nx, c.ny, c.nz, c.nghost = 4, 4, 4, 3
    c.rec_method, c.tvd_limiter, c.riemann, c.shock_sensor = 5, 3, 2, 0
    c.metric_kind, c.geom_kind, c.case_id = 2, 3, 10
    c.dx = c.dy = c.dz = 1.0
    c.adb_idx, c.g1, c.cfl = ADB, G1, 0.4
    c.rho_floor, c.p_floor, c.v_max = 1e-10, 1e-13, V_MAX
    dp = lambda a: a.ctypes.data_as(C.POINTER(C.c_double))
    fallbacks = 0
    for n in range(800):
        A = rng.normal(size=(3, 3)) * 0.3
        g = A @ A.T + np.eye(3) * rng.uniform(0.5, 3.0)
        alpha, beta = rng.uniform(0.2, 1.5), rng.normal(size=3) * rng.choice([0.0, 0.3, 1.5])
        sqg = math.sqrt(np.linalg.det(g))
        qL, qR = _state(rng, g), _state(rng, g)
        if n % 7 == 0:  # a contact: equal pressure and normal velocity
            qR = [qL[DE] * rng.uniform(0.1, 10.0), qL[PR], *qL[VX:]]
        elif n % 7 == 1:
            qR = list(qL)
        d = n % 3
        got = np.zeros(5)
        cnt = B.OrcCounters()
        gf = np.ascontiguousarray(g.T).reshape(-1)
        B.lib().orc_riemann(C.byref(c), dp(np.array(qL)), dp(np.array(qR)), d + 1, alpha,
                            dp(np.ascontiguousarray(beta)), dp(gf), sqg, dp(got), C.byref(cnt))
        want, fb = hllc(qL, qR, d, alpha, beta.tolist(), g.tolist(), sqg)
        assert got.tobytes() == np.array(want).tobytes(), (n, qL, qR, got, want)
        assert cnt.hllc_fallbacks == int(fb), (n, cnt.hllc_fallbacks, fb)
        fallbacks += fb
    assert 0 < fallbacks < 800
