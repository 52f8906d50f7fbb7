"""A second, independent reading of the reference's reconstruction against the oracle's.

The reference holds no known-answer test for its reconstruction, so the oracle's
restatement of reconstruct_1d_core (reconstruction.f90:285-657) and of the schemes it calls
(minmod_2/3/4 :28-45, weno3_interface :141-181, weno5_interface :187-215, mp5_interface
:222-254, tvd_slope :259-278) is checked here against a second restatement written in plain
Python directly from the Fortran, term by term in Fortran's evaluation order.  Python
floats are IEEE doubles with no fused multiply-add, as is the oracle's build, so the two
must agree to the bit: on random strips with smooth stretches, jumps large enough to move
the shock sensor through every branch, atmosphere cells, constant runs (exact zero slopes)
and both the Minkowski and the non-Minkowski overrides, in every sweep direction.  WENO3's
exp is the C library's in the oracle build that uses it (`lib(libm_exp=True)`), as it is in
Python's math.exp; the default build's exp is pinned separately (test_oracle_kats.py).
"""
import ctypes as C
import math

import numpy as np
import pytest

from oracle import binding as B

GODUNOV, TVD, WENO3, MP5, WENO5 = 1, 2, 3, 4, 5
MINMOD, SUPERBEE, MC = 1, 2, 3
DIR_X, DIR_Y, DIR_Z = 1, 2, 3
RHO_FLOOR, P_FLOOR = 1.0e-10, 1.0e-13
NEQ, DE, PR = 5, 0, 1


def sgn(a):
    return math.copysign(1.0, a)


def minmod_2(a, b):
    return 0.5 * (sgn(a) + sgn(b)) * min(abs(a), abs(b))


def minmod_3(a, b, c):
    return sgn(a) * max(0.0, min(abs(a), sgn(a) * b, sgn(a) * c))


def minmod_4(a, b, c, d):
    return (0.125 * (sgn(a) + sgn(b)) * abs(sgn(a) + sgn(c)) * abs(sgn(a) + sgn(d))
            * min(abs(a), abs(b), abs(c), abs(d)))


def tvd_slope(a, b, lim):
    if lim == SUPERBEE:
        if a * b <= 0.0:
            return 0.0
        return sgn(a) * max(min(2.0 * abs(a), abs(b)), min(abs(a), 2.0 * abs(b)))
    if lim == MC:
        return minmod_3(2.0 * b, 0.5 * (a + b), 2.0 * a)
    return minmod_2(a, b)


def weno3(qm1, q0, q1):
    eps_min, d0, d1 = 1.0e-14, 2.0 / 3.0, 1.0 / 3.0
    p0 = 0.5 * q0 + 0.5 * q1
    p1 = -0.5 * qm1 + 1.5 * q0
    beta_0 = (q0 - q1) * (q0 - q1)
    beta_1 = (qm1 - q0) * (qm1 - q0)
    sensor = abs(beta_0 - beta_1) / (max(beta_0, beta_1) + eps_min)
    eps_h = eps_min + (qm1 * qm1 + q0 * q0 + q1 * q1) * math.exp(-10.0 * sensor)
    t0, t1 = eps_h + beta_0, eps_h + beta_1
    a0 = d0 / (t0 * t0)
    a1 = d1 / (t1 * t1)
    w0 = a0 / (a0 + a1)
    w1 = a1 / (a0 + a1)
    return w0 * p0 + w1 * p1


def weno5(qm2, qm1, q0, q1, q2):
    eps, d0, d1, d2 = 1.0e-14, 0.3, 0.6, 0.1
    c = 13.0 / 12.0
    x, y = q0 - 2.0 * q1 + q2, 3.0 * q0 - 4.0 * q1 + q2
    b0 = c * (x * x) + 0.25 * (y * y)
    x, y = qm1 - 2.0 * q0 + q1, qm1 - q1
    b1 = c * (x * x) + 0.25 * (y * y)
    x, y = qm2 - 2.0 * qm1 + q0, qm2 - 4.0 * qm1 + 3.0 * q0
    b2 = c * (x * x) + 0.25 * (y * y)
    tau5 = abs(b0 - b2)
    a0 = d0 * (1.0 + (tau5 / (eps + b0)))
    a1 = d1 * (1.0 + (tau5 / (eps + b1)))
    a2 = d2 * (1.0 + (tau5 / (eps + b2)))
    w0 = a0 / (a0 + a1 + a2)
    w1 = a1 / (a0 + a1 + a2)
    w2 = a2 / (a0 + a1 + a2)
    p0 = (1.0 / 3.0) * q0 + (5.0 / 6.0) * q1 - (1.0 / 6.0) * q2
    p1 = -((1.0 / 6.0) * qm1) + (5.0 / 6.0) * q0 + (1.0 / 3.0) * q1
    p2 = (1.0 / 3.0) * qm2 - (7.0 / 6.0) * qm1 + (11.0 / 6.0) * q0
    return w0 * p0 + w1 * p1 + w2 * p2


def mp5(qm2, qm1, q0, q1, q2):
    alpha, eps = 4.0, 1.0e-10
    val_l = (2.0 * qm2 - 13.0 * qm1 + 47.0 * q0 + 27.0 * q1 - 3.0 * q2) / 60.0
    val_mp = q0 + minmod_2(q1 - q0, alpha * (q0 - qm1))
    if (val_l - q0) * (val_l - val_mp) < eps:
        return val_l
    d_jm1 = qm2 - 2.0 * qm1 + q0
    d_j = qm1 - 2.0 * q0 + q1
    d_jp1 = q0 - 2.0 * q1 + q2
    dm4_jph = minmod_4(4.0 * d_j - d_jp1, 4.0 * d_jp1 - d_j, d_j, d_jp1)
    dm4_jmh = minmod_4(4.0 * d_j - d_jm1, 4.0 * d_jm1 - d_j, d_j, d_jm1)
    val_ul = q0 + alpha * (q0 - qm1)
    val_av = 0.5 * (q0 + q1)
    val_md = val_av - 0.5 * dm4_jph
    val_lc = q0 + 0.5 * (q0 - qm1) + 4.0 * dm4_jmh / 3.0
    val_min = max(min(q0, q1, val_md), min(q0, val_ul, val_lc))
    val_max = min(max(q0, q1, val_md), max(q0, val_ul, val_lc))
    return val_l + minmod_2(val_min - val_l, val_max - val_l)


def reconstruct(prim, nodes, rec, lim, sensor, nonmink, sweep):
    """reconstruct_1d_core on prim[i + g] = prim_1d(:, i), i = -g..nodes+g: (q_L, q_R)."""
    g = (len(prim) - nodes - 1) // 2
    P = lambda k, i: prim[i + g][k]
    qL = [[0.0] * NEQ for _ in range(nodes + 1)]
    qR = [[0.0] * NEQ for _ in range(nodes + 1)]
    atm = 1.0e2 * RHO_FLOOR
    for i in range(nodes + 1):
        p_jump = rho_jump = 0.0
        if rec != GODUNOV and sensor:
            pw = [P(PR, i + m) for m in range(-2, 3)]
            rw = [P(DE, i + m) for m in range(-2, 3)]
            p_max, p_min, r_max, r_min = max(pw), min(pw), max(rw), min(rw)
            p_jump = (p_max - p_min) / max(p_min, P_FLOOR) if p_max > 1.0e3 * P_FLOOR else 0.0
            rho_jump = (r_max - r_min) / max(r_min, RHO_FLOOR) if r_max > 1.0e3 * RHO_FLOOR else 0.0
        inner = nonmink and sweep == DIR_X and i <= 0
        atmo = P(DE, i) <= atm or P(DE, i + 1) <= atm
        cliff = p_jump >= 10.0 or rho_jump >= 10.0
        shock = p_jump >= 0.80 or rho_jump >= 0.50
        smooth_break = p_jump >= 0.40 or rho_jump >= 0.15
        if rec == GODUNOV:
            br = "godunov"
        elif rec == TVD:
            br = "godunov" if sensor and (inner or atmo or cliff) else "tvd"
        elif rec == WENO3:
            if sensor:
                br = "godunov" if (inner or atmo or cliff) else ("mc" if shock else "weno3")
            else:
                br = "godunov" if inner else "weno3"
        elif rec == MP5:
            if sensor:
                edge = ((nonmink and sweep == DIR_X and i <= 3) or
                        (nonmink and sweep == DIR_Y and (i <= 2 or i >= nodes - 2)))
                br = ("godunov" if (inner or atmo or cliff) else "mc" if shock else
                      "weno3" if (smooth_break or edge) else "mp5")
            else:
                br = "godunov" if inner else "mp5"
        else:
            if sensor:
                br = ("godunov" if (inner or atmo or cliff) else "mc" if shock else
                      "weno3" if smooth_break else "weno5")
            else:
                br = "godunov" if inner else "weno5"
        for k in range(NEQ):
            s = lambda m: P(k, i + m)
            if br == "godunov":
                l, r = s(0), s(1)
            elif br in ("tvd", "mc"):
                lm = lim if br == "tvd" else MC
                l = s(0) + 0.5 * tvd_slope(s(0) - s(-1), s(1) - s(0), lm)
                r = s(1) - 0.5 * tvd_slope(s(1) - s(0), s(2) - s(1), lm)
            elif br == "weno3":
                l, r = weno3(s(-1), s(0), s(1)), weno3(s(2), s(1), s(0))
            elif br == "mp5":
                l, r = mp5(s(-2), s(-1), s(0), s(1), s(2)), mp5(s(3), s(2), s(1), s(0), s(-1))
            else:
                l, r = weno5(s(-2), s(-1), s(0), s(1), s(2)), weno5(s(3), s(2), s(1), s(0), s(-1))
            qL[i][k], qR[i][k] = l, r
    for i in range(nodes + 1):  # reconstruction.f90:647-655
        qL[i][DE] = max(qL[i][DE], RHO_FLOOR)
        qR[i][DE] = max(qR[i][DE], RHO_FLOOR)
        qL[i][PR] = max(qL[i][PR], P_FLOOR)
        qR[i][PR] = max(qR[i][PR], P_FLOOR)
    return np.array(qL), np.array(qR)


def strip(rng, n, g):
    """Cells -g..n+g: smooth stretches, jumps of every size the sensor grades, an
    atmosphere patch, constant runs and tiny sub-floor values."""
    m = n + 2 * g + 1
    x = np.linspace(0.0, 1.0, m)
    rho = 1.0 + 0.3 * np.sin(2 * np.pi * rng.uniform(0.5, 3.0) * x + rng.uniform(0, 6.3))
    p = 0.5 + 0.2 * np.cos(2 * np.pi * rng.uniform(0.5, 3.0) * x)
    for _ in range(rng.integers(0, 4)):  # jumps: 10 % .. 2000 %
        at, f = rng.integers(0, m), rng.choice([1.1, 1.3, 1.7, 3.0, 20.0])
        rho[at:] *= f if rng.random() < 0.5 else 1.0 / f
        p[at:] *= rng.choice([1.0, f, 1.0 / f])
    if rng.random() < 0.3:  # atmosphere patch
        a = rng.integers(0, m - 4)
        rho[a:a + 4] = rng.choice([1e-9, 5e-10, 1e-12])
        p[a:a + 4] = rng.choice([1e-12, 1e-14])
    if rng.random() < 0.3:  # constant run: exact zero slopes
        a = rng.integers(0, m - 6)
        rho[a:a + 6] = rho[a]
        p[a:a + 6] = p[a]
    v = rng.uniform(-0.5, 0.5, (m, 3))
    if rng.random() < 0.3:
        v[rng.integers(0, m):, 0] = 0.0
    return np.column_stack([rho, p, v])


def oracle_reconstruct(prim, nodes, rec, lim, sensor, metric, sweep):
    c = B.OrcConfig()
    g = (len(prim) - nodes - 1) // 2
    c.nx, c.ny, c.nz, c.nghost = nodes, 1, 1, g
    c.rec_method, c.tvd_limiter, c.riemann, c.shock_sensor = rec, lim, 1, int(sensor)
    c.metric_kind, c.geom_kind, c.case_id = metric, 0, 1
    c.dx = c.dy = c.dz = 1.0
    c.adb_idx, c.g1, c.cfl = 4.0 / 3.0, 4.0, 0.4
    c.rho_floor, c.p_floor, c.v_max = RHO_FLOOR, P_FLOOR, 1.0 - 1.0e-5
    pr = np.ascontiguousarray(prim, dtype=np.float64)
    qL, qR = np.zeros((nodes + 1, NEQ)), np.zeros((nodes + 1, NEQ))
    cnt = B.OrcCounters()
    dp = lambda a: a.ctypes.data_as(C.POINTER(C.c_double))
    B.lib(libm_exp=True).orc_reconstruct(C.byref(c), dp(pr), nodes, sweep, dp(qL), dp(qR), C.byref(cnt))
    return qL, qR


CASES = [(rec, lim) for rec in (GODUNOV, WENO3, MP5, WENO5) for lim in (MC,)] + \
        [(TVD, lim) for lim in (MINMOD, SUPERBEE, MC)]


@pytest.mark.parametrize("rec,lim", CASES)
@pytest.mark.parametrize("sensor", [False, True])
@pytest.mark.parametrize("metric", [0, 2])  # Minkowski; Kerr-Schild (the inner-radius overrides)
def test_reconstruction_matches_an_independent_restatement(rec, lim, sensor, metric):
    rng = np.random.default_rng(1000 * rec + 100 * lim + 10 * int(sensor) + metric)
    nodes, g = 24, 3
    checked = 0
    for sweep in (DIR_X, DIR_Y, DIR_Z):
        for _ in range(6):
            prim = strip(rng, nodes, g)
            wl, wr = reconstruct(prim, nodes, rec, lim, sensor, metric != 0, sweep)
            ol, orr = oracle_reconstruct(prim, nodes, rec, lim, sensor, metric, sweep)
            assert wl.tobytes() == ol.tobytes(), (sweep, np.argwhere(wl != ol)[:3])
            assert wr.tobytes() == orr.tobytes(), (sweep, np.argwhere(wr != orr)[:3])
            checked += 1
    assert checked == 18


def test_sensor_strips_reach_every_branch():
    """The strips above drive WENO5 with the sensor through all of its branches."""
    rng = np.random.default_rng(7)
    seen = set()
    for _ in range(60):
        prim = strip(rng, 24, 3)
        for i in range(25):
            P = lambda k, j: prim[j + 3][k]
            pw = [P(PR, i + m) for m in range(-2, 3)]
            rw = [P(DE, i + m) for m in range(-2, 3)]
            pj = (max(pw) - min(pw)) / max(min(pw), P_FLOOR) if max(pw) > 1e3 * P_FLOOR else 0.0
            rj = (max(rw) - min(rw)) / max(min(rw), RHO_FLOOR) if max(rw) > 1e3 * RHO_FLOOR else 0.0
            if P(DE, i) <= 1e2 * RHO_FLOOR or P(DE, i + 1) <= 1e2 * RHO_FLOOR:
                seen.add("atmosphere")
            elif pj >= 10.0 or rj >= 10.0:
                seen.add("cliff")
            elif pj >= 0.8 or rj >= 0.5:
                seen.add("tvd")
            elif pj >= 0.4 or rj >= 0.15:
                seen.add("weno3")
            else:
                seen.add("weno5")
    assert seen == {"atmosphere", "cliff", "tvd", "weno3", "weno5"}
