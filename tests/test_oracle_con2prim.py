"""A second, independent reading of the reference's primitive recovery against the oracle's.

cons_to_prim (equations.f90:94-205) with eval_V_and_dV (:211-218), eval_residual
(:221-246), root_safe_newton (:249-336) and root_brent (:339-424) is restated here in plain
Python straight from the Fortran -- gfortran's integer powers as products, its MAX/MIN
returning the non-NaN argument, SIGN by the sign bit -- and compared, bit for bit and
branch for branch (the oracle's failure counters), with the oracle's restatement on cells
of a random general metric: physical states over a range of Lorentz factors, then the
same states pushed into every failure branch (D below the floor, superluminal momentum,
negative tau, NaN, a root finder that must bisect or fall back to Brent).
"""
import ctypes as C
import math

import numpy as np
import pytest

from oracle import binding as B

RHO_FLOOR, P_FLOOR, V_MAX = 1.0e-10, 1.0e-13, 1.0 - 1.0e-5
DE, PR, VX, VY, VZ = 0, 1, 2, 3, 4


def fmax(a, b):  # gfortran MAX: the second argument when it is larger or the first is NaN
    return b if (b > a or a != a) else a


def fmin(a, b):
    return b if (b < a or a != a) else a


def sgn(x, a=1.0):
    return math.copysign(abs(a), x)


def qsq(ginv, cs):
    s = 0.0
    for ii in range(3):
        for jj in range(3):
            s = s + ginv[ii][jj] * cs[VX + ii] * cs[VX + jj]
    return s


def eval_V_and_dV(g1, W, cs):
    denom = g1 * (W * W) - 1.0
    V = (g1 * (W * W) * (cs[PR] + cs[DE]) - cs[DE] * W) / denom
    dV = (g1 * W * (cs[DE] * W - 2.0 * (cs[PR] + cs[DE])) + cs[DE]) / (denom * denom)
    return V, dV


def eval_residual(g1, W, cs, ginv):
    V, dV = eval_V_and_dV(g1, W, cs)
    Q = qsq(ginv, cs)
    W3 = W * W * W
    res = (V * V) * (1.0 - 1.0 / (W * W)) - Q
    dres = 2.0 * V * (dV * (W3 - W) + V) / W3
    return res, dres


def root_brent(g1, cs, ginv):
    EPS, x_acc, x1 = 3.0e-8, 1.0e-8, 1.0
    W_max_guess = (math.sqrt(qsq(ginv, cs)) + cs[DE]) / fmax(cs[DE], RHO_FLOOR)
    x2 = fmax(1.0e4, W_max_guess * 2.0)
    fa, _ = eval_residual(g1, x1, cs, ginv)
    fb, _ = eval_residual(g1, x2, cs, ginv)
    if sgn(fa) * sgn(fb) > 0.0:
        return -1.0
    a, b = x1, x2
    c, fc = b, fb
    d = e = 0.0
    for _ in range(100):
        if sgn(fb) * sgn(fc) > 0.0:
            c, fc = a, fa
            d = b - a
            e = d
        if abs(fc) < abs(fb):
            a = b; b = c; c = a
            fa = fb; fb = fc; fc = fa
        tol1 = 2.0 * EPS * abs(b) + 0.5 * x_acc
        xm = 0.5 * (c - b)
        if abs(xm) <= tol1 or abs(fb) < 1.0e-14:
            return b
        if abs(e) >= tol1 and abs(fa) > abs(fb):
            y1 = fb / fa
            if abs(a - c) < 1.0e-14:
                o = 2.0 * xm * y1
                q = 1.0 - y1
            else:
                q = fa / fc
                r = fb / fc
                o = y1 * (2.0 * xm * q * (q - r) - (b - a) * (r - 1.0))
                q = (q - 1.0) * (r - 1.0) * (y1 - 1.0)
            if o > 0.0:
                q = -q
            o = abs(o)
            if 2.0 * o < fmin(3.0 * xm * q - abs(tol1 * q), abs(e * q)):
                e = d
                d = o / q
            else:
                d = xm
                e = d
        else:
            d = xm
            e = d
        a, fa = b, fb
        b = b + d if abs(d) > tol1 else b + sgn(xm, tol1)
        fb, _ = eval_residual(g1, b, cs, ginv)
    return -1.0


def root_safe_newton(g1, cs, ginv):
    """(W, whether Brent was called)"""
    x_acc, x1 = 1.0e-10, 1.0
    W_max_guess = (math.sqrt(qsq(ginv, cs)) + cs[DE]) / fmax(cs[DE], RHO_FLOOR)
    x2 = fmax(1.0e3, W_max_guess * 2.0)
    f_low, _ = eval_residual(g1, x1, cs, ginv)
    f_high, _ = eval_residual(g1, x2, cs, ginv)
    if abs(f_low) < 1.0e-14:
        return x1, False
    if abs(f_high) < 1.0e-14:
        return x2, False
    if sgn(f_low) * sgn(f_high) > 0.0:
        return -1.0, False
    if f_low < 0.0:
        x_low, x_high = x1, x2
    else:
        x_high, x_low = x1, x2
    root = 0.5 * (x1 + x2)
    diff_x_old = abs(x2 - x1)
    diff_x = diff_x_old
    f, df = eval_residual(g1, root, cs, ginv)
    converged = False
    for _ in range(100):
        if ((root - x_high) * df - f) * ((root - x_low) * df - f) > 0.0 or abs(2.0 * f) > abs(diff_x_old * df):
            diff_x_old = diff_x
            diff_x = 0.5 * (x_high - x_low)
            root = x_low + diff_x
            if abs(x_low - root) < 1.0e-14:
                return root, False
        else:
            diff_x_old = diff_x
            diff_x = f / df
            temp = root
            root = root - diff_x
            if abs(temp - root) < 1.0e-14:
                return root, False
        if abs(diff_x) < x_acc:
            converged = True
            return root, False
        f, df = eval_residual(g1, root, cs, ginv)
        if f < 0.0:
            x_low = root
        else:
            x_high = root
    if not converged or abs(f) > 1.0e-6:
        return root_brent(g1, cs, ginv), True
    return root, False


def cons_to_prim(g1, cons, g, ginv, sqg):
    """(cons after the call, prim, the set of branches taken)"""
    cs = list(cons)
    pr = [0.0] * 5
    taken = set()
    lDf = RHO_FLOOR * sqg
    lTf = P_FLOOR * (g1 - 1.0) * sqg

    def floor():
        return [lDf, lTf, 0.0, 0.0, 0.0], [RHO_FLOOR, P_FLOOR, 0.0, 0.0, 0.0]

    if cs[DE] <= lDf:
        taken.add("floor_pre")
        c2, p2 = floor()
        return c2, p2, taken
    S = cs[VX:VZ + 1]
    S_sq = (S[0] * (ginv[0][0] * S[0] + ginv[0][1] * S[1] + ginv[0][2] * S[2])
            + S[1] * (ginv[1][0] * S[0] + ginv[1][1] * S[1] + ginv[1][2] * S[2])
            + S[2] * (ginv[2][0] * S[0] + ginv[2][1] * S[1] + ginv[2][2] * S[2]))
    E_tot = cs[PR] + cs[DE]
    S_sq_max = fmax(0.0, E_tot * E_tot - cs[DE] * cs[DE]) * V_MAX
    if S_sq > S_sq_max and S_sq > 1.0e-20:
        taken.add("causal")
        sf = math.sqrt(S_sq_max / S_sq)
        cs[VX] = cs[VX] * sf
        cs[VY] = cs[VY] * sf
        cs[VZ] = cs[VZ] * sf
    W, brent = root_safe_newton(g1, cs, ginv)
    if brent:
        taken.add("brent")
    if W < 1.0:
        taken.add("root_fail")
        c2, p2 = floor()
        return c2, p2, taken
    V, _ = eval_V_and_dV(g1, W, cs)
    if V <= 0.0 or V != V:
        taken.add("bad_V")
        c2, p2 = floor()
        return c2, p2, taken
    pr[DE] = cs[DE] / (W * sqg)
    pr[PR] = (V - cs[PR] - cs[DE]) / sqg
    for a in range(3):
        pr[VX + a] = (ginv[a][0] * cs[VX] + ginv[a][1] * cs[VY] + ginv[a][2] * cs[VZ]) / V
    vsq = 0.0
    for ii in range(3):
        for jj in range(3):
            vsq = vsq + g[ii][jj] * pr[VX + ii] * pr[VX + jj]
    if (pr[DE] < RHO_FLOOR or pr[PR] < P_FLOOR or any(x != x for x in pr) or vsq != vsq or vsq >= V_MAX):
        taken.add("sanitise")
        c2, p2 = floor()
        return c2, p2, taken
    return cs, pr, taken


# ---- the comparison -------------------------------------------------------------------
G1 = 4.0  # Gamma / (Gamma - 1) for Gamma = 4/3
COUNTERS = {"floor_pre": "c2p_floor_pre", "causal": "c2p_causal_rescale", "brent": "c2p_brent_used",
            "root_fail": "c2p_root_fail", "bad_V": "c2p_bad_V", "sanitise": "c2p_final_sanitise"}


class Cells:
    """n cells (nx = n, ny = 1), each with its own random positive-definite 3-metric."""

    def __init__(self, rng, n):
        self.n = n
        A = rng.normal(size=(n, 3, 3)) * 0.3
        g = np.einsum("nij,nkj->nik", A, A) + np.eye(3) * rng.uniform(0.5, 3.0, (n, 1, 1))
        self.g = g
        self.ginv = np.linalg.inv(g)
        self.ginv = 0.5 * (self.ginv + self.ginv.transpose(0, 2, 1))  # exactly symmetric
        self.sqg = np.sqrt(np.linalg.det(g))
        # Fortran (3,3) column-major per cell = the transpose in C order; symmetric anyway
        self.gamma_c = np.ascontiguousarray(g.transpose(0, 2, 1)).reshape(-1)
        self.ginv_c = np.ascontiguousarray(self.ginv.transpose(0, 2, 1)).reshape(-1)
        self.m = B.OrcMetric()
        dp = lambda a: a.ctypes.data_as(C.POINTER(C.c_double))
        self.m.gamma_c, self.m.gamma_inv_c, self.m.sqrt_gamma_c = dp(self.gamma_c), dp(self.ginv_c), dp(self.sqg)
        c = B.OrcConfig()
        c.nx, c.ny, c.nz, c.nghost = n, 1, 1, 3
        c.rec_method, c.tvd_limiter, c.riemann, c.shock_sensor = 5, 3, 1, 0
        c.metric_kind, c.geom_kind, c.case_id = 2, 3, 10
        c.dx = c.dy = c.dz = 1.0
        c.adb_idx, c.g1, c.cfl = 4.0 / 3.0, G1, 0.4
        c.rho_floor, c.p_floor, c.v_max = RHO_FLOOR, P_FLOOR, V_MAX
        self.c = c

    def prim_to_cons(self, i, prim):
        p = np.ascontiguousarray(prim, dtype=np.float64)
        u = np.zeros(5)
        dp = lambda a: a.ctypes.data_as(C.POINTER(C.c_double))
        B.lib().orc_prim_to_cons(C.byref(self.c), C.byref(self.m), dp(p), dp(u), i + 1, 1)
        return u

    def oracle(self, i, cons):
        u = np.array(cons, dtype=np.float64)
        p = np.zeros(5)
        cnt = B.OrcCounters()
        dp = lambda a: a.ctypes.data_as(C.POINTER(C.c_double))
        B.lib().orc_cons_to_prim(C.byref(self.c), C.byref(self.m), dp(u), dp(p), i + 1, 1, C.byref(cnt))
        d = cnt.as_dict()
        return u, p, {k for k, name in COUNTERS.items() if d[name]}

    def restated(self, i, cons):
        c2, p2, taken = cons_to_prim(G1, list(cons), self.g[i].tolist(), self.ginv[i].tolist(), float(self.sqg[i]))
        return np.array(c2), np.array(p2), taken


def physical_prims(rng, n, g):
    rho = 10.0 ** rng.uniform(-6, 1, n)
    p = 10.0 ** rng.uniform(-8, 2, n)
    out = np.zeros((n, 5))
    for i in range(n):
        d = rng.normal(size=3)
        vmag = rng.choice([0.0, rng.uniform(0, 0.5), rng.uniform(0.5, 0.99), rng.uniform(0.99, 0.9989)])
        d = d / math.sqrt(d @ g[i] @ d)  # unit length in the metric
        out[i] = [rho[i], p[i], *(vmag * d)]
    return out


def _compare(cells, i, cons, seen):
    ou, op, ot = cells.oracle(i, cons)
    ru, rp, rt = cells.restated(i, cons)
    assert ot == rt, (i, cons, ot, rt)
    assert op.tobytes() == rp.tobytes(), (i, cons, op, rp)
    assert ou.tobytes() == ru.tobytes(), (i, cons, ou, ru)
    seen |= rt or {"ok"}


def test_con2prim_matches_an_independent_restatement_on_physical_states():
    rng = np.random.default_rng(11)
    cells = Cells(rng, 400)
    prims = physical_prims(rng, cells.n, cells.g)
    seen = set()
    for i in range(cells.n):
        _compare(cells, i, cells.prim_to_cons(i, prims[i]), seen)
    assert "ok" in seen


@pytest.mark.parametrize("seed", [1, 2, 3])
def test_con2prim_matches_an_independent_restatement_in_every_branch(seed):
    rng = np.random.default_rng(100 + seed)
    cells = Cells(rng, 300)
    prims = physical_prims(rng, cells.n, cells.g)
    seen = set()
    for i in range(cells.n):
        u = cells.prim_to_cons(i, prims[i])
        kind = i % 8
        if kind == 1:
            u[DE] = RHO_FLOOR * cells.sqg[i] * rng.uniform(0.1, 1.0)    # below the density floor
        elif kind == 2:
            u[VX:] *= rng.uniform(1.5, 20.0)                             # superluminal momentum
        elif kind == 3:
            u[PR] = -abs(u[PR]) * rng.uniform(0.5, 5.0)                  # negative tau
        elif kind == 4:
            u[VX + rng.integers(0, 3)] = float("nan")
        elif kind == 5:
            u[PR] *= rng.uniform(1e-6, 1e-3)                             # near-zero pressure
        elif kind == 6:
            u[DE] *= rng.uniform(1e-4, 1e-2)                             # light, fast
            u[VX:] *= rng.uniform(0.9, 1.2)
        elif kind == 7:
            u = u * rng.uniform(0.9, 1.1, 5)                             # jittered
        _compare(cells, i, u, seen)
    assert {"floor_pre", "causal", "ok"} <= seen
    assert seen & {"root_fail", "bad_V", "sanitise"}


def test_brent_fallback_matches_an_independent_restatement():
    """root_brent on its own (the hybrid Newton-bisection solver converged within its 100
    iterations on every state above and on 2e5 random ones, so the fallback is compared
    directly): bracketed states, unbracketed ones (-1) and NaN."""
    rng = np.random.default_rng(17)
    cells = Cells(rng, 64)
    dp = lambda a: a.ctypes.data_as(C.POINTER(C.c_double))
    prims = physical_prims(rng, cells.n, cells.g)
    outcomes = set()
    for i in range(cells.n):
        u = cells.prim_to_cons(i, prims[i])
        if i % 4 == 1:
            u[PR] = -abs(u[PR])
        elif i % 4 == 2:
            u[VX] = float("nan")
        ginv = np.ascontiguousarray(cells.ginv[i].T).reshape(-1)
        got = B.lib().orc_root_brent(C.byref(cells.c), dp(np.ascontiguousarray(u)), dp(ginv))
        want = root_brent(G1, list(u), cells.ginv[i].tolist())
        assert np.float64(got).tobytes() == np.float64(want).tobytes(), (i, u, got, want)
        outcomes.add("fail" if want == -1.0 else ("nan" if want != want else "root"))
    assert {"root", "fail"} <= outcomes
