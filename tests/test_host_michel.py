"""The host set-up's Michel accretion state against setup_michel_accretion_initial
(conditions.f90:284-410) and cache_michel_injector (:229-246) restated here in plain
Python.

The critical-point constants, the 40-step secant-Newton solve of h u^t = C2 / C1 per
radius (a +-1e-6 central difference for the derivative, stopping at |f| < 1e-12), the
polytrope, and the Eulerian velocity from the quadratic for u^t with the metric at the
cell -- over p(:, 1:nx+nghost, 1:ny, 1:nz), so the injector ghosts take the same solution --
bit for bit, in logarithmic and physical radius.  The metric comes from the host's
calculate_metric probe, itself pinned by the reference's metric tests.
"""
import math

import numpy as np
import pytest

from tests.helpers import michel
from tests.test_host_kats import EF, SPH, metric_at


def michel_state(pb):
    info, cfg = pb.info, pb.config(0)
    M, adb, g1 = info.bh_mass, cfg.adb_idx, cfg.g1
    keys = dict(line.split("=", 1) for line in pb.text.splitlines() if "=" in line)
    keys = {k.strip(): v.strip() for k, v in keys.items()}
    rc = float(keys.get("michel_critical_radius", "100"))
    rhoc = float(keys.get("michel_critical_density", "0.1"))
    log_r = bool(cfg.use_log_r)
    u_c = -math.sqrt(M / (2.0 * rc))
    ut_c = math.sqrt(1.0 - 2.0 * M / rc + u_c * u_c)
    Vc2 = (u_c / ut_c) * (u_c / ut_c)
    pres = (Vc2 * rhoc) / (adb - Vc2 * g1)
    K = pres / math.pow(rhoc, adb)
    h = 1.0 + g1 * pres / rhoc
    C1 = rc * rc * rhoc * u_c
    C2 = rc * rc * rhoc * h * u_c * ut_c
    eps = 1.0e-6
    x, y, _ = pb.coords()
    g = pb.ng
    out = {}
    for i in range(1, pb.nx + g + 1):
        xi = x[i + g]
        r = math.exp(xi) if log_r else xi
        ur = -math.sqrt(2.0 * M / r)
        for _ in range(40):
            ut = math.sqrt(1.0 - 2.0 * M / r + ur * ur)
            rho = C1 / (r * r * ur)
            p = K * math.pow(rho, adb)
            hs = 1.0 + g1 * p / rho
            f = hs * ut - C2 / C1
            urp, urm = ur + eps, ur - eps
            fp = (1.0 + g1 * (K * math.pow(C1 / (r * r * urp), adb)) / (C1 / (r * r * urp))) * \
                math.sqrt(1.0 - 2.0 * M / r + urp * urp) - C2 / C1
            fm = (1.0 + g1 * (K * math.pow(C1 / (r * r * urm), adb)) / (C1 / (r * r * urm))) * \
                math.sqrt(1.0 - 2.0 * M / r + urm * urm) - C2 / C1
            df = (fp - fm) / (2.0 * eps)
            ur = ur - f / df
            if abs(f) < 1.0e-12:
                break
        rho = C1 / (r * r * ur)
        p = K * math.pow(rho, adb)
        for j in range(1, pb.ny + 1):
            alpha, beta, gam = metric_at(EF, SPH, log_r, M, 0.0, pb.ny, xi, y[j + g])[:3]
            ux = ur / r if log_r else ur
            g_tt = -(alpha * alpha)
            for ii in range(3):
                for jj in range(3):
                    g_tt = g_tt + gam[ii][jj] * beta[ii] * beta[jj]
            g_tx = 0.0
            for jj in range(3):
                g_tx = g_tx + gam[0][jj] * beta[jj]
            A, B, Cq = g_tt, 2.0 * g_tx * ux, gam[0][0] * (ux * ux) + 1.0
            ut_con = (-B - math.sqrt(B * B - 4.0 * A * Cq)) / (2.0 * A)
            W = alpha * ut_con
            out[(i, j)] = [rho, p, ux / W + beta[0] / alpha, beta[1] / alpha, beta[2] / alpha]
    return out


@pytest.mark.parametrize("kw", [dict(nx=128), dict(nx=96, logarithmic_r=False, r_min=1.8),
                                dict(nx=64, michel_critical_radius=12.0, michel_critical_density=0.3)])
def test_michel_state_matches_an_independent_restatement(kw):
    pb = michel(**kw)
    want = michel_state(pb)
    p = pb.initial_prims()
    g = pb.ng
    for (i, j), state in want.items():
        for k in range(1, pb.nz + 1):
            assert p[k + g, j + g, i + g].tobytes() == np.array(state).tobytes(), (i, j, k, p[k + g, j + g, i + g],
                                                                                   state)
    inj = np.ctypeslib.as_array(pb.bc_view().michel_injector, (5 * g * pb.ny * pb.nz,)).reshape(pb.nz, pb.ny, g, 5)
    for gg in range(1, g + 1):
        assert inj[0, 0, gg - 1].tobytes() == np.array(want[(pb.nx + gg, 1)]).tobytes()
