"""The reference's HLLC/HLLE known-answer tests (tests/test_hllc_fluxes.f90:95-292) through
the GPU C-ABI entry points grhd2_gpu_riemann_faces / grhd2_gpu_physical_flux, plus a
face-by-face comparison with the oracle on random states."""
import numpy as np
import pytest

from grhd_b200.solver import GpuGrid
from tests.helpers import shock_tube, torus_2p5d
from tests.test_oracle_kats import G_GEN, I3, cfg, close, phys_flux, riemann

pytestmark = pytest.mark.gpu


def grid(metric_ks: bool, rs: str):
    # Gamma = 4/3 as in the fixture of tests/test_hllc_fluxes.f90:11
    pb = (torus_2p5d(nx=8, nz=4, rs=rs) if metric_ks
          else shock_tube(nx=8, rs=rs, adiabatic_index=1.3333333333333333))
    return GpuGrid(pb, upload_initial=False)


def g_riemann(G, qL, qR, d, alpha, beta, g, sqg):
    return G.riemann_faces(d, np.array([qL], float), np.array([qR], float), alpha, beta, g, sqg)[0]


def g_flux(G, q, d, alpha, beta, g, sqg):
    return G.physical_flux(d, np.array([q], float), alpha, beta, g, sqg)[0]


def test_kats_cartesian():
    G = grid(False, "hllc")
    z = np.zeros(3)
    q = [1.2, 0.25, 0.12, -0.07, 0.05]
    for d in (1, 2, 3):
        close(g_riemann(G, q, q, d, 1.0, z, I3, 1.0), g_flux(G, q, d, 1.0, z, I3, 1.0), 2e-12)
    qL, qR = [1.0, 0.4, 0, 0, 0], [0.125, 0.4, 0, 0, 0]
    close(g_riemann(G, qL, qR, 1, 1.0, z, I3, 1.0), g_flux(G, qL, 1, 1.0, z, I3, 1.0), 2e-12)
    qL, qR = [1.0, 0.1, 0.2, 0.03, -0.02], [0.2, 0.1, 0.2, 0.03, -0.02]
    close(g_riemann(G, qL, qR, 1, 1.0, z, I3, 1.0), g_flux(G, qL, 1, 1.0, z, I3, 1.0), 3e-12)
    qL, qR = [1.0, 0.2, 0.0, 0.30, -0.10], [0.4, 0.2, 0.0, -0.20, 0.15]
    close(g_riemann(G, qL, qR, 1, 1.0, z, I3, 1.0), np.array([0, 0, 0.2, 0, 0]), 3e-12)
    qL, qR = [4e-10, 2e-13, 0.12, 0, 0], [1.2e-10, 2e-13, 0.12, 0, 0]
    close(g_riemann(G, qL, qR, 1, 1.0, z, I3, 1.0), g_flux(G, qL, 1, 1.0, z, I3, 1.0), 1e-18)
    qL, qR = np.array([1.0, 1.0, 0.30, 0.10, 0.0]), np.array([0.125, 0.10, -0.10, -0.05, 0.02])
    sL, sR = qL.copy(), qR.copy()
    sL[:2] *= 1e-10
    sR[:2] *= 1e-10
    close(g_riemann(G, sL, sR, 1, 1.0, z, I3, 1.0) / 1e-10, g_riemann(G, qL, qR, 1, 1.0, z, I3, 1.0), 2e-11)
    assert np.all(np.isfinite(g_riemann(G, [1.0, 1e3, 0, 0, 0], [1.0, 1e-2, 0, 0, 0], 1, 1.0, z, I3, 1.0)))


def test_kats_general_metric():
    G = grid(True, "hllc")
    sqg = np.sqrt(np.linalg.det(G_GEN))
    beta = np.array([0.18, -0.05, 0.09])
    q = [0.9, 0.12, 0.08, -0.04, 0.06]
    for d in (1, 2, 3):
        close(g_riemann(G, q, q, d, 0.73, beta, G_GEN, sqg), g_flux(G, q, d, 0.73, beta, G_GEN, sqg), 5e-12)
    b = np.array([0.3, 0, 0])
    qL, qR = [1.0, 0.1, 0.2, 0.03, -0.02], [0.2, 0.1, 0.2, 0.03, -0.02]
    close(g_riemann(G, qL, qR, 1, 0.8, b, I3, 1.0), g_flux(G, qR, 1, 0.8, b, I3, 1.0), 3e-12)
    g = np.diag([2.2, 1.4, 3.1])
    g[0, 2] = g[2, 0] = -0.45
    s = np.sqrt(np.linalg.det(g))
    qL, qR = [1.0, 0.15, 0.0, 0.04, 0.08], [0.3, 0.15, 0.0, -0.03, -0.05]
    close(g_riemann(G, qL, qR, 1, 0.75, np.zeros(3), g, s), g_flux(G, qL, 1, 0.75, np.zeros(3), g, s), 5e-12)
    b = np.array([0.02, -0.01, 0.03])
    qL, qR = [1.1, 0.12, 0.08, -0.04, 0.06], [0.25, 0.12, 0.08, -0.04, 0.06]
    close(g_riemann(G, qL, qR, 1, 0.8, b, G_GEN, sqg), g_flux(G, qL, 1, 0.8, b, G_GEN, sqg), 8e-12)


@pytest.mark.parametrize("rs,metric_ks", [("hlle", False), ("hllc", False), ("hlle", True), ("hllc", True)])
def test_random_faces_match_oracle(rs, metric_ks):
    """Random admissible face problems: GPU flux == oracle flux (FP64, same operation order)."""
    rng = np.random.default_rng(11)
    n = 2000
    qL = np.column_stack([10 ** rng.uniform(-3, 1, n), 10 ** rng.uniform(-4, 2, n), rng.uniform(-0.5, 0.5, (n, 3))])
    qR = np.column_stack([10 ** rng.uniform(-3, 1, n), 10 ** rng.uniform(-4, 2, n), rng.uniform(-0.5, 0.5, (n, 3))])
    G = grid(metric_ks, rs)
    c = cfg(metric=2 if metric_ks else 0, geom=3 if metric_ks else 0, rs=2 if rs == "hllc" else 1)
    g = G_GEN if metric_ks else I3
    beta = np.array([0.18, -0.05, 0.09]) if metric_ks else np.zeros(3)
    alpha = 0.73 if metric_ks else 1.0
    sqg = float(np.sqrt(np.linalg.det(g)))
    for d in (1, 2, 3):
        fg = G.riemann_faces(d, qL, qR, alpha, beta, g, sqg)
        fo = np.array([riemann(c, qL[f], qR[f], d, alpha, beta, g, sqg) for f in range(n)])
        assert np.array_equal(fg, fo), np.abs(fg - fo).max()
