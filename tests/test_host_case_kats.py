"""The reference's case-correction tests of the set-up (tests/test_case_corrections.f90)
against the host set-up (grhd_b200/csrc/host/problem.cpp), which builds the metric tables
and initial data of both the oracle and the GPU path (and, since metric_eval.h is shared,
of the device-built metric tables too):

* check_axisymmetric_jet_preset (:27-46): the jet preset's azimuthal faces 0 and pi;
* check_cylindrical_geometry (:48-91): Minkowski in cylindrical coordinates, every quantity
  of calculate_metric, calculate_christoffel_symbols and calculate_metric_derivatives;
* check_khi_perturbation (:94-144): the Kelvin-Helmholtz base state and its transverse,
  interface-localised perturbation;
* check_offaxis_logarithmic_radius (:147-183): the off-axis blast measured in physical
  radius on a logarithmic grid;
* check_dust_solution_and_boundaries (:186-232): the stationary dust solution's mass flux,
  free-fall energy, cold pressure and its logarithmic-coordinate transformation (its
  boundary half, :234-261, is in tests/test_oracle_kats.py, as is check_shift_aware_outflow).

The reference sets module globals and coordinates directly; here the set-up is driven
through .par keys on uniform grids, so the KHI and off-axis checks place their cells with
the grid's own spacing (the KHI test on dyadic coordinates, so that a cell centre can sit
exactly on the interface as the reference's z(2) = 0.25 does).  Tolerances are the
reference's: 2e-13, and 2e-12 for the dust solution.
"""
import ctypes as C
import math

import numpy as np

from grhd_b200 import native as N
from grhd_b200.problem import Problem
from tests.test_host_kats import CART, CYL, EF, MINK, SPH, metric_at

TOL = 2.0e-13
PI = math.pi


def test_axisymmetric_jet_preset_azimuth():
    info = Problem.from_keys("axisymmetric_jet").info
    assert abs(info.y_min - 0.0) <= TOL
    assert abs(info.y_max - PI) <= TOL
    assert abs(0.5 * (info.y_min + info.y_max) - 0.5 * PI) <= TOL


def test_cylindrical_geometry():
    rho = 2.5
    alpha, beta, gamma, gmunu, det, dlna, ch, dg = metric_at(MINK, CYL, False, 0.0, 0.0, 1, rho, 0.0)
    g3 = np.diag([1.0, rho ** 2, 1.0])
    g4 = np.diag([-1.0, 1.0, 1.0 / rho ** 2, 1.0])
    ech = np.zeros((4, 4, 4))
    ech[1, 2, 2] = -rho
    ech[2, 1, 2] = ech[2, 2, 1] = 1.0 / rho
    edg = np.zeros((4, 4, 3))
    edg[2, 2, 0] = 2.0 * rho
    assert abs(alpha - 1.0) <= TOL
    assert abs(det - rho ** 2) <= TOL
    assert np.max(np.abs(beta)) <= TOL
    assert np.max(np.abs(gamma - g3)) <= TOL
    assert np.max(np.abs(gmunu - g4)) <= TOL
    assert np.max(np.abs(dlna)) <= TOL
    assert np.max(np.abs(ch - ech)) <= TOL
    assert np.max(np.abs(dg - edg)) <= TOL


def _interior(pb):
    """p(v, i, j, k) of the interior as a [k, j, i, v] array (1-based i, j, k at [k-1, j-1, i-1])."""
    p = pb.initial_prims()
    g = pb.ng
    return p[g + 1:g + 1 + pb.nz, g + 1:g + 1 + pb.ny, g + 1:g + 1 + pb.nx, :]


def test_khi_perturbation():
    # cells at x = 1/16, 1/8 and z = 3/16, 1/4, 5/16: the interface at |z| = 1/4, the
    # envelope width 1/16 (so z = 3/16 lies one width inside), the wave number 8 (so
    # sin(8 pi x) is 1 at x = 1/16 and has a node at x = 1/8)
    amp, width = 0.01, 0.0625
    pb = Problem.from_keys("khi", nx=2, ny=1, nz=3, r_min=0.03125, r_max=0.15625, z_min=0.15625, z_max=0.34375,
                           khi_half_width=0.25, khi_density_inner=2.0, khi_density_outer=1.0,
                           khi_velocity_inner=0.5, khi_velocity_outer=-0.5, khi_pressure=2.5,
                           khi_perturbation_amplitude=amp, khi_perturbation_wave_number=8.0,
                           khi_perturbation_width=width, perturbation="none")
    x, _, z = pb.coords()
    g = pb.ng
    assert x[g + 1] == 0.0625 and x[g + 2] == 0.125 and z[g + 1] == 0.1875 and z[g + 2] == 0.25
    q = _interior(pb)
    vx, vy, vz = 2, 3, 4
    assert abs(q[0, 0, 0, vx] - 0.5) <= TOL                    # inner base velocity unchanged
    assert abs(q[1, 0, 0, vx] - (-0.5)) <= TOL                 # outer base velocity unchanged
    assert abs(q[0, 0, 0, vz] - amp * math.exp(-0.5)) <= TOL   # transverse, one width off
    assert abs(q[1, 0, 0, vz] - amp) <= TOL                    # peaks at the interface
    assert abs(q[1, 0, 1, vz]) <= TOL                          # longitudinal node
    assert np.all(np.abs(q[0, 0, :, vy]) <= TOL)               # no y velocity


def test_offaxis_blast_logarithmic_radius():
    rc, w = 15.0, 1.5
    dx = math.log((rc + w) / rc)
    r_min = math.exp(math.log(rc) - 0.5 * dx)
    r_max = math.exp(math.log(rc) + 1.5 * dx)
    pb = Problem.from_keys("offaxis_blast", logarithmic_r=True, nx=2, ny=1, nz=1, r_min=r_min, r_max=r_max,
                           theta_min=0.0, theta_max=1.0, phi_min=0.0, phi_max=2.0,
                           offaxis_radial_center=rc, offaxis_phi_center=1.0, offaxis_width=w,
                           offaxis_background_density=0.1, offaxis_background_pressure=0.2,
                           offaxis_density_amplitude=1.0, offaxis_pressure_amplitude=0.5, perturbation="none")
    x, y, z = pb.coords()
    g = pb.ng
    assert abs(math.exp(x[g + 1]) - rc) <= 1e-12 and abs(math.exp(x[g + 2]) - (rc + w)) <= 1e-12
    assert abs(y[g + 1] - 0.5 * PI) <= TOL and abs(z[g + 1] - PI) <= TOL
    q = _interior(pb)
    assert abs(q[0, 0, 0, 0] - (0.1 + 1.0)) <= TOL                  # peak density
    assert abs(q[0, 0, 0, 1] - (0.2 + 0.5)) <= TOL                  # peak pressure
    assert abs(q[0, 0, 1, 0] - (0.1 + 1.0 * math.exp(-1.0))) <= TOL  # one physical width out


def _dust(log_r, x):
    s = np.zeros(5)
    assert N.host_lib().grhd2_host_dust_state(int(log_r), 1.0, -0.5, 1.0e-12, x, N.dptr(s)) == 0
    return s


def test_dust_accretion_solution():
    radius, M, c, tol = 5.0, 1.0, -0.5, 2.0e-12
    sp = _dust(False, radius)
    alpha, beta, gamma = metric_at(EF, SPH, False, M, 0.0, 1, radius, 0.5 * PI)[:3]
    W = 1.0 / math.sqrt(1.0 - gamma[0, 0] * sp[2] ** 2)
    u_r = W * (sp[2] - beta[0] / alpha)
    u_t = W / alpha
    assert abs(radius ** 2 * sp[0] * u_r - c) <= tol                                  # mass flux
    assert abs(-(1.0 - 2.0 * M / radius) * u_t + (2.0 * M / radius) * u_r - (-1.0)) <= tol  # free fall
    assert abs(sp[1] - 1.0e-12) <= tol                                                # cold pressure
    sl = _dust(True, math.log(radius))
    alpha, beta, gamma = metric_at(EF, SPH, True, M, 0.0, 1, math.log(radius), 0.5 * PI)[:3]
    W = 1.0 / math.sqrt(1.0 - gamma[0, 0] * sl[2] ** 2)
    u_r = radius * W * (sl[2] - beta[0] / alpha)
    assert abs(radius ** 2 * sl[0] * u_r - c) <= tol
    assert abs(sl[0] - sp[0]) <= tol
    assert abs(radius * sl[2] - sp[2]) <= tol


def test_dust_state_rejects_the_reference_failures():
    s = np.zeros(5)
    lib = N.host_lib()
    assert lib.grhd2_host_dust_state(0, 1.0, -0.5, 1e-12, 0.0, N.dptr(s)) == -1   # r <= 0
    assert lib.grhd2_host_dust_state(0, 0.0, -0.5, 1e-12, 5.0, N.dptr(s)) == -1   # M <= 0
    assert lib.grhd2_host_dust_state(0, 1.0, 0.5, 1e-12, 5.0, N.dptr(s)) == -1    # constant >= 0
    assert lib.grhd2_host_dust_state(0, 1.0, -0.5, 1e-12, 5.0, None) == -1
