"""Shared problem factories and comparisons for the parity tests.

The five workloads (shock tube, Michel accretion, 2.5D Kerr-Schild torus, 3D Kerr-Schild
torus, batched Riemann problems) are built with the reference's .par keys; the parity
tests run them at sizes the CPU oracle finishes in seconds.
"""
from __future__ import annotations

import numpy as np

from grhd_b200.problem import Problem


def shock_tube(nx=400, rec="weno5", rs="hlle", sensor=False, **kw) -> Problem:
    """Relativistic blast wave: rho 10|1, p 13.33|1e-6, Gamma 5/3, x in [0,1], t = 0.4."""
    keys = dict(nx=nx, adiabatic_index=1.6666666666666667, sod_interface=0.5, sod_density_left=10,
                sod_pressure_left=13.33, sod_density_right=1, sod_pressure_right=1e-6,
                reconstruction=rec, riemann_solver=rs, cfl=0.4, final_time=0.4, shock_sensor=sensor)
    keys.update(kw)
    return Problem.from_keys("sod", **keys)


def shock_tube_xy(nx=96, ny=24, rec="mp5", rs="hllc", sensor=False, **kw) -> Problem:
    """The shock tube on an x-y grid (nz = 1) with a moving left state and 5 % seeded
    pressure noise, so that every row along y differs: the layout with a y extent and no
    k extent."""
    keys = dict(ny=ny, sod_velocity_left=0.3, perturbation="pressure_noise", perturbation_amplitude=0.05,
                perturbation_time=0.0, perturbation_seed=11)
    keys.update(kw)
    return shock_tube(nx=nx, rec=rec, rs=rs, sensor=sensor, **keys)


def michel(nx=1024, rec="mp5", rs="hlle", sensor=False, **kw) -> Problem:
    """Michel accretion onto Schwarzschild (M=1), ingoing EF, log r in [1.8, 20], Gamma 4/3,
    sonic radius 8, 1e-3 isentropic density noise at t=0."""
    keys = dict(metric="eddington_finkelstein", geometry="spherical", logarithmic_r=True, bh_mass=1.0,
                nx=nx, ny=1, nz=1, r_min=1.8, r_max=20.0, adiabatic_index=1.3333333333333333,
                michel_critical_radius=8.0, reconstruction=rec, riemann_solver=rs, final_time=500.0,
                shock_sensor=sensor, perturbation="density_noise", perturbation_amplitude=0.001,
                perturbation_time=0.0, perturbation_seed=3435)
    keys.update(kw)
    return Problem.from_keys("michel", **keys)


def torus_2p5d(nx=400, nz=200, rec="weno5", rs="hlle", sensor=False, **kw) -> Problem:
    """Equatorial Fishbone-Moncrief torus, Kerr-Schild a=0.9, log r in [1.2,40], r_in 6,
    r_max 12, K 0.0015 (the preset's), Gamma 4/3, 1% pressure noise."""
    keys = dict(metric="kerr_schild", geometry="spheroidal", logarithmic_r=True, spin=0.9, bh_mass=1.0,
                nx=nx, ny=1, nz=nz, r_min=1.2, r_max=40.0, theta_min=0, theta_max=1, phi_min=0, phi_max=2,
                fm_inner_radius=6.0, fm_pressure_max_radius=12.0, fm_polytropic_constant=0.0015,
                adiabatic_index=1.3333333333333333, reconstruction=rec, riemann_solver=rs,
                shock_sensor=sensor, cfl=0.4, perturbation="pressure_noise",
                perturbation_amplitude=0.01, perturbation_time=0.0, perturbation_seed=3435)
    keys.update(kw)
    return Problem.from_keys("fishbone_equatorial", **keys)


def torus_3d(nx=256, ny=128, nz=128, rec="mp5", rs="hllc", sensor=True, **kw) -> Problem:
    """3D Fishbone-Moncrief torus, Kerr-Schild a=0.9, log r in [1.2,40], theta [0,pi],
    phi [0,2pi], the torus parameters of the 2.5D case, 1% pressure noise."""
    keys = dict(metric="kerr_schild", geometry="spheroidal", logarithmic_r=True, spin=0.9, bh_mass=1.0,
                nx=nx, ny=ny, nz=nz, r_min=1.2, r_max=40.0, theta_min=0, theta_max=1, phi_min=0, phi_max=2,
                fm_inner_radius=6.0, fm_pressure_max_radius=12.0, fm_polytropic_constant=0.0015,
                adiabatic_index=1.3333333333333333, reconstruction=rec, riemann_solver=rs,
                shock_sensor=sensor, cfl=0.4, perturbation="pressure_noise",
                perturbation_amplitude=0.01, perturbation_time=0.0, perturbation_seed=3435)
    keys.update(kw)
    return Problem.from_keys("fishbone_3d", **keys)


def initial_state(pb: Problem) -> np.ndarray:
    """Initial primitives with the configured t=0 perturbation applied on the host."""
    p = pb.initial_prims()
    if pb.info.perturbation_type != 0 and pb.info.perturbation_time <= 0.0:
        pb.perturb(p)
    return p


def interior(pb: Problem, p: np.ndarray) -> np.ndarray:
    g = pb.ng
    return p[g + 1:g + 1 + pb.nz, g + 1:g + 1 + pb.ny, g + 1:g + 1 + pb.nx, :]


def face_ghost_mask(pb: Problem) -> np.ndarray:
    """True for interior cells and ghost cells outside the domain in exactly one direction."""
    g = pb.ng
    k = np.arange(-g, pb.nz + g + 1)[:, None, None]
    j = np.arange(-g, pb.ny + g + 1)[None, :, None]
    i = np.arange(-g, pb.nx + g + 1)[None, None, :]
    out = (i < 1) | (i > pb.nx), (j < 1) | (j > pb.ny), (k < 1) | (k > pb.nz)
    n_out = out[0].astype(int) + out[1].astype(int) + out[2].astype(int)
    return n_out <= 1


def rel_l1(a: np.ndarray, b: np.ndarray) -> np.ndarray:
    a = a.reshape(-1, 5)
    b = b.reshape(-1, 5)
    den = np.abs(b).sum(axis=0)
    return np.abs(a - b).sum(axis=0) / np.where(den > 0, den, 1.0)
