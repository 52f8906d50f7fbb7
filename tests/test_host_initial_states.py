"""The host set-up's initial states against set_initial_conditions (conditions.f90:26-214)
restated here in plain Python for the presets the other set-up tests leave out: Sod,
strong shock, Shu-Osher, Kelvin-Helmholtz, jet, convergence wave, dust and the off-axis
blast (the Fishbone-Moncrief tori and Michel have tests of their own).

p starts at zero and each case writes exactly the cells the reference writes -- the 1D
shock tubes every ghost layer, the Kelvin-Helmholtz and jet states the interior only, the
convergence wave its density inside and velocity and pressure everywhere, the dust state
from x(1) outwards with the inner ghosts copied from cell 1, the off-axis blast every i
and k but only the interior j -- so the arrays must agree to the bit, ghosts included.
"""
import math

import numpy as np
import pytest

from grhd_b200 import native as N
from grhd_b200.problem import Problem

PI = math.pi
DE, PR, VX, VY, VZ = 0, 1, 2, 3, 4


def initial_state(pb, keys):
    nx, ny, nz, g = pb.nx, pb.ny, pb.nz, pb.ng
    x, _, z = pb.coords()
    p = np.zeros(pb.prim_shape)
    X = lambda i: x[i + g]
    Z = lambda k: z[k + g]
    P = lambda i, j, k: p[k + g, j + g, i + g]
    case = pb.info.case_id
    allr = range(-g, nx + g + 1)
    if case in (1, 2, 3):
        pre = {1: "sod", 2: "strong", 3: "shu"}[case]
        for i in allr:
            if X(i) < keys[pre + "_interface"]:
                rho, pr = keys[pre + "_density_left"], keys[pre + "_pressure_left"]
            elif case == 3:
                rho = keys["shu_density_right"] + keys["shu_density_amplitude"] * math.sin(keys["shu_wave_number"] * X(i))
                pr = keys["shu_pressure_right"]
            else:
                rho, pr = keys[pre + "_density_right"], keys[pre + "_pressure_right"]
            p[:, :, i + g, DE] = rho
            p[:, :, i + g, PR] = pr
    elif case == 4:
        for k in range(1, nz + 1):
            for j in range(1, ny + 1):
                for i in range(1, nx + 1):
                    c = P(i, j, k)
                    inner = abs(Z(k)) < keys["khi_half_width"]
                    c[DE] = keys["khi_density_inner"] if inner else keys["khi_density_outer"]
                    c[VX] = keys["khi_velocity_inner"] if inner else keys["khi_velocity_outer"]
                    c[PR] = keys["khi_pressure"]
                    c[VY] = 0.0
                    d = abs(abs(Z(k)) - keys["khi_half_width"])
                    t = d / keys["khi_perturbation_width"]
                    env = math.exp(-0.5 * (t * t))
                    c[VZ] = keys["khi_perturbation_amplitude"] * math.sin(keys["khi_perturbation_wave_number"] * PI * X(i)) * env
    elif case == 5:
        for k in range(1, nz + 1):
            for j in range(1, ny + 1):
                for i in range(1, nx + 1):
                    c = P(i, j, k)
                    c[DE], c[PR], c[VZ] = keys["jet_ambient_density"], keys["jet_ambient_pressure"], keys["jet_ambient_velocity"]
                    if X(i) <= keys["jet_nozzle_radius"] and Z(k) <= keys["jet_nozzle_length"]:
                        c[DE], c[PR], c[VZ] = keys["jet_density"], keys["jet_pressure"], keys["jet_velocity"]
    elif case == 6:
        kw = keys["convergence_wave_number"]
        arg = 0.5 * kw * PI * pb.config(0).dx
        sinc = math.sin(arg) / arg if abs(arg) > np.finfo(float).eps else 1.0
        for i in range(1, nx + 1):
            p[:, :, i + g, DE] = keys["convergence_density"] + keys["convergence_amplitude"] * sinc * math.sin(kw * PI * X(i))
        p[..., VX] = keys["convergence_velocity"]
        p[..., PR] = keys["convergence_pressure"]
    elif case == 8:
        cfg = pb.config(0)
        for i in range(1, nx + g + 1):  # evaluate_dust_accretion_state through the host probe
            s = np.zeros(5)
            assert N.host_lib().grhd2_host_dust_state(cfg.use_log_r, pb.info.bh_mass, keys["dust_accretion_constant"],
                                                      cfg.p_floor, X(i), N.dptr(s)) == 0
            p[:, :, i + g, :] = s
        for i in range(-g, 1):
            p[:, :, i + g, :] = p[:, :, 1 + g, :]
    elif case == 9:
        log_r = bool(pb.config(0).use_log_r)
        rc, phic, w = keys["offaxis_radial_center"], keys["offaxis_phi_center"] * PI, keys["offaxis_width"]
        for k in range(-g, nz + g + 1):
            for j in range(1, ny + 1):
                for i in allr:
                    r = math.exp(X(i)) if log_r else X(i)
                    d2 = r * r + rc * rc - 2.0 * rc * r * math.cos(Z(k) - phic)
                    e = -d2 / (w * w)
                    gp = 0.0 if e < -40.0 else math.exp(e)
                    c = P(i, j, k)
                    c[DE] = keys["offaxis_background_density"] + keys["offaxis_density_amplitude"] * gp
                    c[PR] = keys["offaxis_background_pressure"] + keys["offaxis_pressure_amplitude"] * gp
    return p


CASES = [
    ("sod", dict(nx=40, ny=3, nz=2, sod_interface=0.37, sod_density_left=10.0, sod_density_right=1.0,
                 sod_pressure_left=13.3, sod_pressure_right=1e-6)),
    ("strong_shock", dict(nx=40, strong_interface=0.5, strong_density_left=1.0, strong_density_right=1.0,
                          strong_pressure_left=1000.0, strong_pressure_right=0.01)),
    ("shu_osher", dict(nx=64, shu_interface=0.2, shu_density_left=5.0, shu_pressure_left=50.0,
                       shu_density_right=2.0, shu_density_amplitude=0.3, shu_wave_number=50.0,
                       shu_pressure_right=5.0)),
    ("khi", dict(nx=16, ny=1, nz=12, khi_half_width=0.25, khi_density_inner=2.0, khi_density_outer=1.0,
                 khi_velocity_inner=0.5, khi_velocity_outer=-0.5, khi_pressure=2.5, khi_perturbation_amplitude=0.01,
                 khi_perturbation_wave_number=10.0, khi_perturbation_width=0.05)),
    ("axisymmetric_jet", dict(nx=16, ny=1, nz=20, jet_ambient_density=10.0, jet_ambient_pressure=0.01,
                              jet_ambient_velocity=0.0, jet_nozzle_radius=0.1, jet_nozzle_length=0.2,
                              jet_density=1.0, jet_pressure=0.01, jet_velocity=0.99)),
    ("convergence", dict(nx=48, convergence_density=1.0, convergence_amplitude=0.1, convergence_velocity=0.5,
                         convergence_pressure=1.0, convergence_wave_number=2.0)),
    ("dust", dict(nx=32, dust_accretion_constant=-0.5)),
    ("offaxis_blast", dict(nx=24, ny=1, nz=16, offaxis_radial_center=15.0, offaxis_phi_center=1.0,
                           offaxis_width=1.5, offaxis_background_density=0.1, offaxis_background_pressure=0.1,
                           offaxis_density_amplitude=1.0, offaxis_pressure_amplitude=1.0)),
]


@pytest.mark.parametrize("name,keys", CASES, ids=[c[0] for c in CASES])
def test_initial_state_matches_an_independent_restatement(name, keys):
    pb = Problem.from_keys(name, perturbation="none", **keys)
    got = pb.initial_prims()
    want = initial_state(pb, keys)
    assert got.tobytes() == want.tobytes(), np.argwhere(got != want)[:5]
