"""The host set-up's perturbations against inject_pressure_noise, inject_density_noise and
inject_density_mode (conditions.f90:603-768) restated here in plain Python.

gfortran's random_number stream cannot be reproduced outside gfortran, so the host set-up
draws from SplitMix64 (Steele, Lea and Flood 2014) seeded with perturbation_seed -- a
documented deviation; everything else must be the reference's: the density maximum over
the interior before any change, the selection rho > 0.05 rho_max, the loop order (i
fastest, one draw per selected cell), u in [0, 1) mapped to 2u - 1, pressure scaled by
1 + A r, density by the same factor with pressure by factor**Gamma (isentropic), and the
coherent mode's 1 + A cos(m phi).  Bit for bit, on a torus (its atmosphere is skipped)
and a shock tube (every cell selected), for each of the three kinds.
"""
import math

import numpy as np
import pytest

from tests.helpers import shock_tube, torus_2p5d, torus_3d

MASK = (1 << 64) - 1


class SplitMix64:
    def __init__(self, seed):
        self.s = seed & MASK

    def uniform(self):
        self.s = (self.s + 0x9E3779B97F4A7C15) & MASK
        z = self.s
        z = ((z ^ (z >> 30)) * 0xBF58476D1CE4E5B9) & MASK
        z = ((z ^ (z >> 27)) * 0x94D049BB133111EB) & MASK
        z = z ^ (z >> 31)
        return (z >> 11) * (1.0 / 9007199254740992.0)


def perturb(p, pb, kind, amp, seed, mode, adb):
    g = pb.ng
    interior = p[g + 1:g + 1 + pb.nz, g + 1:g + 1 + pb.ny, g + 1:g + 1 + pb.nx, :]
    rho_max = float(interior[..., 0].max())
    _, _, z = pb.coords()
    rng = SplitMix64(seed)
    for k in range(pb.nz):
        phi = z[k + 1 + g]
        for j in range(pb.ny):
            for i in range(pb.nx):
                c = interior[k, j, i]
                if not c[0] > 0.05 * rho_max:
                    continue
                if kind == 1:
                    r = 2.0 * rng.uniform() - 1.0
                    c[1] = c[1] * (1.0 + amp * r)
                elif kind == 2:
                    r = 2.0 * rng.uniform() - 1.0
                    f = 1.0 + amp * r
                    c[0] = c[0] * f
                    c[1] = c[1] * math.pow(f, adb)
                else:
                    f = 1.0 + amp * math.cos(mode * phi)
                    c[0] = c[0] * f
                    c[1] = c[1] * math.pow(f, adb)


KINDS = {"pressure_noise": 1, "density_noise": 2, "density_mode": 3}


@pytest.mark.parametrize("kind", list(KINDS))
@pytest.mark.parametrize("maker,kw", [(torus_2p5d, dict(nx=32, nz=16)), (torus_3d, dict(nx=12, ny=8, nz=8)),
                                      (shock_tube, dict(nx=64))])
def test_perturbations_match_an_independent_restatement(kind, maker, kw):
    amp, seed, mode = 0.037, 987654321, 3.0
    pb = maker(perturbation=kind, perturbation_amplitude=amp, perturbation_seed=seed, perturbation_mode=mode,
               perturbation_time=0.0, **kw)
    assert pb.info.perturbation_type == KINDS[kind]
    p0 = pb.initial_prims().copy()
    got = pb.perturb(p0.copy())
    want = p0.copy()
    perturb(want, pb, KINDS[kind], amp, seed, mode, pb.config(0).adb_idx)
    assert got.tobytes() == want.tobytes()
    assert not np.array_equal(got, p0)


@pytest.mark.parametrize("amp", [-0.1, 1.0])
def test_perturbation_amplitude_outside_the_reference_range_is_refused(amp):
    """inject_pressure_noise and inject_density_noise stop on A < 0 or A >= 1; the host
    set-up refuses the problem or the perturbation."""
    with pytest.raises(ValueError):
        pb = shock_tube(nx=16, perturbation="pressure_noise", perturbation_amplitude=amp, perturbation_time=0.0)
        pb.perturb(pb.initial_prims().copy())
