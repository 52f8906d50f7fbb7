"""Diagnostics of the resident state: the reference's mass monitor (grhd2.f90:283-301),
accretion rate (output.f90:951-992), PPI azimuthal modes (output.f90:995-1049) and global
diagnostics (output.f90:1052-1125).

CPU: the oracle's serial restatement agrees with an independent numpy formulation.
GPU: the device reductions agree with the oracle -- per-cell terms are the reference's
arithmetic, sums differ only by summation order (relative 1e-12), extrema and counts are
exact; the mixed policy agrees within its stated 1e-5."""
import numpy as np
import pytest

from oracle.binding import OracleRun
from tests.helpers import initial_state, interior, michel, torus_2p5d, torus_3d

CASES = [(torus_3d, dict(nx=24, ny=12, nz=12), 3), (torus_2p5d, dict(nx=64, nz=32), 5), (michel, dict(nx=128), 40)]
SUM_KEYS = ("mass_total", "disk_mass", "angular_momentum")
EXACT_KEYS = ("rho_min", "p_min", "rho_max", "p_max", "max_v_sq", "atmosphere_cells", "invalid_cells")


def oracle_state(maker, kw, steps):
    pb = maker(**kw)
    o = OracleRun(pb, initial_state(pb))
    o.prim_to_cons()
    o.set_boundary()
    o.run(0.0, 1e30, steps - 1)
    u = o.up.copy()  # u of the last step: the state at its start
    o.run(0.0, 1e30, 1)
    return pb, o, u


def z_centres(pb):
    return pb.coords()[2][pb.ng + 1:pb.ng + 1 + pb.nz]


@pytest.mark.parametrize("maker,kw,steps", CASES)
def test_oracle_diagnostics_match_numpy(maker, kw, steps):
    pb, o, u = oracle_state(maker, kw, steps)
    cfg = o.cfg
    vol = cfg.dx * cfg.dy * cfg.dz
    up = o.up.reshape(pb.nz, pb.ny, pb.nx, 5)
    p = interior(pb, o.p)
    g = np.ctypeslib.as_array(pb.metric_view().gamma_c, shape=(pb.ny, pb.nx, 3, 3))  # Fortran (3,3,nx,ny)
    v = p[..., 2:5]
    vsq = np.einsum("jiba,kjia,kjib->kji", g, v, v)
    d = o.global_diagnostics()
    cut = 1e3 * cfg.rho_floor
    assert np.isclose(d["mass_total"], (up[..., 0] * vol).sum(), rtol=1e-12, atol=0)
    assert np.isclose(d["disk_mass"], (up[..., 0] * vol)[p[..., 0] > cut].sum(), rtol=1e-12, atol=0)
    assert np.isclose(d["angular_momentum"], (up[..., 4] * vol).sum(), rtol=1e-12, atol=1e-300)
    assert d["rho_min"] == p[..., 0].min() and d["p_max"] == p[..., 1].max()
    assert np.isclose(d["max_v_sq"], vsq.max(), rtol=1e-14)
    assert d["atmosphere_cells"] == int((p[..., 0] <= cut).sum())
    assert np.isclose(o.total_mass(u), (u.reshape(-1, 5)[:, 0] * cfg.dx * cfg.dy * cfg.dz).sum(), rtol=1e-12)
    vals = o.ppi_modes(z_centres(pb))
    if pb.nz >= 2:
        am = np.where(p[..., 0] > cut, up[..., 0] * vol, 0.0).sum(axis=(1, 2))
        m = np.arange(1, 5)[:, None]
        z = z_centres(pb)[None, :]
        cr, ci = (am * np.cos(m * z)).sum(1), -(am * np.sin(m * z)).sum(1)
        assert np.isclose(vals[0], am.sum(), rtol=1e-12)
        assert np.allclose(vals[1::4], cr, rtol=1e-10, atol=1e-12 * am.sum())
        assert np.allclose(vals[2::4], ci, rtol=1e-10, atol=1e-12 * am.sum())
    else:
        assert np.all(vals == 0.0)
    idx = pb.accretion_probe()
    if idx >= 1:
        a = np.ctypeslib.as_array(pb.metric_view().alpha_c, shape=(pb.ny, pb.nx))[:, idx - 1]
        b1 = np.ctypeslib.as_array(pb.metric_view().beta_c, shape=(pb.ny, pb.nx, 3))[:, idx - 1, 0]
        veff = a[None, :] * p[:, :, idx - 1, 2] - b1[None, :]
        ref = -(up[:, :, idx - 1, 0] * veff * cfg.dy * cfg.dz).sum()
        assert np.isclose(o.mdot(idx), ref, rtol=1e-12, atol=1e-300)


@pytest.mark.gpu
@pytest.mark.parametrize("precision", ["fp64", "mixed"])
@pytest.mark.parametrize("maker,kw,steps", CASES)
def test_gpu_diagnostics_match_oracle(maker, kw, steps, precision):
    from grhd_b200.solver import GpuError, GpuGrid
    pb, o, u = oracle_state(maker, kw, steps)
    g = GpuGrid(pb, precision=precision, upload_initial=False)
    g.upload(p=initial_state(pb))
    g.prim_to_cons()
    with pytest.raises(GpuError):
        g.total_mass()  # no step yet: u is not defined
    g.run(0.0, 1e30, steps)
    rtol = 1e-12 if precision == "fp64" else 1e-5
    d, r = g.global_diagnostics(), o.global_diagnostics()
    for k in SUM_KEYS:
        assert np.isclose(d[k], r[k], rtol=rtol, atol=0), (k, d[k], r[k])
    if precision == "fp64":
        for k in EXACT_KEYS:
            assert d[k] == r[k], (k, d[k], r[k])
    assert np.isclose(g.total_mass(), o.total_mass(u), rtol=rtol, atol=0)
    vg, vo = g.ppi_modes(), o.ppi_modes(z_centres(pb))
    scale = max(abs(vo[0]), 1e-300)
    assert np.allclose(vg[[0, 1, 2, 5, 6, 9, 10, 13, 14]], vo[[0, 1, 2, 5, 6, 9, 10, 13, 14]], rtol=0,
                       atol=rtol * scale)
    idx = pb.accretion_probe()
    if idx >= 1:
        mg, mo = g.mdot(idx), o.mdot(idx)
        assert np.isclose(mg, mo, rtol=rtol * (1 if precision == "fp64" else 10), atol=1e-30), (mg, mo)
        with pytest.raises(GpuError):
            g.mdot(pb.nx + 1)
    g.close()


def numpy_gw(pb, o, spin):
    """calc_gw_strain (output.f90:852-948) vectorised: Ixx, Iyy, Ixy."""
    cfg = o.cfg
    g = pb.ng
    x, y, z = (a[g + 1:g + 1 + n] for a, n in zip(pb.coords(), (pb.nx, pb.ny, pb.nz)))
    log_r = bool(pb.config(0).use_log_r)
    r = (np.exp(x) if log_r else x)[None, None, :]
    m_bh = pb.info.bh_mass
    r_h = m_bh + np.sqrt(max(0.0, m_bh * m_bh - spin * spin))
    q = interior(pb, o.p)
    rho = np.maximum(q[..., 0] - cfg.rho_floor, 0.0)
    pres = np.maximum(q[..., 1] - cfg.p_floor, 0.0)
    mv = pb.metric_view()
    alpha = np.ctypeslib.as_array(mv.alpha_c, shape=(pb.ny, pb.nx))[None]
    beta = np.ctypeslib.as_array(mv.beta_c, shape=(pb.ny, pb.nx, 3))[None]
    rates = alpha[..., None] * q[..., 2:5] - beta
    if log_r:
        rates[..., 0] = r * rates[..., 0]
    st, ct = np.sin(y)[None, :, None], np.cos(y)[None, :, None]
    sp, cp = np.sin(z)[:, None, None], np.cos(z)[:, None, None]
    pole = np.abs(st) <= 64 * np.finfo(float).eps
    pos0 = np.where(pole, 0.0, (r * cp - spin * sp) * st)
    pos1 = np.where(pole, 0.0, (r * sp + spin * cp) * st)
    pos2 = np.where(pole, np.copysign(np.abs(r), ct), r * ct)
    v0 = rates[..., 0] * cp * st + rates[..., 1] * (r * cp - spin * sp) * ct - rates[..., 2] * (r * sp + spin * cp) * st
    v1 = rates[..., 0] * sp * st + rates[..., 1] * (r * sp + spin * cp) * ct + rates[..., 2] * (r * cp - spin * sp) * st
    dV = (r * r + spin * spin * ct * ct) * st * (r if log_r else 1.0) * cfg.dx * cfg.dy * cfg.dz
    r2 = pos0 ** 2 + pos1 ** 2 + pos2 ** 2
    mr3 = m_bh / (r2 * np.sqrt(r2))
    keep = (r > r_h) & ~((rho <= 0) & (pres <= 0))
    ixx = ((2 * rho * v0 ** 2 + 2 * pres - 2 * rho * mr3 * pos0 ** 2) * dV)[keep].sum()
    iyy = ((2 * rho * v1 ** 2 + 2 * pres - 2 * rho * mr3 * pos1 ** 2) * dV)[keep].sum()
    ixy = ((2 * rho * v0 * v1 - 2 * rho * mr3 * pos0 * pos1) * dV)[keep].sum()
    return np.array([ixx, iyy, ixy])


GW_CASES = [(torus_3d, dict(nx=24, ny=12, nz=12), 3), (torus_2p5d, dict(nx=64, nz=32), 5), (michel, dict(nx=128), 20)]


def _spin(pb):
    return pb.info.a_spin if pb.config(0).metric_kind == 2 else 0.0


@pytest.mark.parametrize("maker,kw,steps", GW_CASES)
def test_oracle_gw_matches_numpy(maker, kw, steps):
    pb, o, _ = oracle_state(maker, kw, steps)
    spin = _spin(pb)
    got = o.gw_strain(bool(pb.config(0).use_log_r), pb.info.bh_mass, spin)
    want = numpy_gw(pb, o, spin)
    scale = np.abs(want).max()
    assert scale > 0 and np.allclose(got[2:], want, rtol=0, atol=1e-10 * scale)
    assert got[0] == (got[2] - got[3]) / 1000.0 and got[1] == 2.0 * got[4] / 1000.0


@pytest.mark.gpu
@pytest.mark.parametrize("precision", ["fp64", "mixed"])
@pytest.mark.parametrize("maker,kw,steps", GW_CASES)
def test_gpu_gw_matches_oracle(maker, kw, steps, precision):
    from grhd_b200.solver import GpuGrid
    pb, o, _ = oracle_state(maker, kw, steps)
    g = GpuGrid(pb, precision=precision, upload_initial=False)
    g.upload(p=initial_state(pb))
    g.prim_to_cons()
    g.run(0.0, 1e30, steps)
    got = g.gw_strain()
    want = o.gw_strain(bool(pb.config(0).use_log_r), pb.info.bh_mass, _spin(pb))
    scale = np.abs(want[2:]).max()
    tol = 1e-12 if precision == "fp64" else 1e-5
    assert np.allclose(got[2:], want[2:], rtol=0, atol=tol * scale), (got, want)
    g.close()
