"""Parity of the sm_100a path (through the C-ABI) with the CPU oracle.

The oracle restates the reference's arithmetic in its own operation order without FMA
contraction; the FP64 kernels do the same, so the FP64 results agree to round-off.  The
parity bar is a relative L1 of at most 1e-12 per conserved variable with identical
con2prim failure/floor counts; most cases here are bit-identical.
"""
import numpy as np
import pytest

from grhd_b200.solver import GpuGrid
from oracle.binding import OracleRun
from tests.helpers import (face_ghost_mask, initial_state, interior, michel, rel_l1, shock_tube, shock_tube_xy,
                           torus_2p5d, torus_3d)

pytestmark = pytest.mark.gpu

L1_TOL = 1e-12  # relative L1 per conserved variable, FP64 path


def run_pair(pb, nsteps=None, final_time=None, precision="fp64"):
    p0 = initial_state(pb)
    o = OracleRun(pb, p0)
    o.prim_to_cons()
    o.set_boundary()
    g = GpuGrid(pb, precision=precision, upload_initial=False)
    g.upload(p=p0)
    g.prim_to_cons()
    tf = final_time if final_time is not None else 1e30
    ms = -1 if nsteps is None else nsteps
    n_o, t_o = o.run(0.0, tf, ms)
    n_g, t_g = g.run(0.0, tf, ms)
    assert n_o == n_g and t_o == t_g
    up_g, p_g = g.download(p_template=o.p)
    return o, g, up_g, p_g


def assert_parity(pb, o, g, up_g, p_g, tol=L1_TOL):
    l1 = rel_l1(up_g, o.up)
    assert np.all(l1 <= tol), f"relative L1 per variable {l1}"
    mask = face_ghost_mask(pb)
    dp = np.abs(p_g - o.p)[mask]
    scale = np.abs(o.p)[mask].max()
    assert dp.max() <= 1e-9 * scale, f"primitive max diff {dp.max()}"
    co, cg = o.counters.as_dict(), g.counters()
    for k in ("c2p_floor_pre", "c2p_causal_rescale", "c2p_brent_used", "c2p_root_fail", "c2p_bad_V",
              "c2p_final_sanitise"):
        assert co[k] == cg[k], f"counter {k}: oracle {co[k]} gpu {cg[k]}"
    return l1


def test_shock_tube_full_run():
    """400-cell relativistic blast wave, WENO5 + HLLE, SSP-RK3, CFL 0.4 to t = 0.4 (400 steps)."""
    pb = shock_tube()
    o, g, up, p = run_pair(pb, final_time=0.4)
    assert_parity(pb, o, g, up, p)
    assert np.array_equal(up, o.up), "FP64 shock tube is expected to be bit-identical"


@pytest.mark.parametrize("rec,rs,sensor,lim", [
    ("godunov", "hlle", False, "mc"), ("tvd", "hlle", False, "minmod"), ("tvd", "hllc", False, "superbee"),
    ("tvd", "hlle", True, "mc"), ("weno3", "hllc", False, "mc"), ("weno3", "hlle", True, "mc"),
    ("mp5", "hlle", False, "mc"), ("mp5", "hllc", True, "mc"), ("weno5", "hllc", False, "mc"),
    ("weno5", "hlle", True, "mc")])
def test_shock_tube_schemes(rec, rs, sensor, lim):
    pb = shock_tube(nx=200, rec=rec, rs=rs, sensor=sensor, tvd_limiter=lim, sod_velocity_left=0.3,
                    sod_velocity_right=-0.2)
    o, g, up, p = run_pair(pb, nsteps=60)
    assert_parity(pb, o, g, up, p)


@pytest.mark.parametrize("maker,kw", [
    (torus_2p5d, dict(nx=96, nz=48)),
    (torus_2p5d, dict(nx=96, nz=48, rec="mp5", rs="hllc", sensor=True)),
    (torus_3d, dict(nx=40, ny=24, nz=24)),
    (torus_3d, dict(nx=40, ny=24, nz=24, rec="weno5", rs="hlle", sensor=False)),
    (michel, dict(nx=256)),
    (michel, dict(nx=256, rec="weno3", rs="hllc", sensor=True)),
])
def test_rhs_parity(maker, kw):
    """calc_rhs of the same perturbed state through the C-ABI and the oracle."""
    pb = maker(**kw)
    p0 = initial_state(pb)
    o = OracleRun(pb, p0)
    o.set_boundary()
    r_o = o.calc_rhs()
    g = GpuGrid(pb, upload_initial=False)
    g.upload(p=p0)
    r_g = g.calc_rhs()
    # WENO3 calls exp(); CUDA's and the host libm's differ by up to 1 ulp, and the flux
    # difference -(F_i - F_{i-1})/dx amplifies that in the pointwise RHS.  The bar is the
    # parity norm (relative L1 per variable); the pointwise maximum gets a loose bound.
    l1 = rel_l1(r_g, r_o)
    assert np.all(l1 <= 1e-12), f"rhs relative L1 per variable {l1}"
    scale = np.abs(r_o).reshape(-1, 5).max(axis=0)
    err = np.abs(r_g - r_o).reshape(-1, 5).max(axis=0) / np.where(scale > 0, scale, 1)
    assert np.all(err <= 1e-9), f"rhs relative max error per variable {err}"
    assert g.counters()["hllc_fallbacks"] == o.counters.as_dict()["hllc_fallbacks"]
    assert g.counters()["recon_floor_clamps"] == o.counters.as_dict()["recon_floor_clamps"]


@pytest.mark.parametrize("maker,kw", [
    (torus_3d, dict(nx=40, ny=24, nz=24)),
    (michel, dict(nx=256, rec="weno3", rs="hllc", sensor=True)),
])
def test_rhs_against_libm_exp_oracle(maker, kw):
    """Against the oracle variant that calls the C library's exp in WENO3, as the reference
    build does: the RHS stays within the relative-L1 bar (the exp choice is sub-ulp noise)."""
    pb = maker(**kw)
    p0 = initial_state(pb)
    o = OracleRun(pb, p0, libm_exp=True)
    o.set_boundary()
    r_o = o.calc_rhs()
    g = GpuGrid(pb, upload_initial=False)
    g.upload(p=p0)
    r_g = g.calc_rhs()
    l1 = rel_l1(r_g, r_o)
    assert np.all(l1 <= 1e-12), f"rhs relative L1 per variable {l1}"


def test_michel_run():
    """Michel accretion, MP5 + HLLE, 1024 log-spaced cells, 300 steps."""
    pb = michel()
    o, g, up, p = run_pair(pb, nsteps=300)
    assert_parity(pb, o, g, up, p)


def test_torus_2p5d_run():
    """Equatorial KS torus, WENO5 + HLLE, 200 x 1 x 100, 40 steps."""
    pb = torus_2p5d(nx=200, nz=100)
    o, g, up, p = run_pair(pb, nsteps=40)
    assert_parity(pb, o, g, up, p)


def test_xy_grid_run():
    """A grid with a y extent and no k extent (nz = 1): x-y block tiles, y faces without k
    rows, the cell update reading the metric table from global memory (its shared-memory
    slice needs a k extent).  Shock tube 96 x 24 with 5 % pressure noise, MP5 + HLLC, 30
    steps."""
    pb = shock_tube_xy()
    o, g, up, p = run_pair(pb, nsteps=30)
    assert_parity(pb, o, g, up, p)


def test_torus_3d_run():
    """3D KS torus, MP5 + HLLC + shock sensor, trans-polar boundaries, 48 x 24 x 24, 12 steps."""
    pb = torus_3d(nx=48, ny=24, nz=24)
    o, g, up, p = run_pair(pb, nsteps=12)
    assert_parity(pb, o, g, up, p)


def test_cons_to_prim_injected_failures():
    """Floors and failure branches of cons_to_prim on injected bad states (NaN, negative D,
    superluminal momentum, tiny D): identical categories and counts."""
    pb = torus_2p5d(nx=64, nz=32)
    p0 = initial_state(pb)
    o = OracleRun(pb, p0)
    o.prim_to_cons()
    up = o.up.copy()
    rng = np.random.default_rng(7)
    flat = up.reshape(-1, 5)
    idx = rng.choice(flat.shape[0], size=400, replace=False)
    flat[idx[:80], 0] = np.nan
    flat[idx[80:160], 0] = -1.0
    flat[idx[160:240], 2:5] *= 1e3           # superluminal S
    flat[idx[240:320], 0] = 1e-14            # below the D floor
    flat[idx[320:400], 1] = -5 * flat[idx[320:400], 0]  # negative total energy
    o.up = up.copy()
    o.cons_to_prim()
    g = GpuGrid(pb, upload_initial=False)
    g.upload(up=up, p=p0)
    g.cons_to_prim()
    up_g, p_g = g.download(p_template=o.p)
    co, cg = o.counters.as_dict(), g.counters()
    for k in co:
        assert co[k] == cg[k], f"{k}: oracle {co[k]} gpu {cg[k]}"
    assert np.array_equal(np.nan_to_num(up_g), np.nan_to_num(o.up))
    assert np.array_equal(interior(pb, p_g), interior(pb, o.p))


def test_download_ghosts_match_reference_fill():
    """Single-direction ghosts of the downloaded primitives equal set_boundary_conditions."""
    pb = torus_3d(nx=24, ny=16, nz=16)
    p0 = initial_state(pb)
    o = OracleRun(pb, p0)
    o.set_boundary()
    g = GpuGrid(pb, upload_initial=False)
    g.upload(p=p0)
    # index -nghost is never written by the boundary routine: it keeps the caller's value
    _, p_g = g.download(p_template=p0, want_up=False)
    mask = face_ghost_mask(pb)
    assert np.array_equal(p_g[mask], o.p[mask])


def test_cfl_matches_oracle():
    for pb in (shock_tube(), michel(nx=256), torus_2p5d(nx=64, nz=32), torus_3d(nx=24, ny=16, nz=16)):
        o = OracleRun(pb)
        g = GpuGrid(pb)
        assert g.cfl() == o.cfl()


# Relative L1 per conserved variable (D, tau, S_1, S_2, S_3), each in its own norm, that
# the mixed policies must meet against the FP64 oracle after the steps of each case.  The
# stated bar is 1e-5 on the 2.5D torus.  Measured (all three mixed policies agree to three
# digits): 2.5D torus 2.0e-8 .. 3.7e-8; 3D torus (MP5 + HLLC) ~1e-7 for D, tau, S_r and
# S_phi; Michel 2.9e-7 .. 3.7e-7; shock tube 2.2e-7 .. 9.8e-7.  S_theta of the 3D torus is
# ~0 by symmetry, so its own norm is tiny and its relative error large although its
# absolute error is that of the other momenta (2.3e-5 after 500 steps at 256x128x128);
# its bound is 1e-3.
MIXED_L1_BOUND = {
    "torus_2p5d": [1e-5] * 5,
    "torus_3d": [1e-5, 1e-5, 1e-5, 1e-3, 1e-5],
    "michel": [1e-5] * 5,
    "shock_tube": [1e-5] * 5,
}


@pytest.mark.parametrize("precision", ["mixed", "mixed_comp64", "mixed_comp32"])
@pytest.mark.parametrize("name,maker,kw,steps", [
    ("torus_2p5d", torus_2p5d, dict(nx=128, nz=64), 60),
    ("torus_3d", torus_3d, dict(nx=32, ny=16, nz=16), 10),
    ("michel", michel, dict(nx=512), 200),
    ("shock_tube", shock_tube, dict(nx=400), 200),
])
def test_mixed_policy_l1(name, maker, kw, steps, precision):
    """Mixed policies (FP32 reconstruction, Riemann fluxes and metric contraction; FP64
    lapse and sqrt(gamma) factors, con2prim with the seeded root finder and RK state, the
    RK accumulation plain or compensated with an FP64 or FP32 carry) against the FP64
    oracle after the same steps: relative L1 per conserved variable, each in its own norm,
    within MIXED_L1_BOUND."""
    pb = maker(**kw)
    o, g, up, p = run_pair(pb, nsteps=steps, precision=precision)
    l1 = rel_l1(up, o.up)
    assert np.all(l1 <= np.array(MIXED_L1_BOUND[name])), f"{precision} relative L1 per variable {l1}"


def test_async_upload_download_match_sync():
    """grhd2_gpu_upload_async / grhd2_gpu_download_async move the same bytes as the
    synchronous calls once the stream is synchronised (page-locked and ordinary buffers)."""
    from grhd_b200 import native as N
    pb = torus_2p5d(nx=48, nz=24)
    p0 = initial_state(pb)
    g = GpuGrid(pb, upload_initial=False)
    g.upload(p=p0)
    g.prim_to_cons()
    g.run(0.0, 1e30, 3)
    up_sync, p_sync = g.download(p_template=p0)
    lib = g.lib
    up_a = np.empty(pb.cons_shape)
    p_a = np.array(p0)
    assert lib.grhd2_gpu_download_async(g._h, N.dptr(up_a), N.dptr(p_a)) == 0
    g.synchronize()
    assert np.array_equal(up_a, up_sync) and np.array_equal(p_a, p_sync)
    # round trip: upload the state asynchronously into a fresh grid and read it back
    h = GpuGrid(pb, upload_initial=False)
    assert lib.grhd2_gpu_upload_async(h._h, N.dptr(up_a), N.dptr(p_a)) == 0
    h.synchronize()
    up_b, p_b = h.download(p_template=p0)
    assert np.array_equal(up_b, up_sync) and np.array_equal(p_b, p_sync)
    g.close()
    h.close()


@pytest.mark.parametrize("precision", ["mixed_comp64", "mixed_comp32"])
def test_compensated_accumulation_carries(precision):
    """The compensated policies keep a carry beside u and up: after the same steps their
    state differs from the plain mixed policy's in the last bits (the rounding the FP64
    combination drops is carried, not lost), and the carries restart at zero when up is
    uploaded -- a grid that re-uploads its own downloaded state continues exactly as a
    fresh grid started from that state."""
    pb = torus_2p5d(nx=64, nz=32)
    p0 = initial_state(pb)
    runs = {}
    for prec in ("mixed", precision):
        g = GpuGrid(pb, precision=prec, upload_initial=False)
        g.upload(p=p0)
        g.prim_to_cons()
        g.run(0.0, 1e30, 20)
        runs[prec] = g
    up_m, _ = runs["mixed"].download(want_p=False)
    up_c, p_c = runs[precision].download(p_template=p0)
    assert not np.array_equal(up_m, up_c), "the carries change nothing"
    # a last-bit correction, which the FP32 fluxes amplify to ~3e-12 over these steps: far
    # below the mixed policy's own error against FP64 (~1e-8 here)
    assert np.all(rel_l1(up_c, up_m) <= 1e-9)
    a = runs[precision]
    a.upload(up=up_c, p=p_c)  # the carries restart at zero
    a.run(0.0, 1e30, 7)
    b = GpuGrid(pb, precision=precision, upload_initial=False)
    b.upload(up=up_c, p=p_c)
    b.run(0.0, 1e30, 7)
    assert np.array_equal(a.download(want_p=False)[0], b.download(want_p=False)[0])
    for g in (*runs.values(), b):
        g.close()
