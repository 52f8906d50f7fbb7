"""The allocation-free face-flux entry point (grhd2_gpu_riemann_faces_noalloc) against
the allocating one (grhd2_gpu_riemann_faces): same inputs, same fluxes, on two calls in a
row, with the scratch reused between calls of different sizes.  The file is named so that
it is collected last; it builds its own grids and passes alone or after the other tests.
"""
import numpy as np
import pytest

from grhd_b200.solver import GpuError, GpuGrid
from tests.helpers import shock_tube, torus_2p5d

pytestmark = pytest.mark.gpu

MAX_FACES = 16384  # GRHD2_GPU_NOALLOC_MAX_FACES
RTOL = 1e-13       # both entry points run the same kernel: equal to round-off (in practice bitwise)


def random_faces(rng, n, general_metric):
    qL = np.column_stack([10 ** rng.uniform(-3, 1, n), 10 ** rng.uniform(-4, 2, n), rng.uniform(-0.5, 0.5, (n, 3))])
    qR = np.column_stack([10 ** rng.uniform(-3, 1, n), 10 ** rng.uniform(-4, 2, n), rng.uniform(-0.5, 0.5, (n, 3))])
    if not general_metric:
        return qL, qR, np.ones(n), np.zeros((n, 3)), np.broadcast_to(np.eye(3), (n, 3, 3)).copy(), np.ones(n)
    a = rng.uniform(-0.3, 0.3, (n, 3, 3))
    g = np.eye(3)[None] * rng.uniform(0.8, 3.0, (n, 1, 1)) + np.einsum("nij,nkj->nik", a, a)
    g = 0.5 * (g + g.transpose(0, 2, 1))  # exactly symmetric
    alpha = rng.uniform(0.3, 1.0, n)
    beta = rng.uniform(-0.3, 0.3, (n, 3))
    sqg = np.sqrt(np.linalg.det(g))
    return qL, qR, alpha, beta, g, sqg


def check_pair(G, rng, n, general_metric):
    qL, qR, alpha, beta, g, sqg = random_faces(rng, n, general_metric)
    for d in (1, 2, 3):
        ref = G.riemann_faces(d, qL, qR, alpha, beta, g, sqg)
        first = G.riemann_faces_noalloc(d, qL, qR, alpha, beta, g, sqg)
        second = G.riemann_faces_noalloc(d, qL, qR, alpha, beta, g, sqg)
        assert np.all(np.isfinite(ref))
        np.testing.assert_allclose(first, ref, rtol=RTOL, atol=0.0)
        np.testing.assert_allclose(second, ref, rtol=RTOL, atol=0.0)


@pytest.mark.parametrize("rs", ["hlle", "hllc"])
@pytest.mark.parametrize("general_metric", [False, True])
def test_noalloc_matches_riemann_faces(rs, general_metric):
    rng = np.random.default_rng(2026)
    pb = (torus_2p5d(nx=8, nz=4, rs=rs) if general_metric
          else shock_tube(nx=8, rs=rs, adiabatic_index=1.3333333333333333))
    G = GpuGrid(pb, upload_initial=False)
    check_pair(G, rng, 3000, general_metric)
    check_pair(G, rng, MAX_FACES, general_metric)  # the largest call the scratch takes
    check_pair(G, rng, 17, general_metric)         # smaller call after a larger one
    G.close()


def test_noalloc_mixed_precision_handle():
    rng = np.random.default_rng(7)
    G = GpuGrid(torus_2p5d(nx=8, nz=4, rs="hllc"), precision="mixed", upload_initial=False)
    check_pair(G, rng, 1000, True)
    G.close()


def test_noalloc_rejects_oversize_and_bad_args():
    rng = np.random.default_rng(3)
    G = GpuGrid(shock_tube(nx=8), upload_initial=False)
    qL, qR, alpha, beta, g, sqg = random_faces(rng, MAX_FACES + 1, False)
    with pytest.raises(GpuError) as e:
        G.riemann_faces_noalloc(1, qL, qR, alpha, beta, g, sqg)
    assert e.value.code == -1 and "exceed" in str(e.value)
    with pytest.raises(GpuError):
        G.riemann_faces_noalloc(4, qL[:4], qR[:4], alpha[:4], beta[:4], g[:4], sqg[:4])
    # the handle stays usable after a rejected call
    check_pair(G, rng, 64, False)
    G.close()
