"""VTK cell data produced on the device (write_vtk_cell_data, output.f90:398-453): the 7
big-endian fields equal, byte for byte, what a host writer produces from the downloaded
state and the metric tables (v^r and beta^r scaled by exp(x) on log-r grids)."""
import math

import numpy as np
import pytest

from grhd_b200.solver import GpuGrid
from tests.helpers import initial_state, interior, shock_tube, torus_2p5d, torus_3d

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("maker,kw", [(torus_2p5d, dict(nx=48, nz=24)), (torus_3d, dict(nx=20, ny=10, nz=8)),
                                      (shock_tube, dict(nx=90))])
@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_vtk_cell_data_bytes(maker, kw, precision):
    pb = maker(**kw)
    p0 = initial_state(pb)
    g = GpuGrid(pb, precision=precision, upload_initial=False)
    g.upload(p=p0)
    g.prim_to_cons()
    g.run(0.0, 1e30, 3)
    got = g.vtk_cell_data()
    _, p = g.download(p_template=p0)
    q = interior(pb, p)  # (nz, ny, nx, 5)
    mv = pb.metric_view()
    alpha = np.ctypeslib.as_array(mv.alpha_c, shape=(pb.ny, pb.nx))
    beta1 = np.ctypeslib.as_array(mv.beta_c, shape=(pb.ny, pb.nx, 3))[..., 0]
    f = [q[..., v] for v in range(5)] + [np.broadcast_to(alpha, q.shape[:3]), np.broadcast_to(beta1, q.shape[:3])]
    if g.cfg.use_log_r:
        x = pb.coords()[0][pb.ng + 1:pb.ng + 1 + pb.nx]
        scale = np.array([math.exp(v) for v in x])
        f[2] = f[2] * scale
        f[6] = f[6] * scale
    want = np.stack([np.asarray(a, dtype=np.float64) for a in f]).astype(">f8")
    assert got.dtype == np.dtype(">f8") and got.tobytes() == want.tobytes()
    g.close()
