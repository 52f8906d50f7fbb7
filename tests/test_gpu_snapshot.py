"""Checkpoint snapshots: grhd2_gpu_snapshot_begin copies up (reference layout) out on its
own stream while later steps run; after grhd2_gpu_snapshot_wait the host buffer holds the
state of the moment the snapshot was taken (FP64: bitwise the oracle's), and the steps
that ran meanwhile are unaffected."""
import numpy as np
import pytest

from grhd_b200 import native as N
from grhd_b200.solver import GpuGrid
from oracle.binding import OracleRun
from tests.helpers import initial_state, torus_2p5d

pytestmark = pytest.mark.gpu


def test_snapshots_overlap_steps_and_hold_their_state():
    import torch
    pb = torus_2p5d(nx=64, nz=32)
    p0 = initial_state(pb)
    o = OracleRun(pb, p0)
    o.prim_to_cons()
    o.set_boundary()
    g = GpuGrid(pb, upload_initial=False)
    g.upload(p=p0)
    g.prim_to_cons()
    lib = g.lib
    bufs = [torch.empty(pb.cons_shape, dtype=torch.float64).pin_memory() for _ in range(2)]
    refs = []
    for k, steps in enumerate((3, 4)):
        g.run(0.0, 1e30, steps)
        o.run(0.0, 1e30, steps)
        refs.append(o.up.copy())
        assert lib.grhd2_gpu_snapshot_begin(g._h, N.dptr(bufs[k].numpy())) == 0
    g.run(0.0, 1e30, 5)  # runs while the second copy may still be in flight
    o.run(0.0, 1e30, 5)
    assert lib.grhd2_gpu_snapshot_wait(g._h) == 0
    for k in range(2):
        assert np.array_equal(bufs[k].numpy(), refs[k]), f"snapshot {k}"
    assert np.array_equal(g.download(want_p=False)[0], o.up)
    assert lib.grhd2_gpu_snapshot_wait(g._h) == 0  # nothing pending: returns at once
    g.close()
