"""Committed golden vectors (tests/golden/golden_small.npz, written by
tests/golden/make_golden.py from the CPU oracle) on small seeded cases: the oracle must
still reproduce them bit for bit (CPU), and the sm_100a FP64 path must match them
(GPU; bit-identical in practice, asserted at the relative L1 bar of 1e-12 per conserved
variable plus identical con2prim counters)."""
import os

import numpy as np
import pytest

from tests.golden.make_golden import OUT, cases, compute
from tests.helpers import initial_state, rel_l1

GOLD = np.load(OUT)
CASES = {c[0]: c for c in cases()}
C2P = ["c2p_bad_V", "c2p_brent_used", "c2p_causal_rescale", "c2p_final_sanitise", "c2p_floor_pre", "c2p_root_fail"]


def test_fixture_is_complete():
    names = {k.split("/")[0] for k in GOLD.files}
    assert names == set(CASES) and os.path.getsize(OUT) < 512 * 1024


@pytest.mark.parametrize("name", sorted(CASES))
def test_oracle_reproduces_golden(name):
    out = compute(*CASES[name])
    for key, val in out.items():
        assert np.array_equal(val, GOLD[key]), key


@pytest.mark.gpu
@pytest.mark.parametrize("name", sorted(CASES))
def test_gpu_matches_golden(name):
    from grhd_b200.solver import GpuGrid
    _, maker, kw, kind, steps = CASES[name]
    pb = maker(**kw)
    g = GpuGrid(pb, upload_initial=False)
    g.upload(p=initial_state(pb))
    g.prim_to_cons()
    if kind == "rhs":
        rhs = g.calc_rhs()
        assert np.all(rel_l1(rhs, GOLD[f"{name}/rhs"]) <= 1e-12)
    else:
        n, t = g.run(0.0, 1e30, steps)
        assert n == GOLD[f"{name}/steps"][0] and t == GOLD[f"{name}/t"][0]
        up = g.download(want_p=False)[0]
        assert np.all(rel_l1(up, GOLD[f"{name}/up"]) <= 1e-12)
        names = sorted(g.counters())
        cnt = dict(zip(names, GOLD[f"{name}/counters"]))
        got = g.counters()
        for k in C2P:
            assert got[k] == cnt[k], k
    g.close()
