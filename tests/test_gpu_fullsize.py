"""FP64 parity at the configurations' full sizes and final times.

The oracle needs minutes to hours of host time for these runs, so its results are
committed fixtures (tests/golden/make_fullsize.py writes them): the whole final state of
the 1D Michel run to t = 500, and for the tori the SHA-256 of the final conserved state,
its value at 2048 seeded cells, the step count, the final time and the counters.  The bar
is the one stated for the FP64 path -- relative L1 at most 1e-12 per conserved variable at
the final time, identical con2prim failure and floor counts -- and the FP64 kernels are
expected to meet it with equality to the bit, which the digest checks over every cell.
"""
import os

import numpy as np
import pytest

from grhd_b200.solver import GpuGrid
from tests.golden.make_fullsize import CASES, path_of, state_digest
from tests.helpers import initial_state, rel_l1

L1_TOL = 1e-12
C2P_COUNTERS = ("c2p_floor_pre", "c2p_causal_rescale", "c2p_brent_used", "c2p_root_fail", "c2p_bad_V",
                "c2p_final_sanitise")


def run_gpu(name):
    maker, run, _ = CASES[name]
    pb = maker()
    g = GpuGrid(pb, upload_initial=False)
    g.upload(p=initial_state(pb))
    g.prim_to_cons()
    n, t = g.run(0.0, run.get("final_time", 1e30), run.get("nsteps", -1))
    up, _ = g.download(want_p=False)
    cnt = g.counters()
    g.close()
    return n, t, up, cnt


@pytest.mark.gpu
@pytest.mark.parametrize("name", list(CASES))
def test_fullsize_fp64_against_oracle(name):
    ref = np.load(path_of(name))
    n, t, up, cnt = run_gpu(name)
    assert n == int(ref["steps"]) and t == float(ref["t"]), f"clock: gpu ({n}, {t!r}) oracle ({int(ref['steps'])}, {float(ref['t'])!r})"
    flat = up.reshape(-1, 5)
    if "up" in ref.files:  # the whole final state is in the fixture
        l1 = rel_l1(up, ref["up"])
        assert np.all(l1 <= L1_TOL), f"relative L1 per conserved variable {l1}"
    # over every cell: the digest of the final state (equality to the bit), with the
    # sampled cells and the per-variable sums of |up| to show where a mismatch lies
    sample_l1 = rel_l1(flat[ref["sample_index"]], ref["sample_up"])
    sums = np.abs(flat).sum(axis=0)
    assert state_digest(up) == str(ref["sha256"]), (
        f"final state differs from the oracle's: relative L1 over the sampled cells {sample_l1}, "
        f"sum|up| gpu {sums} oracle {ref['abs_sum']}")
    names = [str(s) for s in ref["counter_names"]]
    oc = dict(zip(names, ref["counters"].tolist()))
    for k in C2P_COUNTERS + ("recon_floor_clamps", "hllc_fallbacks"):
        assert cnt[k] == oc[k], f"counter {k}: gpu {cnt[k]} oracle {oc[k]}"


def test_fullsize_fixtures_consistent():
    """Every fixture the parity test reads is committed and agrees with itself: where the
    whole state is stored, its digest, sampled cells and sums are the stored ones."""
    missing = [nm for nm in CASES if not os.path.exists(path_of(nm))]
    assert not missing, f"missing fixtures {missing}"
    for nm in CASES:
        ref = np.load(path_of(nm))
        assert int(ref["steps"]) > 0 and len(str(ref["sha256"])) == 64
        if "up" in ref.files:
            up = ref["up"]
            assert state_digest(up) == str(ref["sha256"])
            flat = up.reshape(-1, 5)
            assert np.array_equal(flat[ref["sample_index"]], ref["sample_up"])
            assert np.array_equal(np.abs(flat).sum(axis=0), ref["abs_sum"])
