"""The continuous-batching solve server on the GPU: a stream of Riemann and Michel
requests, admitted under a memory budget that forces some to wait, stepped together in
shared batches that change as requests arrive and finish.  Each result must equal the
same request solved alone (FP64 path: bit for bit, same step count and final time)."""
import numpy as np
import pytest

from grhd_b200.problem import Problem
from grhd_b200.serve import GpuEngine, SolveServer, make_stream, summarize
from grhd_b200.solver import GpuGrid

pytestmark = pytest.mark.gpu


def solo(req, precision="fp64"):
    pb = Problem.from_keys(req.problem, **req.keys)
    g = GpuGrid(pb, precision=precision, upload_initial=False)
    g.upload(p=pb.initial_prims())
    g.prim_to_cons()
    n, t = g.run(0.0, req.final_time)
    up = g.download(want_p=False)[0]
    g.close()
    return n, t, up


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_results_equal_solo_runs(precision):
    reqs = make_stream(24, seed=77, rate=400.0, michel_final_time=1.5, riemann_cells=(64, 384),
                       michel_cells=(128, 256))
    eng = GpuEngine(precision)
    budget = sum(sorted(eng.bytes_needed(r) for r in reqs)[-6:])  # about six grids at a time
    srv = SolveServer(eng, budget_bytes=budget, steps_per_round=8, keep_results=True)
    res = srv.run(reqs)
    eng.close()
    assert len(res) == len(reqs) and srv.peak_bytes <= budget
    assert srv.rebuilds > 1 and 1 < srv.peak_active < len(reqs)
    for r, q in zip(res, reqs):
        n, t, up = solo(q, precision)
        assert (r.steps, r.t) == (n, t), f"request {q.id}: ({r.steps}, {r.t}) vs alone ({n}, {t})"
        assert np.array_equal(r.up, up), f"request {q.id} ({q.kind}, {q.cells} cells) differs from its solo run"
    s = summarize(res)
    assert s["tts_p99_s"] >= s["tts_p50_s"] > 0 and s["zone_updates_per_s"] > 0
