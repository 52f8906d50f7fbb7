"""The solve server's scheduling on the CPU with a simulated engine: every request
completes with its own step count, admission never exceeds the memory budget and follows
arrival order, requests that arrive while others run join the batch (continuous
batching), and the request stream follows its specification."""
import math

import numpy as np
import pytest

from grhd_b200.serve import SolveServer, make_stream, summarize


class FakeGrid:
    def __init__(self, req):
        self.req = req
        self.need = max(1, req.cells // 64)  # steps to the final time
        self.steps = 0


class FakeBatch:
    def __init__(self, grids):
        self.grids = list(grids)


class FakeEngine:
    """Deterministic stand-in: simulated time advances 1e-4 s per batched step."""

    def __init__(self):
        self.now = 0.0
        self.live = 0
        self.max_live = 0
        self.admitted = []

    def clock(self):
        return self.now

    def sleep(self, d):
        self.now += d

    def free_bytes(self):
        return 10 ** 9

    def bytes_needed(self, req):
        return req.cells * 1000

    def prepare(self, req):
        self.live += self.bytes_needed(req)
        self.max_live = max(self.max_live, self.live)
        self.admitted.append(req.id)
        return FakeGrid(req)

    def batch(self, grids, new_clocks):
        assert len(grids) == len(new_clocks)
        return FakeBatch(grids)

    def step(self, b, k):
        for g in b.grids:
            g.steps = min(g.need, g.steps + k)
        self.now += 1e-4 * k

    def clocks(self, b):
        st = np.array([g.steps for g in b.grids])
        act = np.array([g.steps < g.need for g in b.grids])
        return st * 1e-3, st, act

    def finish(self, g, keep):
        self.live -= self.bytes_needed(g.req)
        return np.array([g.req.id, g.steps]) if keep else None

    def close_batch(self, b):
        pass


def _server(eng, budget, **kw):
    return SolveServer(eng, budget_bytes=budget, clock=eng.clock, sleep=eng.sleep, **kw)


def test_all_complete_with_their_own_steps():
    reqs = make_stream(300, seed=5, rate=5000.0, riemann_cells=(128, 1024), michel_cells=(128, 512))
    eng = FakeEngine()
    res = _server(eng, 40 * 1024 * 1000, keep_results=True).run(reqs)
    assert [r.id for r in res] == [q.id for q in reqs]
    for r, q in zip(res, reqs):
        assert r.steps == max(1, q.cells // 64)
        assert r.arrival <= r.admitted <= r.done
        assert r.up[0] == q.id
    assert eng.live == 0


def test_admission_respects_budget_and_arrival_order():
    reqs = make_stream(200, seed=9, rate=20000.0, riemann_cells=(128, 2048), michel_cells=(256, 1024))
    budget = 3 * 2048 * 1000
    eng = FakeEngine()
    srv = _server(eng, budget)
    srv.run(reqs)
    assert eng.max_live <= budget and srv.peak_bytes <= budget
    assert eng.admitted == sorted(eng.admitted)  # first come, first served


def test_continuous_batching_admits_while_others_run():
    reqs = make_stream(100, seed=3, rate=2000.0, riemann_cells=(512, 4096), michel_cells=(512, 1024))
    eng = FakeEngine()
    res = _server(eng, 10 ** 9, steps_per_round=4).run(reqs)
    # some request was admitted while an earlier one was still running, and grids of
    # different arrival share rounds (more than one active at a time)
    overlap = any(b.admitted < a.done and b.id > a.id for a in res for b in res)
    assert overlap
    s = summarize(res)
    assert s["requests"] == 100 and s["tts_p99_s"] >= s["tts_p50_s"] > 0


def test_oversized_request_is_rejected():
    reqs = make_stream(3, seed=1, rate=100.0, riemann_cells=(4096, 4096), michel_cells=(4096, 4096))
    with pytest.raises(ValueError):
        _server(FakeEngine(), 1000).run(reqs)


def test_stream_follows_specification():
    reqs = make_stream(4096, seed=20260901, rate=1000.0)
    assert reqs == make_stream(4096, seed=20260901, rate=1000.0)  # seeded
    arr = np.array([r.arrival for r in reqs])
    assert np.all(np.diff(arr) > 0)
    assert abs(arr[-1] / 4096 - 1e-3) < 1e-4  # mean inter-arrival 1/rate
    rie = [r for r in reqs if r.kind == "riemann"]
    mic = [r for r in reqs if r.kind == "michel"]
    assert abs(len(rie) / 4096 - 0.7) < 0.03
    assert all(128 <= r.cells <= 8192 for r in rie) and all(512 <= r.cells <= 4096 for r in mic)
    lc = np.log([r.cells for r in rie])
    assert abs(lc.mean() - 0.5 * (math.log(128) + math.log(8192))) < 0.1  # log-uniform
    for r in rie:
        k = r.keys
        assert 0.1 <= k["sod_density_left"] <= 10 and 1e-3 <= k["sod_pressure_right"] <= 100
        assert -0.9 <= k["sod_velocity_left"] <= 0.9
        assert k["adiabatic_index"] in (4 / 3, 5 / 3) and k["reconstruction"] in ("weno5", "mp5")
        assert k["riemann_solver"] in ("hlle", "hllc") and r.final_time == 0.4
    assert {r.keys["reconstruction"] for r in mic} == {"mp5"}
