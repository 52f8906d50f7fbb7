"""Batched stepping: many grids of uneven sizes and different schemes in one launch per
kernel kind, each on its own device clock, replayed as a CUDA graph.

A grid's result in a batch must be the result it has alone (and the oracle's): the batch
changes how blocks are scheduled, never what a cell computes.
"""
import numpy as np
import pytest

from grhd_b200.solver import GpuBatch, GpuGrid
from oracle.binding import OracleRun
from tests.helpers import initial_state, michel, rel_l1, shock_tube, shock_tube_xy, torus_2p5d, torus_3d

pytestmark = pytest.mark.gpu


def _stream():
    import torch
    return torch.cuda.Stream(device=0)


def _cases():
    # (problem, final time, step limit)
    return [
        (shock_tube(nx=400), 0.4, -1),
        (shock_tube(nx=257, rec="mp5", rs="hllc", sensor=True), 0.2, -1),
        (shock_tube(nx=96, rec="tvd", rs="hlle", tvd_limiter="superbee"), 1e30, 37),
        (michel(nx=256), 1e30, 60),
        (torus_2p5d(nx=64, nz=32), 1e30, 20),
        (torus_3d(nx=24, ny=12, nz=12), 1e30, 6),
        (torus_2p5d(nx=48, nz=24, rec="weno3", rs="hllc", sensor=True), 1e30, 15),
        (shock_tube_xy(nx=80, ny=20), 1e30, 12),
    ]


def _make(pb, stream, precision="fp64"):
    p0 = initial_state(pb)
    g = GpuGrid(pb, precision=precision, upload_initial=False, stream=stream.cuda_stream)
    g.upload(p=p0)
    g.prim_to_cons()
    return g, p0


@pytest.mark.parametrize("graph,variant,tile,mode,stage", [
    (True, "split", 0, "graph", "off"), (False, "split", 128, "graph", "off"), (True, "fused", 0, "graph", "off"),
    (False, "fused", 64, "graph", "off"), (True, "split", 256, "graph", "off"), (True, "split", 0, "persistent", "auto"),
    (True, "split_var", 0, "graph", "off"), (False, "split_var", 64, "graph", "off"), (True, "split", 0, "graph", "on"),
    (False, "fused", 0, "graph", "on")])
def test_batch_matches_oracle_per_grid(graph, variant, tile, mode, stage):
    s = _stream()
    cases = _cases()
    grids, p0s = zip(*[_make(pb, s) for pb, _, _ in cases])
    b = GpuBatch(list(grids))
    b.set_flux_variant(variant)
    b.set_tile(tile)
    b.set_stage_kernel(stage)
    b.set_step_mode(mode)
    assert b.step_mode == mode
    if mode == "graph":
        # every case but the 3D torus is a 1D or 2D grid; scheme groups are per tile shape
        # 1D grids step with the stage kernel unless it is off
        assert (b.stage_groups > 0) == (stage != "off")
    for k, (pb, tf, ms) in enumerate(cases):
        b.set_clock(k, 0.0, tf, ms)
    # enough replays for the longest grid; finished grids idle
    for _ in range(8):
        b.step(64, graph=graph)
        if not any(b.clock(k)[2] for k in range(len(cases))):
            break
    for k, (pb, tf, ms) in enumerate(cases):
        o = OracleRun(pb, p0s[k])
        o.prim_to_cons()
        o.set_boundary()
        n_o, t_o = o.run(0.0, tf, ms)
        t_g, n_g, active = b.clock(k)
        assert not active
        assert (n_g, t_g) == (n_o, t_o), f"grid {k}: clock ({n_g}, {t_g}) vs oracle ({n_o}, {t_o})"
        up, _ = grids[k].download(want_p=False)
        l1 = rel_l1(up, o.up)
        assert np.all(l1 <= 1e-12), f"grid {k}: relative L1 {l1}"
        co, cg = o.counters.as_dict(), grids[k].counters()
        for key in ("c2p_floor_pre", "c2p_causal_rescale", "c2p_brent_used", "c2p_root_fail", "c2p_bad_V",
                    "c2p_final_sanitise"):
            assert co[key] == cg[key], f"grid {k} counter {key}"
    b.close()
    for g in grids:
        g.close()


@pytest.mark.parametrize("mode", ["graph", "persistent"])
def test_step_modes_agree(mode):
    """The persistent step kernel and the graph of stage kernels give bit-identical FP64
    states, clocks and counters (both against a solo run in the other mode)."""
    s = _stream()
    pbs = [torus_3d(nx=24, ny=12, nz=12), michel(nx=200), shock_tube(nx=333, rec="mp5", rs="hllc")]
    other = "graph" if mode == "persistent" else "persistent"
    ref = []
    for pb in pbs:
        g, _ = _make(pb, s)
        b1 = GpuBatch([g])
        b1.set_step_mode(other)
        b1.set_clock(0, 0.0, 1e30, 9)
        b1.step(12)
        ref.append((g.download(want_p=False)[0], g.counters(), b1.clock(0)))
        b1.close()
        g.close()
    grids = [_make(pb, s)[0] for pb in pbs]
    b = GpuBatch(grids)
    b.set_step_mode(mode)
    for k in range(len(grids)):
        b.set_clock(k, 0.0, 1e30, 9)
    b.step(5)
    b.step(7)
    for k, g in enumerate(grids):
        assert b.clock(k) == ref[k][2]
        assert np.array_equal(g.download(want_p=False)[0], ref[k][0])
        assert g.counters() == ref[k][1]
    b.close()
    for g in grids:
        g.close()


def test_batch_equals_alone_with_mixed_member():
    """FP64 grids give bit-identical results alone and in a batch that also holds a
    mixed-precision grid; the mixed grid itself matches its own solo run bit for bit."""
    s = _stream()
    pbs = [torus_2p5d(nx=64, nz=32), shock_tube(nx=300), torus_2p5d(nx=40, nz=20)]
    precs = ["fp64", "fp64", "mixed"]
    solo = []
    for pb, pr in zip(pbs, precs):
        g, _ = _make(pb, s, pr)
        g.run(0.0, 1e30, 10)
        solo.append(g.download(want_p=False)[0])
        g.close()
    grids = [_make(pb, s, pr)[0] for pb, pr in zip(pbs, precs)]
    b = GpuBatch(grids)
    for k in range(len(grids)):
        b.set_clock(k, 0.0, 1e30, 10)
    b.step(12, graph=True)
    for k, g in enumerate(grids):
        assert b.clock(k)[1] == 10
        up = g.download(want_p=False)[0]
        assert np.array_equal(up, solo[k]), f"grid {k} ({precs[k]}) differs in the batch"
    b.close()
    for g in grids:
        g.close()


def test_large_group_split_into_parallel_halves():
    """A scheme group of 2e6 cells or more runs as two halves on parallel graph branches;
    each grid still gets the result it has alone, bit for bit (two 3D tori of 1.05e6 cells,
    MP5 + HLLC + sensor, the split kernels and the fused ones)."""
    s = _stream()
    pbs = [torus_3d(nx=128, ny=64, nz=128, perturbation_seed=21 + k) for k in range(2)]
    solo = []
    for pb in pbs:
        g, _ = _make(pb, s)
        g.run(0.0, 1e30, 3)
        solo.append(g.download(want_p=False)[0])
        g.close()
    for variant in ("split", "fused"):
        grids = [_make(pb, s)[0] for pb in pbs]
        b = GpuBatch(grids)
        # the tuner reports one choice per group and direction: two groups of three directions
        assert len(b.autotune(reps=1)) == 6
        b.set_flux_variant(variant)
        for k in range(len(grids)):
            b.set_clock(k, 0.0, 1e30, 3)
        b.step(4, graph=True)
        for k, g in enumerate(grids):
            assert b.clock(k)[1] == 3
            up = g.download(want_p=False)[0]
            assert np.array_equal(up, solo[k]), f"grid {k} differs in the split batch ({variant})"
        b.close()
        for g in grids:
            g.close()


def test_batch_cons_to_prim_equals_per_grid():
    """grhd2_gpu_batch_cons_to_prim: every grid's primitives, conserved state and counters
    equal grhd2_gpu_cons_to_prim_all's on the same uploaded state (FP64 grids of six
    schemes and layouts, and a mixed-precision grid, after a few steps)."""
    s = _stream()
    pbs = [pb for pb, _, _ in _cases()] + [torus_2p5d(nx=48, nz=24)]
    precs = ["fp64"] * (len(pbs) - 1) + ["mixed"]
    grids = [_make(pb, s, pr)[0] for pb, pr in zip(pbs, precs)]
    b = GpuBatch(grids)
    for k in range(len(grids)):
        b.set_clock(k, 0.0, 1e30, 5)
    b.step(5, graph=True)
    ups = [g.download(want_p=False)[0] for g in grids]

    def recover(batched):
        for g, up in zip(grids, ups):
            g.upload(up=up)
            g.reset_counters()
        if batched:
            b.cons_to_prim()
        else:
            for g in grids:
                g.cons_to_prim()
        return [(*g.download(), g.counters()) for g in grids]

    alone, together = recover(False), recover(True)
    for k, ((up_a, p_a, c_a), (up_b, p_b, c_b)) in enumerate(zip(alone, together)):
        assert np.array_equal(up_a, up_b), f"grid {k}: conserved state differs"
        assert np.array_equal(p_a, p_b), f"grid {k}: primitives differ"
        assert c_a == c_b, f"grid {k}: counters {c_a} vs {c_b}"
    b.close()
    for g in grids:
        g.close()


def test_batch_profile_names():
    s = _stream()
    grids = [_make(pb, s)[0] for pb in (torus_3d(nx=16, ny=8, nz=8), shock_tube(nx=64))]
    b = GpuBatch(grids)
    b.set_step_mode("graph")
    b.set_flux_variant("split")
    b.set_stage_kernel("off")
    for k in range(2):
        b.set_clock(k, 0.0, 1e30, 1)
    names = [n for n, _ in b.profile_step()]
    assert names.count("cell_update") == 3 * 2  # two scheme groups, three stages
    assert "recon_z" in names and "riemann_y" in names and names[-1] == "advance_clocks"
    b.set_flux_variant("fused")
    names = [n for n, _ in b.profile_step()]
    assert names.count("flux_x") == 3 * 2 and names.count("flux_z") == 3 and "recon_x" not in names
    b.set_stage_kernel("on")  # the 1D grid: one stage kernel per stage; the 3D grid keeps its kernels
    names = [n for n, _ in b.profile_step()]
    assert names.count("stage") == 3 and names.count("cell_update") == 3 and names.count("flux_x") == 3
    b.set_step_mode("persistent")
    # one launch per scheme group: the 3D grid's persistent step kernel, the 1D grid's
    # persistent form of the stage kernel
    assert [n for n, _ in b.profile_step()] == ["persistent_step", "persistent_stage"]
    b.close()
    for g in grids:
        g.close()


def test_autotune_leaves_state_and_counters():
    """Autotuning times the flux variants on the live state: afterwards the state and the
    counters are unchanged, and stepping with the tuned variants gives the solo result."""
    s = _stream()
    pbs = [torus_3d(nx=24, ny=12, nz=12), shock_tube(nx=200, rec="weno5", rs="hlle", sensor=True)]
    solo = []
    for pb in pbs:
        g, _ = _make(pb, s)
        g.run(0.0, 1e30, 4)
        solo.append((g.download(want_p=False)[0], g.counters()))
        g.close()
    grids = [_make(pb, s)[0] for pb in pbs]
    b = GpuBatch(grids)
    b.set_step_mode("graph")
    for k in range(len(grids)):
        b.set_clock(k, 0.0, 1e30, 4)
    before = [(g.download(want_p=False)[0], g.counters()) for g in grids]
    chosen = b.autotune(reps=2)
    assert len(chosen) == 3 + 1
    assert all(v in ("split", "split_var", "fused") and t in (32, 64, 128) for v, t in chosen)
    for g, (up, cnt) in zip(grids, before):
        up2 = g.download(want_p=False)[0]
        assert np.array_equal(up, up2) and g.counters() == cnt
    b.step(6, graph=True)
    for k, g in enumerate(grids):
        assert np.array_equal(g.download(want_p=False)[0], solo[k][0])
        assert g.counters() == solo[k][1]
    b.close()
    for g in grids:
        g.close()


def _stage_cases():
    """Grids whose tiles end part-way in both directions, grids smaller than one tile, and
    every tile shape (1D, x-y, x-z), with the shock sensor, HLLC and the two-ghost schemes."""
    return [
        shock_tube(nx=5), shock_tube(nx=257, rec="mp5", rs="hllc", sensor=True),
        shock_tube(nx=300, rec="weno3", rs="hlle", sensor=True), shock_tube(nx=70, rec="tvd", rs="hllc"),
        shock_tube(nx=64, rec="godunov"), michel(nx=333, rec="weno5", rs="hllc", sensor=True),
        torus_2p5d(nx=37, nz=11), torus_2p5d(nx=70, nz=30, rec="mp5", rs="hllc", sensor=True),
        torus_2p5d(nx=20, nz=4, rec="weno3", rs="hlle", sensor=True),
        shock_tube_xy(nx=33, ny=9), shock_tube_xy(nx=80, ny=20, rec="weno5", rs="hlle", sensor=True),
    ]


def _run_cases(pbs, precision, stage, s, steps=13):
    grids = [_make(pb, s, precision)[0] for pb in pbs]
    b = GpuBatch(grids)
    b.set_stage_kernel(stage)
    assert (b.stage_groups > 0) == (stage == "on")
    for k in range(len(grids)):
        b.set_clock(k, 0.0, 1e30, steps)
    b.step(5, graph=False)
    b.step(steps - 5 + 1, graph=True)
    out = [(g.download(p_template=np.zeros(pb.prim_shape)), g.counters(), b.clock(k))
           for k, (g, pb) in enumerate(zip(grids, pbs))]
    b.close()
    for g in grids:
        g.close()
    return out


def test_stage_kernel_equals_face_and_cell_kernels():
    """The stage kernel (every face of a tile and its cell update through shared memory)
    gives the FP64 state, primitives, clock and all eight counters of the face and cell
    kernels, bit for bit, on 1D, x-y and x-z grids of awkward sizes."""
    s = _stream()
    pbs = _stage_cases()
    off = _run_cases(pbs, "fp64", "off", s)
    on = _run_cases(pbs, "fp64", "on", s)
    for k, pb in enumerate(pbs):
        (up0, p0), c0, k0 = off[k]
        (up1, p1), c1, k1 = on[k]
        assert k0 == k1 and k0[1] == 13, f"case {k}: clocks {k0} {k1}"
        assert np.array_equal(up0, up1), f"case {k} ({pb.nx}x{pb.ny}x{pb.nz}): state differs"
        assert np.array_equal(p0, p1), f"case {k}: primitives differ"
        assert c0 == c1, f"case {k}: counters {c0} vs {c1}"


def _stage_cases_mixed():
    """The shapes of _stage_cases with states the FP32 arithmetic of the mixed policy can
    represent: the shock tubes at a 10:1 pressure ratio (Sod's states) instead of the
    1.3e7 of the blast wave, whose 1e-6 right-state pressure is below FP32 round-off of
    the left state's energy in the fluxes."""
    sod = dict(sod_density_left=1.0, sod_pressure_left=1.0, sod_density_right=0.125, sod_pressure_right=0.1)
    return [
        shock_tube(nx=5, **sod), shock_tube(nx=257, rec="mp5", rs="hllc", sensor=True, **sod),
        shock_tube(nx=300, rec="weno3", rs="hlle", sensor=True, **sod), shock_tube(nx=70, rec="tvd", rs="hllc", **sod),
        michel(nx=333, rec="weno5", rs="hllc", sensor=True),
        torus_2p5d(nx=37, nz=11), torus_2p5d(nx=70, nz=30, rec="mp5", rs="hllc", sensor=True),
        torus_2p5d(nx=20, nz=4, rec="weno3", rs="hlle", sensor=True),
        shock_tube_xy(nx=33, ny=9, **sod),
        shock_tube_xy(nx=80, ny=20, rec="weno5", rs="hlle", sensor=True, **sod),
    ]


def test_stage_kernel_mixed_policy_within_bar():
    """Under the mixed policy the stage kernel and the face and cell kernels are two FP32
    evaluations (the FP32 units contract to FMA, and which product of a sum is contracted
    depends on the kernel a function is inlined into): each stays within the policy's bar
    of the FP64 path, relative L1 per conserved variable at most 1e-5, with the same
    clocks, on every tile shape."""
    s = _stream()
    pbs = _stage_cases_mixed()
    ref = _run_cases(pbs, "fp64", "on", s)
    for stage in ("off", "on"):
        got = _run_cases(pbs, "mixed", stage, s)
        for k, pb in enumerate(pbs):
            assert got[k][2] == ref[k][2], f"case {k}: clocks"
            l1 = rel_l1(got[k][0][0], ref[k][0][0])
            assert np.all(l1 <= 1e-5), f"stage {stage}, case {k} ({pb.nx}x{pb.ny}x{pb.nz}): relative L1 {l1}"
