"""Batched cases: merged grids (psst_grid_merge), per-case residual columns,
per-case run flags and CUDA-graph replay.

The merge is checked on the host; on the GPU every case of a merged grid must
evolve bit for bit as it does alone (FP64), stopped cases must keep their
state, and graph replays must equal plain launches.
"""
import numpy as np
import pytest

from supersonicflowsolver_b200 import meshgen
from supersonicflowsolver_b200.psst import Grid, PsstError, Solver

# (nx, ny, ramp angle, Mach): uneven sizes and inflows, as in the batch workload
CASES = [(30, 10, 15.0, 2.5), (24, 8, 10.0, 3.0), (36, 12, 20.0, 2.0)]


def build(tmp_path, precision=64, cases=CASES, **scheme):
    kw = dict(flux=3, order=2, limiter=4, lc=1)
    kw.update(scheme)
    grids, schemes, prims = [], [], []
    for i, (nx, ny, angle, mach) in enumerate(cases):
        d = str(tmp_path / ("case%d" % i))
        meshgen.write_case(d, "case", mach=mach, max_iter=1, **kw)
        g = Grid.from_mesh(meshgen.wedge2d(nx, ny, angle))
        sc, prim = g.read_case(d, "case")
        sc.precision = precision
        sc.lc1_mode = 1
        grids.append(g)
        schemes.append(sc)
        prims.append(prim)
    return grids, schemes, prims, Grid.merge(grids)


def case_part(prim, merged, i, nvar):
    """Case i's values of a merged prim array, in the case's own layout."""
    ptr, nv = merged.cases(), merged.nvol
    return np.concatenate([prim[q * nv + ptr[i]:q * nv + ptr[i + 1]] for q in range(nvar)])


def test_merge_concatenates_cases(tmp_path):
    grids, _, prims, m = build(tmp_path)
    ptr = m.cases()
    assert list(np.diff(ptr)) == [g.nvol for g in grids]
    assert m.nvol == sum(g.nvol for g in grids) and m.nface == sum(g.nface for g in grids)
    assert m.ninterior == sum(g.ninterior for g in grids)
    assert np.array_equal(m.get("vol_V"), np.concatenate([g.get("vol_V") for g in grids]))
    assert np.array_equal(m.get("face_n"), np.concatenate([g.get("face_n") for g in grids]))
    assert np.array_equal(m.get("face_beta"), np.concatenate([g.get("face_beta") for g in grids]))
    c0 = m.get("face_c0")
    off = 0
    f = 0
    for g, base in zip(grids, ptr[:-1]):
        gc0 = g.get("face_c0")
        assert np.array_equal(c0[f:f + g.nface], np.where(gc0 < 0, -1, gc0 + base))
        f += g.nface
    prim = m.initial_state()
    for i, p in enumerate(prims):
        assert np.array_equal(case_part(prim, m, i, 4), p)
    assert m.min_vol == min(g.min_vol for g in grids)
    assert len(Grid.merge([grids[0]]).cases()) == 2


def test_merge_rejects_mixed_dimensions(tmp_path):
    g2 = Grid.from_mesh(meshgen.wedge2d(6, 3, 15.0))
    g3 = Grid.from_mesh(meshgen.wedge3d(3, 2, 2, 12.0))
    with pytest.raises(PsstError):
        Grid.merge([g2, g3])


@pytest.mark.gpu
def test_merged_cases_evolve_as_alone(tmp_path):
    grids, schemes, prims, m = build(tmp_path)
    n = 6
    solo = []
    for g, sc, prim in zip(grids, schemes, prims):
        s = Solver(g, sc)
        s.set_state(prim)
        linf, _ = s.explicit_solve(n)
        solo.append((s.get_state(), linf))
    b = Solver(m, schemes[0])
    b.set_state(m.initial_state())
    b.explicit_solve(n)
    state, per_case = b.get_state(), b.case_residuals(n)
    for i, (st, linf) in enumerate(solo):
        assert np.array_equal(case_part(state, m, i, 4), st), "case %d state" % i
        assert np.array_equal(per_case[:, i, :], linf), "case %d residual columns" % i


@pytest.mark.gpu
def test_stopped_case_keeps_its_state(tmp_path):
    grids, schemes, prims, m = build(tmp_path)
    b = Solver(m, schemes[0])
    b.set_state(m.initial_state())
    b.explicit_solve(2)
    before = b.get_state()
    b.set_active([1, 0, 1])
    b.explicit_solve(3)
    after = b.get_state()
    per_case = b.case_residuals(3)
    assert np.array_equal(case_part(after, m, 1, 4), case_part(before, m, 1, 4))
    assert np.all(per_case[:, 1, :] == 0.0)
    assert not np.array_equal(case_part(after, m, 0, 4), case_part(before, m, 0, 4))
    # the running cases are unaffected by the stopped one
    s = Solver(grids[2], schemes[2])
    s.set_state(prims[2])
    s.explicit_solve(5)
    assert np.array_equal(case_part(after, m, 2, 4), s.get_state())
    b.set_active([1, 1, 1])
    linf, _ = b.explicit_solve(1)
    assert np.all(b.case_residuals(1)[0, 1, :] > 0.0)


@pytest.mark.gpu
@pytest.mark.parametrize("rk_level", [1, 4])
def test_graph_replay_equals_plain_launches(tmp_path, rk_level):
    """RK1 with 3 iterations per call flips the state buffers an odd number of
    times per call, so replays alternate between the two captured parities."""
    grids, schemes, prims, m = build(tmp_path, rk_level=rk_level)
    runs = []
    for graphs in (False, True):
        b = Solver(m, schemes[0])
        b.use_graphs(graphs)
        b.set_state(m.initial_state())
        cols = [b.explicit_solve(3)[0] for _ in range(4)]
        runs.append((b.get_state(), np.concatenate(cols), b.case_residuals(3), b.iter))
    for x, y in zip(runs[0], runs[1]):
        assert np.array_equal(x, y)


@pytest.mark.gpu
def test_merged_grid_limits(tmp_path):
    grids, schemes, prims, m = build(tmp_path)
    sc = schemes[0]
    sc.lc1_mode = 0
    with pytest.raises(PsstError):
        Solver(m, sc)
    sc.lc1_mode = 1
    b = Solver(m, sc)
    b.set_state(m.initial_state())
    with pytest.raises(PsstError):
        b.stage_update(0)
    s = Solver(grids[0], schemes[0])
    with pytest.raises(PsstError):
        s.set_active([1])


@pytest.mark.gpu
def test_mixed_precision_batch_reaches_the_fp64_field(tmp_path):
    """FP32 down to a 1e-4 drop, then FP64 from that state down to 1e-6:
    every case converges and lands on the pure-FP64 converged field."""
    from supersonicflowsolver_b200 import batch as bt
    from supersonicflowsolver_b200.convergence import field_error

    cases = [{"nx": 60, "ny": 20, "angle": a, "mach": m} for a, m in ((8.0, 2.5), (12.0, 3.1), (10.0, 2.2))]
    grids, sc = bt.build_cases(cases, str(tmp_path), precision=32, flux=3, limiter=5)
    merged = Grid.merge(grids)
    cells = [g.ninterior for g in grids]
    r = bt.run_mixed(merged, sc, cells, drop=1e-6, switch=1e-4, max_iter=20000, chunk=100)
    assert r["switched"] == len(cases) and r["converged"] == len(cases)
    sc64 = type(sc).from_buffer_copy(sc)
    sc64.precision = 64
    s = Solver(merged, sc64)
    s.set_state(merged.initial_state())
    p = bt.run_batch(s, cells, drop=1e-6, max_iter=20000, chunk=100)
    assert p["converged"] == len(cases)
    e = field_error(r["state"], s.get_state(), merged)
    assert all(e[k]["rms_rel"] < 1e-5 for k in e), e


@pytest.mark.gpu
def test_device_stop_rule_stops_each_case_at_its_own_iteration(tmp_path):
    """The stop rule runs on the device after every iteration: each case stops
    at exactly the iteration where its normalised residual column first drops
    below the threshold (as DropMonitor finds it on the case run alone), or at
    its cap, whatever the chunk length of the calls; a stopped case keeps the
    state it had at that iteration."""
    from supersonicflowsolver_b200.convergence import DropMonitor

    cases = [(12, 4, 10.0, 2.5), (16, 6, 15.0, 3.0), (10, 4, 8.0, 2.2)]
    grids, schemes, prims, m = build(tmp_path, cases=cases, flux=2, order=1, cfl=0.8, rk_level=1)
    drop, caps = 0.05, [3000, 3000, 7]
    solo_at, solo_state = [], []
    for i, (g, sc, prim) in enumerate(zip(grids, schemes, prims)):
        s = Solver(g, sc)
        s.set_state(prim)
        mon = DropMonitor(drop)
        states = {}
        for it in range(1, caps[i] + 1):
            linf, _ = s.explicit_solve(1)
            states[it] = s.get_state()
            if mon.update(linf):
                break
        solo_at.append(mon.converged_at)
        solo_state.append(states[mon.converged_at or caps[i]])
    assert solo_at[0] is not None and solo_at[1] is not None and solo_at[2] is None
    b = Solver(m, schemes[0])
    b.set_state(m.initial_state())
    b.use_graphs(True)
    b.set_stop_rule(drop, scale_iters=5, caps=caps)
    while b.case_status()["active"].any():
        b.explicit_solve(13)
    st = b.case_status()
    assert list(st["converged_at"]) == [solo_at[0], solo_at[1], 0]
    assert list(st["iterations"]) == [solo_at[0], solo_at[1], caps[2]]
    state = b.get_state()
    for i in range(3):
        assert np.array_equal(case_part(state, m, i, 4), solo_state[i]), "case %d" % i


@pytest.mark.gpu
def test_run_to_stop_is_one_launch_with_the_same_result(tmp_path):
    """psst_solver_run_to_stop: one CUDA-graph launch whose while-loop node the
    device ends once no case runs. Each case stops at the same iteration, the
    final state and the merged residual columns equal those of host-driven
    chunked calls bit for bit; the loop runs whole blocks and no more blocks
    than max_iter allows; an odd chunk x RK-stage count is refused."""
    cases = [(12, 4, 10.0, 2.5), (16, 6, 15.0, 3.0), (10, 4, 8.0, 2.2)]
    grids, schemes, prims, m = build(tmp_path, cases=cases, flux=2, order=1, cfl=0.8, rk_level=1)
    drop, caps = 0.05, [3000, 3000, 7]
    a = Solver(m, schemes[0])
    a.set_state(m.initial_state())
    a.use_graphs(True)
    a.set_stop_rule(drop, scale_iters=5, caps=caps)
    rows = []
    while a.case_status()["active"].any():
        rows.append(a.explicit_solve(13)[0])
    ref_linf = np.concatenate(rows)
    b = Solver(m, schemes[0])
    b.set_state(m.initial_state())
    b.set_stop_rule(drop, scale_iters=5, caps=caps)
    n, linf, l2 = b.run_to_stop(3000, chunk=14)
    sa, sb = a.case_status(), b.case_status()
    for k in ("active", "iterations", "converged_at"):
        assert np.array_equal(sa[k], sb[k]), k
    assert n % 14 == 0 and n >= int(sb["iterations"].max()) and n - 14 < int(sb["iterations"].max())
    assert b.last_stats()[0] > 0  # launches counted: the blocks run times the kernels of one block
    k = min(len(ref_linf), len(linf))
    assert np.array_equal(linf[:k], ref_linf[:k])
    assert np.array_equal(a.get_state(), b.get_state())
    # the iteration bound ends the loop with cases still running
    c = Solver(m, schemes[0])
    c.set_state(m.initial_state())
    c.set_stop_rule(drop, scale_iters=5)
    n, linf, _ = c.run_to_stop(20, chunk=14)
    st = c.case_status()
    assert n == 28 and len(linf) == 20 and st["active"].any()
    assert all(it == 28 for it, on in zip(st["iterations"], st["active"]) if on)
    with pytest.raises(PsstError):
        c.run_to_stop(20, chunk=7)


@pytest.mark.gpu
def test_run_to_stop_fp32_rk4_matches_chunked_calls(tmp_path):
    """The single launch on the FP32 path with RK4 and MUSCL (the batched
    workload's scheme): same stopping iterations and final state as 100-
    iteration chunked calls; without a stop rule the call is refused."""
    cases = [(12, 4, 10.0, 2.5), (16, 6, 15.0, 3.0)]
    grids, schemes, prims, m = build(tmp_path, precision=32, cases=cases, flux=3, order=2, limiter=5, rk_level=4)
    drop = 1e-3
    a = Solver(m, schemes[0])
    a.set_state(m.initial_state())
    a.use_graphs(True)
    a.set_stop_rule(drop, scale_iters=5, caps=[4000, 4000])
    while a.case_status()["active"].any():
        a.explicit_solve(100)
    b = Solver(m, schemes[0])
    b.set_state(m.initial_state())
    with pytest.raises(PsstError):
        b.run_to_stop(100, chunk=50)
    b.set_stop_rule(drop, scale_iters=5, caps=[4000, 4000])
    n, _, _ = b.run_to_stop(4000, chunk=50)
    sa, sb = a.case_status(), b.case_status()
    for k in ("iterations", "converged_at"):
        assert np.array_equal(sa[k], sb[k]), k
    assert not sb["active"].any() and n % 50 == 0
    assert np.array_equal(a.get_state(), b.get_state())


def test_unconverged_summary_bins_every_case():
    from supersonicflowsolver_b200 import batch as bt

    cases = bt.sample_cases(64, seed=3)
    its = [None if c["angle"] > 15.0 else 100 for c in cases]
    w = bt.unconverged_summary(cases, its)
    tot = sum(int(v.split("/")[1]) for v in w["by_mach_angle"].values())
    ok = sum(int(v.split("/")[0]) for v in w["by_mach_angle"].values())
    assert tot == 64 and ok == sum(i is not None for i in its)
    assert sum(int(v.split("/")[1]) for v in w["by_mesh"].values()) == 64
    assert {c["index"] for c in w["unconverged"]} == {i for i, x in enumerate(its) if x is None}
