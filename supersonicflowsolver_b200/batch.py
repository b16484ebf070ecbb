"""Many ramp cases of uneven size and inflow solved together on one GPU.

The cases' grids are merged into one (psst_grid_merge), so every kernel
launch advances all of them; launch shapes come from the solver's own tuner
(psst_solver_autotune). The stop rule runs on the device after every
iteration (psst_solver_set_stop_rule): each case's residual column,
normalised by its first five iterations, is checked against the drop, and a
converged (or capped) case is skipped by every later launch, so it stops at
exactly its converging iteration. The whole solve is one CUDA-graph launch
(psst_solver_run_to_stop): a while-loop node repeats a captured block of
`chunk` iterations, and the block's last kernel ends the loop on the device
once no case runs; the host waits once, at the end. (chunked=True instead
replays one graph per chunk and reads the run flags between chunks.)

Workload (seeded): mesh sizes uniform over {60x20, 120x40, 180x60, 240x80}
quads (x by y), ramp angle U[5, 20] deg, Mach U[1.8, 4.0], p = 101325 Pa,
T = 300 K; FP32, HLLC, cell-limited MUSCL, Green-Gauss, RK4, LocalAccTime1
from stage-start values, CFL 0.5.

    python -m supersonicflowsolver_b200.batch --cases 256 --seed 0
"""
import argparse
import json
import os
import tempfile
import time

import numpy as np

from . import meshgen
from .psst import Grid, Solver

SIZES = [(60, 20), (120, 40), (180, 60), (240, 80)]


def sample_cases(n, seed=0):
    """n case descriptions: mesh size (nx, ny), ramp angle (deg), Mach."""
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(n):
        nx, ny = SIZES[int(rng.integers(len(SIZES)))]
        out.append({"nx": nx, "ny": ny, "angle": float(rng.uniform(5.0, 20.0)), "mach": float(rng.uniform(1.8, 4.0))})
    return out


def build_cases(cases, directory, precision=32, flux=3, limiter=5, cfl=0.5, rk_level=4):
    """Per-case grids set up from written case files; returns (grids, scheme)."""
    grids, scheme = [], None
    for i, c in enumerate(cases):
        d = os.path.join(directory, "case%d" % i)
        meshgen.write_case(d, "case", mach=c["mach"], max_iter=1, flux=flux, order=2, limiter=limiter, lc=1,
                           cfl=cfl, rk_level=rk_level)
        g = Grid.from_mesh(meshgen.wedge2d(c["nx"], c["ny"], c["angle"]))
        sc, _ = g.read_case(d, "case")
        sc.precision = precision
        sc.lc1_mode = 1
        sc.renumber = 1
        grids.append(g)
        scheme = sc
    return grids, scheme


def run_batch(solver, cells, drop=1e-6, max_iter=50000, chunk=100, scales=None, caps=None, chunked=False):
    """Iterates all cases until every case has stopped: at the residual drop,
    after caps[i] iterations (optional), or after max_iter. cells[i] =
    interior cells of case i; scales[i] (optional) a fixed residual
    normalisation per case. The stop rule is evaluated on the device after
    every iteration, so the counts are exact. One CUDA-graph launch for the
    whole solve (blocks of `chunk` iterations; chunk x RK stages even), or,
    with chunked=True, one graph replay per chunk with the run flags read in
    between. Returns per case the iteration of the drop (None: not reached)
    and the iterations run, the normalisations used, timings and the
    cell-iterations of running cases."""
    ncase = len(cells)
    cap = np.full(ncase, max_iter, dtype=np.int64)
    if caps is not None:
        cap = np.minimum(cap, np.asarray(caps, dtype=np.int64))
    solver.set_stop_rule(drop, scale_iters=5, scales=scales, caps=np.maximum(cap, 0))
    done, dev_s = 0, 0.0
    t0 = time.perf_counter()
    if not chunked:
        if solver.case_status()["active"].any():
            done = solver.run_to_stop(max_iter, chunk, history=False)[0]
            dev_s = solver.last_stats()[1] / 1000.0
    while chunked and done < max_iter and solver.case_status()["active"].any():
        n = min(chunk, max_iter - done)
        solver.explicit_solve(n)
        dev_s += solver.last_stats()[1] / 1000.0
        done += n
    wall = time.perf_counter() - t0
    st = solver.case_status()
    ran = st["iterations"].astype(np.int64)
    return {"iterations": [int(c) if c > 0 else None for c in st["converged_at"]], "ran": ran.tolist(),
            "scales": st["scales"], "run": done, "wall_s": wall, "device_s": dev_s,
            "converged": int((st["converged_at"] > 0).sum()),
            "cell_iterations": int(np.dot(ran, np.asarray(cells, dtype=np.int64)))}


def run_mixed(merged, scheme, cells, drop=1e-6, switch=1e-4, max_iter=50000, chunk=100, chunked=False):
    """FP32 until each case's residual has dropped by `switch` (above the FP32
    floor, where FP32 still makes progress), then FP64 from the FP32 state
    down to `drop`. Both phases judge the same absolute residual: the FP32
    run's iterations 1..5 normalise it. Returns per-case FP32 and FP64
    iterations, the wall time of the two phases and the hand-over (solver
    set-up and launch-shape tuning excluded, as in run_batch), the final
    state and the phases' cell-iterations."""
    sc32 = type(scheme).from_buffer_copy(scheme)
    sc32.precision = 32
    sc64 = type(scheme).from_buffer_copy(scheme)
    sc64.precision = 64
    s32 = Solver(merged, sc32)
    s64 = Solver(merged, sc64)
    s32.set_state(merged.initial_state())
    shapes = s32.autotune(2)
    s32.use_graphs(True)
    s64.launch_shape(shapes["gradient"], shapes["face"], shapes["cell"])
    s64.use_graphs(True)
    a = run_batch(s32, cells, drop=switch, max_iter=max_iter, chunk=chunk, chunked=chunked)
    t0 = time.perf_counter()
    s64.set_state(s32.get_state())
    hand = time.perf_counter() - t0
    s32.close()
    # every case keeps the iteration budget of a pure run: max_iter in all
    # (a case that did not reach the switch drop ran max_iter in FP32: cap 0)
    caps = [max_iter - r if x is not None else 0 for x, r in zip(a["iterations"], a["ran"])]
    b = run_batch(s64, cells, drop=drop, max_iter=max_iter, chunk=chunk, scales=a["scales"], caps=caps,
                  chunked=chunked)
    state = s64.get_state()
    s64.close()
    wall = a["wall_s"] + hand + b["wall_s"]
    total = [None if (x is None or y is None) else x + y for x, y in zip(a["iterations"], b["iterations"])]
    return {"iterations": total, "fp32_iterations": a["iterations"], "fp64_iterations": b["iterations"],
            "switched": a["converged"], "converged": b["converged"], "wall_s": wall,
            "fp32_wall_s": a["wall_s"], "fp64_wall_s": b["wall_s"], "handover_s": hand, "state": state,
            "cell_iterations": a["cell_iterations"] + b["cell_iterations"], "threads_per_block": shapes}


def unconverged_summary(cases, iterations):
    """Where the cases that never reach the drop sit: counts (converged / all)
    per Mach and ramp-angle bin and per mesh size, and the list of the
    unconverged cases."""
    mach_edges, angle_edges = [1.8, 2.35, 2.9, 3.45, 4.0], [5.0, 10.0, 15.0, 20.0]
    grid = {}
    for c, it in zip(cases, iterations):
        mb = min(int(np.searchsorted(mach_edges, c["mach"], side="right")) - 1, len(mach_edges) - 2)
        ab = min(int(np.searchsorted(angle_edges, c["angle"], side="right")) - 1, len(angle_edges) - 2)
        key = "M %.2f-%.2f, %g-%g deg" % (mach_edges[mb], mach_edges[mb + 1], angle_edges[ab], angle_edges[ab + 1])
        g = grid.setdefault(key, [0, 0])
        g[1] += 1
        g[0] += it is not None
    sizes = {}
    for c, it in zip(cases, iterations):
        k = "%dx%d" % (c["nx"], c["ny"])
        g = sizes.setdefault(k, [0, 0])
        g[1] += 1
        g[0] += it is not None
    bad = [dict(c, index=i) for i, (c, it) in enumerate(zip(cases, iterations)) if it is None]
    return {"by_mach_angle": {k: "%d/%d" % tuple(v) for k, v in sorted(grid.items())},
            "by_mesh": {k: "%d/%d" % tuple(v) for k, v in sorted(sizes.items())}, "unconverged": bad}


def main():
    ap = argparse.ArgumentParser(description=__doc__, formatter_class=argparse.RawDescriptionHelpFormatter)
    ap.add_argument("--cases", type=int, default=256)
    ap.add_argument("--seed", type=int, default=0)
    ap.add_argument("--drop", type=float, default=1e-6)
    ap.add_argument("--max-iter", type=int, default=50000)
    ap.add_argument("--chunk", type=int, default=100, help="iterations per captured block")
    ap.add_argument("--chunked", action="store_true",
                    help="one graph replay per chunk, run flags read in between (default: one launch)")
    ap.add_argument("--flux", type=int, default=3, help="1 AUSM, 2 HLL, 3 HLLC")
    ap.add_argument("--limiter", type=int, default=5)
    ap.add_argument("--precision", type=int, default=32)
    ap.add_argument("--mixed", type=float, default=None, metavar="SWITCH",
                    help="FP32 down to this residual drop, then FP64 to --drop")
    a = ap.parse_args()
    cases = sample_cases(a.cases, a.seed)
    if a.mixed is not None:
        with tempfile.TemporaryDirectory() as d:
            t0 = time.perf_counter()
            grids, sc = build_cases(cases, d, precision=32, flux=a.flux, limiter=a.limiter)
            merged = Grid.merge(grids)
            setup_s = time.perf_counter() - t0
            r = run_mixed(merged, sc, [g.ninterior for g in grids], drop=a.drop, switch=a.mixed,
                          max_iter=a.max_iter, chunk=a.chunk, chunked=a.chunked)
        its = [x for x in r["iterations"] if x is not None]
        f32 = [x for x in r["fp32_iterations"] if x is not None]
        f64 = [x for x in r["fp64_iterations"] if x is not None]
        print(json.dumps({"cases": a.cases, "seed": a.seed, "flux": a.flux, "limiter": a.limiter,
                          "precision": "fp32 to %g, then fp64" % a.mixed, "cells": int(merged.ninterior),
                          "setup_s": setup_s, "threads_per_block": r["threads_per_block"],
                          "switched": r["switched"], "converged": r["converged"], "wall_s": r["wall_s"],
                          "fp32_wall_s": r["fp32_wall_s"], "fp64_wall_s": r["fp64_wall_s"],
                          "cell_updates_per_s": r["cell_iterations"] / r["wall_s"],
                          "iterations_median": float(np.median(its)) if its else None,
                          "iterations_max": max(its) if its else None,
                          "fp32_iterations_median": float(np.median(f32)) if f32 else None,
                          "fp64_iterations_median": float(np.median(f64)) if f64 else None,
                          "where": unconverged_summary(cases, r["iterations"])}))
        return
    with tempfile.TemporaryDirectory() as d:
        t0 = time.perf_counter()
        grids, sc = build_cases(cases, d, precision=a.precision, flux=a.flux, limiter=a.limiter)
        merged = Grid.merge(grids)
        solver = Solver(merged, sc)
        solver.set_state(merged.initial_state())
        setup_s = time.perf_counter() - t0
        shapes = solver.autotune(2)
        solver.use_graphs(True)
        r = run_batch(solver, [g.ninterior for g in grids], drop=a.drop, max_iter=a.max_iter, chunk=a.chunk,
                      chunked=a.chunked)
    its = [x for x in r["iterations"] if x is not None]
    out = {"cases": a.cases, "seed": a.seed, "flux": a.flux, "limiter": a.limiter, "precision": a.precision,
           "cells": int(merged.ninterior), "setup_s": setup_s,
           "threads_per_block": shapes, "converged": r["converged"], "iterations_run": r["run"],
           "wall_s": r["wall_s"], "device_s": r["device_s"],
           "cell_updates_per_s": r["cell_iterations"] / r["wall_s"],
           "iterations_median": float(np.median(its)) if its else None,
           "iterations_max": max(its) if its else None,
           "where": unconverged_summary(cases, r["iterations"])}
    print(json.dumps(out))


if __name__ == "__main__":
    main()
