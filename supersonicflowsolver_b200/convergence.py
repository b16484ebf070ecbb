"""Runs ramp cases to a residual drop and compares converged fields.

Residual-drop criterion: each component of the reference's residual column
(max over RK stages and cells of |res|, psstFiniteVolumeGrid.cpp:331-332) is
normalised by its own maximum over iterations 1..5 (the rho*v component of a
freestream start is ~1e-12 at iteration 1, so iteration 1 alone is no scale);
a run has converged when every normalised component is <= `drop`.

Command line (one GPU):
    python -m supersonicflowsolver_b200.convergence jitter --nx 240 --ny 80
compares the FP32 production path against the FP64 path (bit-exact with the
oracle per iteration) at convergence for HLL, HLLC and AUSM on the jittered,
shuffled quad ramp and prints one JSON line per flux.
"""
import argparse
import json
import math
import tempfile
import time

import numpy as np

from . import meshgen
from .psst import Grid, Solver


class DropMonitor:
    """Tracks the normalised residual columns of consecutive iterations."""

    def __init__(self, drop=1e-6, scale_iters=5, scale=None):
        """scale: a fixed normalisation (e.g. another run's iterations 1..5, so
        that two starts of one case must reach the same absolute residual)."""
        self.drop = drop
        self.scale_iters = 0 if scale is not None else scale_iters
        self.rows = 0
        self.scale = None if scale is None else np.asarray(scale, dtype=np.float64)
        self.converged_at = None
        self.last = None

    def update(self, linf):
        """Feeds rows (n, nv) of residual columns; returns True once converged."""
        for row in np.asarray(linf, dtype=np.float64):
            self.rows += 1
            if self.rows <= self.scale_iters:
                self.scale = row.copy() if self.scale is None else np.maximum(self.scale, row)
            if self.rows < self.scale_iters:
                continue
            norm = row / np.where(self.scale > 0, self.scale, 1.0)
            self.last = norm
            if self.converged_at is None and np.all(norm <= self.drop):
                self.converged_at = self.rows
        return self.converged_at is not None


def ramp2d_case(directory, nx, ny, angle, mach, *, jitter=0.0, seed=0, shuffle_seed=None, flux=3, order=2,
                limiter=4, precision=64, lc=1, cfl=0.5, rk_level=4, mesh=None):
    """Quad ramp channel (meshgen.wedge2d) with supersonic inlet, extrapolated
    outlet and slip walls; returns (grid, scheme, prim) with LocalAccTime1
    evaluated from stage-start values (the parallel mode)."""
    if mesh is None:
        mesh = meshgen.wedge2d(nx, ny, angle, jitter=jitter, seed=seed, shuffle_seed=shuffle_seed,
                               interior_first=shuffle_seed is not None)
    meshgen.write_case(directory, "case", mach=mach, max_iter=1, flux=flux, order=order, limiter=limiter, lc=lc,
                       cfl=cfl, rk_level=rk_level)
    grid = Grid.from_mesh(mesh)
    sc, prim = grid.read_case(directory, "case")
    sc.precision = precision
    sc.lc1_mode = 1
    sc.renumber = 1
    return grid, sc, prim


def run_to_drop(solver, drop=1e-6, max_iter=100000, chunk=200):
    """Iterates in chunks until the residual drop is reached (or max_iter);
    returns iterations to the drop, iterations run, device and wall seconds."""
    mon = DropMonitor(drop)
    done = 0
    dev_ms = 0.0
    t0 = time.perf_counter()
    while done < max_iter:
        n = min(chunk, max_iter - done)
        linf, _ = solver.explicit_solve(n)
        dev_ms += solver.last_stats()[1]
        done += n
        if not np.all(np.isfinite(linf)):
            break
        if mon.update(linf):
            break
    wall = time.perf_counter() - t0
    return {"converged": mon.converged_at is not None, "iterations": mon.converged_at, "run": done,
            "device_s": dev_ms / 1000.0, "wall_s": wall,
            "final_drop": None if mon.last is None else float(np.max(mon.last))}


def fields(prim, grid, gamma=1.4, R=287.0):
    """Interior density, pressure and Mach number from a prim array."""
    nv, dim = grid.nvol, grid.dim
    interior = grid.get("vol_bc") == 1
    p, T = prim[:nv], prim[nv:2 * nv]
    u = prim[2 * nv:].reshape(dim, nv)
    rho = p / (R * T)
    mach = np.sqrt((u * u).sum(axis=0)) / np.sqrt(gamma * R * T)
    return {"rho": rho[interior], "p": p[interior], "mach": mach[interior]}


def field_error(a, b, grid):
    """Max and RMS relative difference of rho, p, Mach between two prim arrays
    (b is the reference)."""
    fa, fb = fields(a, grid), fields(b, grid)
    out = {}
    for k in ("rho", "p", "mach"):
        rel = np.abs(fa[k] - fb[k]) / np.maximum(np.abs(fb[k]), 1e-300)
        out[k] = {"max_rel": float(rel.max()), "rms_rel": float(math.sqrt(np.mean(rel * rel)))}
    return out


def precision_study(nx, ny, angle=15.0, mach=2.5, fluxes=(2, 3, 1), order=2, limiter=5, jitter=0.15, seed=0,
                    shuffle_seed=1, drop=1e-6, max_iter=100000, device=0):
    """FP64 and FP32 runs of each flux to the residual drop on one mesh; yields
    one result dict per flux with the FP32 field error against FP64."""
    mesh = meshgen.wedge2d(nx, ny, angle, jitter=jitter, seed=seed, shuffle_seed=shuffle_seed,
                           interior_first=shuffle_seed is not None)
    names = {1: "AUSM", 2: "HLL", 3: "HLLC"}
    for flux in fluxes:
        res = {"mesh": "%dx%d quads" % (nx, ny), "jitter": jitter, "flux": names[flux], "order": order,
               "limiter": limiter if order == 2 else None, "angle": angle, "mach": mach, "drop": drop}
        states = {}
        for prec in (64, 32):
            with tempfile.TemporaryDirectory() as d:
                grid, sc, prim = ramp2d_case(d, nx, ny, angle, mach, flux=flux, order=order, limiter=limiter,
                                             precision=prec, mesh=mesh)
                s = Solver(grid, sc, device=device)
                s.use_graphs(True)
                s.set_state(prim)
                r = run_to_drop(s, drop=drop, max_iter=max_iter)
                states[prec] = s.get_state()
                res["fp%d" % prec] = r
                s.close()
        res["fp32_vs_fp64"] = field_error(states[32], states[64], grid)
        yield res


def main():
    ap = argparse.ArgumentParser(description=__doc__, formatter_class=argparse.RawDescriptionHelpFormatter)
    ap.add_argument("study", choices=["jitter", "plain"])
    ap.add_argument("--nx", type=int, default=240)
    ap.add_argument("--ny", type=int, default=80)
    ap.add_argument("--order", type=int, default=2)
    ap.add_argument("--limiter", type=int, default=5)
    ap.add_argument("--angle", type=float, default=15.0)
    ap.add_argument("--mach", type=float, default=2.5)
    ap.add_argument("--drop", type=float, default=1e-6)
    ap.add_argument("--max-iter", type=int, default=100000)
    a = ap.parse_args()
    jitter, shuffle = (0.15, 1) if a.study == "jitter" else (0.0, None)
    for r in precision_study(a.nx, a.ny, angle=a.angle, mach=a.mach, order=a.order, limiter=a.limiter, jitter=jitter,
                             shuffle_seed=shuffle, drop=a.drop, max_iter=a.max_iter):
        print(json.dumps(r), flush=True)


if __name__ == "__main__":
    main()
