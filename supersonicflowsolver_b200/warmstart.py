"""Learned warm start: converged ramp fields from the batched solver train the
coordinate MLP (tensor-core kernels of csrc/mlp.cu), whose prediction then
replaces the freestream initial field of unseen cases.

Pipeline (one GPU):
  1. training data: seeds 1..8 of the batch workload (256 cases each), each
     case run to the residual drop (or an iteration cap) from freestream; the
     interior cells' (Mach, angle, x, y) -> (rho, u, v, p) become samples;
  2. training: Adam on the MSE of the normalised fields, BF16 tensor cores;
  3. evaluation on seed 9: the same 256 cases solved from freestream and from
     the network's prediction (inference timed in), iterations and wall time
     to the drop per case, and the field difference between the two converged
     solutions. The solver's own residual judges the prediction: a case is
     done only when its residual has dropped, whatever the start.

    python -m supersonicflowsolver_b200.warmstart --train-seeds 1-8 --test-seed 9
"""
import argparse
import json
import math
import os
import tempfile
import time

import numpy as np

from . import batch as bt
from .convergence import field_error
from .mlp import MLP, fields_from_outputs, normalise_inputs, targets
from .psst import Grid, Solver

R_GAS, GAMMA, P_INF, T_INF = 287.0, 1.4, 101325.0, 300.0


def freestream(mach):
    rho = P_INF / (R_GAS * T_INF)
    return rho, mach * math.sqrt(GAMMA * R_GAS * T_INF), P_INF


def solve_batch(cases, precision, flux, limiter, max_iter, chunk, init=None, scales=None, device=0):
    """Merged solve of `cases` from freestream, or from init(case_index, grid,
    prim_of_case) -> prim_of_case; scales: per-case residual normalisations
    (default: each run's own iterations 1..5). Returns per-case results and
    states."""
    with tempfile.TemporaryDirectory() as d:
        grids, sc = bt.build_cases(cases, d, precision=precision, flux=flux, limiter=limiter)
    merged = Grid.merge(grids)
    prim = merged.initial_state()
    ptr, nv = merged.cases(), merged.nvol
    t_init = 0.0
    if init is not None:
        t0 = time.perf_counter()
        for i, g in enumerate(grids):
            sl = [slice(q * nv + ptr[i], q * nv + ptr[i + 1]) for q in range(4)]
            own = np.concatenate([prim[s] for s in sl])
            new = init(i, g, own)
            for q in range(4):
                prim[sl[q]] = new[q * g.nvol:(q + 1) * g.nvol]
        t_init = time.perf_counter() - t0
    s = Solver(merged, sc, device=device)
    s.set_state(prim)
    s.use_graphs(True)
    r = bt.run_batch(s, [g.ninterior for g in grids], max_iter=max_iter, chunk=chunk, scales=scales)
    state = s.get_state()
    per_case = []
    for i, g in enumerate(grids):
        per_case.append(np.concatenate([state[q * nv + ptr[i]:q * nv + ptr[i + 1]] for q in range(4)]))
    r["init_s"] = t_init
    s.close()
    return r, grids, per_case


def samples(case, grid, prim):
    """(inputs, targets) of one converged case's interior cells."""
    nv = grid.nvol
    interior = grid.get("vol_bc") == 1
    xy = grid.get("vol_x").reshape(nv, 2)[interior]
    p, T = prim[:nv][interior], prim[nv:2 * nv][interior]
    u, v = prim[2 * nv:3 * nv][interior], prim[3 * nv:][interior]
    rho_inf, speed, p_inf = freestream(case["mach"])
    return normalise_inputs(case["mach"], case["angle"], xy), targets(p / (R_GAS * T), u, v, p, rho_inf, speed, p_inf)


def predict_prim(net, case, grid, prim):
    """Initial prim of one case: the network's fields in interior cells, the
    freestream state (case file) in ghost cells."""
    import torch

    nv = grid.nvol
    interior = grid.get("vol_bc") == 1
    xy = grid.get("vol_x").reshape(nv, 2)[interior]
    x = torch.from_numpy(normalise_inputs(case["mach"], case["angle"], xy)).cuda()
    y = net.forward(x).cpu().numpy()
    rho_inf, speed, p_inf = freestream(case["mach"])
    rho, u, v, p = fields_from_outputs(y, rho_inf, speed, p_inf)
    # keep the start physical whatever the network says: the solver, not the
    # network, decides when the case has converged
    rho = np.clip(rho, 0.3 * rho_inf, 20.0 * rho_inf)
    p = np.clip(p, 0.3 * p_inf, 40.0 * p_inf)
    u = np.clip(u, -1.5 * speed, 1.5 * speed)
    v = np.clip(v, -1.5 * speed, 1.5 * speed)
    out = prim.copy()
    out[:nv][interior] = p
    out[nv:2 * nv][interior] = p / (R_GAS * rho)
    out[2 * nv:3 * nv][interior] = u
    out[3 * nv:][interior] = v
    return out


def train(net, X, Y, epochs, batch, lr, seed=0, log=None):
    import torch

    n = len(X)
    Xd, Yd = torch.from_numpy(X).cuda(), torch.from_numpy(Y).cuda()
    g = torch.Generator(device="cuda").manual_seed(seed)
    steps = 0
    total = epochs * max(1, n // batch)
    t0 = time.perf_counter()
    hist = []
    for ep in range(epochs):
        perm = torch.randperm(n, device="cuda", generator=g)
        ls = []
        for b0 in range(0, n - batch + 1, batch):
            idx = perm[b0:b0 + batch]
            rate = lr * 0.5 * (1.0 + math.cos(math.pi * steps / total))  # cosine schedule
            ls.append(net.train_step(Xd[idx].contiguous(), Yd[idx].contiguous(), rate))
            steps += 1
        hist.append(float(np.mean(ls)))
        if log:
            log("epoch %d loss %.3e" % (ep, hist[-1]))
    torch.cuda.synchronize()
    return {"epochs": epochs, "steps": steps, "train_s": time.perf_counter() - t0, "loss": hist}


def main():
    ap = argparse.ArgumentParser(description=__doc__, formatter_class=argparse.RawDescriptionHelpFormatter)
    ap.add_argument("--train-seeds", default="1-8")
    ap.add_argument("--test-seed", type=int, default=9)
    ap.add_argument("--cases", type=int, default=256)
    ap.add_argument("--flux", type=int, default=3)
    ap.add_argument("--limiter", type=int, default=5)
    ap.add_argument("--precision", type=int, default=64)
    ap.add_argument("--max-iter", type=int, default=20000)
    ap.add_argument("--chunk", type=int, default=100)
    ap.add_argument("--epochs", type=int, default=20)
    ap.add_argument("--batch", type=int, default=16384)
    ap.add_argument("--lr", type=float, default=2e-3)
    ap.add_argument("--out", default=None, help="write the trained parameters here (.npy)")
    ap.add_argument("--params", default=None, help="skip data and training: load parameters (.npy)")
    a = ap.parse_args()
    lo, hi = (int(v) for v in a.train_seeds.split("-"))
    log = lambda m: print(m, flush=True)
    Xs, Ys, gen = [], [], []
    for seed in ([] if a.params else range(lo, hi + 1)):
        cases = bt.sample_cases(a.cases, seed)
        r, grids, states = solve_batch(cases, a.precision, a.flux, a.limiter, a.max_iter, a.chunk)
        gen.append({"seed": seed, "converged": r["converged"], "wall_s": r["wall_s"]})
        log("data seed %d: %d/%d converged, %.1f s" % (seed, r["converged"], a.cases, r["wall_s"]))
        for c, g, st in zip(cases, grids, states):
            x, y = samples(c, g, st)
            Xs.append(x)
            Ys.append(y)
    net = MLP(seed=0)
    if a.params:
        net.set_params(np.load(a.params))
        X, tr = np.zeros((0, 4)), {"epochs": 0, "steps": 0, "train_s": 0.0, "loss": [float("nan")]}
    else:
        X, Y = np.concatenate(Xs), np.concatenate(Ys)
        tr = train(net, X, Y, a.epochs, a.batch, a.lr, log=log)
    if a.out:
        np.save(a.out, net.params())
    cases = bt.sample_cases(a.cases, a.test_seed)
    plain, grids, plain_states = solve_batch(cases, a.precision, a.flux, a.limiter, a.max_iter, a.chunk)
    # the warm start must reach the same absolute residual as the freestream start
    warm, _, warm_states = solve_batch(cases, a.precision, a.flux, a.limiter, a.max_iter, a.chunk,
                                       init=lambda i, g, pr: predict_prim(net, cases[i], g, pr),
                                       scales=plain["scales"])
    both = [i for i in range(a.cases) if plain["iterations"][i] and warm["iterations"][i]]
    ratio = [plain["iterations"][i] / warm["iterations"][i] for i in both]
    errs = [field_error(warm_states[i], plain_states[i], grids[i]) for i in both]
    # the network's own error: its prediction against the plain converged field
    pred = [field_error(predict_prim(net, cases[i], grids[i], plain_states[i]), plain_states[i], grids[i])
            for i in both]
    q = lambda v: [float(np.quantile(v, f)) for f in (0.1, 0.5, 0.9)] if len(v) else None
    out = {"train_points": int(len(X)), "generation": gen, "training": {k: tr[k] for k in ("epochs", "steps", "train_s")},
           "final_loss": tr["loss"][-1],
           "test": {"cases": a.cases, "both_converged": len(both),
                    "plain_converged": plain["converged"], "warm_converged": warm["converged"],
                    "iterations_plain_median": float(np.median([plain["iterations"][i] for i in both])) if both else None,
                    "iterations_warm_median": float(np.median([warm["iterations"][i] for i in both])) if both else None,
                    "iteration_ratio_median": float(np.median(ratio)) if ratio else None,
                    "iteration_ratio_total": (sum(plain["iterations"][i] for i in both) /
                                              sum(warm["iterations"][i] for i in both)) if both else None,
                    "wall_plain_s": plain["wall_s"], "wall_warm_s": warm["wall_s"] + warm["init_s"],
                    "warm_inference_s": warm["init_s"],
                    "iteration_ratio_q10_q50_q90": q(ratio),
                    "cases_with_ratio_ge_3": int(sum(r >= 3.0 for r in ratio)),
                    "prediction_rms_rel_q10_q50_q90": {k: q([e[k]["rms_rel"] for e in pred]) for k in ("rho", "p", "mach")},
                    "converged_field_diff_rms_rel_q50_max": {k: [float(np.median([e[k]["rms_rel"] for e in errs])),
                                                                 float(max(e[k]["rms_rel"] for e in errs))]
                                                             for k in ("rho", "p", "mach")} if errs else None,
                    "converged_field_diff_max_rel": {k: max(e[k]["max_rel"] for e in errs) for k in ("rho", "p", "mach")}
                    if errs else None}}
    print(json.dumps(out), flush=True)


if __name__ == "__main__":
    main()
