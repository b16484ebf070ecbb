"""What the learned warm start gains, on a small scale: a network trained on
converged ramp cases predicts an unseen case's field far closer to its
converged solution than the freestream start is, the solver started from that
prediction reaches the same converged field, and its residual judges the
prediction (both starts are held to the same absolute residual)."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")

TRAIN = [{"nx": 60, "ny": 20, "angle": a, "mach": m} for a in (8.0, 10.0, 12.0) for m in (2.5, 3.1)]
TEST = [{"nx": 60, "ny": 20, "angle": 10.0, "mach": 2.8}]


def test_learned_start_is_closer_and_converges_to_the_same_field():
    from supersonicflowsolver_b200 import warmstart as ws
    from supersonicflowsolver_b200.convergence import field_error
    from supersonicflowsolver_b200.mlp import MLP

    r, grids, states = ws.solve_batch(TRAIN, 64, 3, 5, 12000, 200)
    assert r["converged"] == len(TRAIN)
    xs, ys = zip(*[ws.samples(c, g, s) for c, g, s in zip(TRAIN, grids, states)])
    X, Y = np.concatenate(xs), np.concatenate(ys)
    net = MLP(seed=3)
    tr = ws.train(net, X, Y, epochs=600, batch=512, lr=2e-3)
    assert tr["loss"][-1] < 0.05 * tr["loss"][0]

    plain, tgrids, pstates = ws.solve_batch(TEST, 64, 3, 5, 12000, 200)
    assert plain["converged"] == 1
    g = tgrids[0]
    free = g.initial_state()
    pred = ws.predict_prim(net, TEST[0], g, free)
    e_free = field_error(free, pstates[0], g)
    e_pred = field_error(pred, pstates[0], g)
    import hashlib

    digest = lambda a: hashlib.sha1(np.ascontiguousarray(a).tobytes()).hexdigest()[:12]
    print("train states %s, params %s, prediction %s; start error rms (free -> learned): %s"
          % (digest(np.concatenate(states)), digest(net.params()), digest(pred),
             ", ".join("%s %.3g -> %.3g" % (k, e_free[k]["rms_rel"], e_pred[k]["rms_rel"]) for k in e_free)))
    for k in ("rho", "p", "mach"):
        assert e_pred[k]["rms_rel"] < 0.5 * e_free[k]["rms_rel"], (k, e_pred[k], e_free[k])

    warm, _, wstates = ws.solve_batch(TEST, 64, 3, 5, 12000, 200, init=lambda i, gg, pr: ws.predict_prim(net, TEST[i], gg, pr),
                                      scales=plain["scales"])
    assert warm["converged"] == 1
    diff = field_error(wstates[0], pstates[0], g)
    assert all(diff[k]["rms_rel"] < 1e-5 for k in diff), diff
    print("freestream start: %d iterations, learned start: %d iterations; start error rms p %.3g -> %.3g"
          % (plain["iterations"][0], warm["iterations"][0], e_free["p"]["rms_rel"], e_pred["p"]["rms_rel"]))
