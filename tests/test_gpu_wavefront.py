"""Sequential LocalAccTime1 as one persistent launch (the wavefront schedule).

* the reference's own published case -- wedge80_240.msh with wedge.inp (HLL,
  first order, LocalAccTime1 in the reference's in-loop order, RK1, CFL 2.08,
  3000 iterations) -- run on the GPU: the .sav it writes equals the shipped
  wedge.sav byte for byte and every residual column equals the shipped
  wedge_residual.dat (tests/golden/shipped_wedge, packed by
  make_shipped_wedge.py from the reference's files);
* the wavefront and the level-by-level walk give the same bits over calls of
  different lengths, on meshes whose schedules differ (period 2 on ordered
  quads, large periods on shuffled and adapted meshes, tets);
* a grid-barrier wait that runs out is reported as PSST_ERR_TIMEOUT and the
  solver stays usable.
"""
import os
import sys

import numpy as np
import pytest

from conftest import make_case, oracle_prim
from oracle.pyoracle import Oracle
from supersonicflowsolver_b200 import meshgen
from supersonicflowsolver_b200.psst import Grid, PsstError, Solver, write_sav

pytestmark = pytest.mark.gpu

GOLDEN_DIR = os.path.join(os.path.dirname(__file__), "golden")
sys.path.insert(0, GOLDEN_DIR)
import make_shipped_wedge  # noqa: E402


def test_reference_published_case_bit_exact(tmp_path):
    mesh, sav, res = make_shipped_wedge.unpack(str(tmp_path))
    g = Grid.read_fluent(mesh)
    sc, prim = g.read_case(str(tmp_path), "wedge")
    assert (sc.flux, sc.order, sc.lc, sc.rk_level, sc.max_iter) == (2, 1, 1, 1, 3000)
    sc.precision, sc.lc1_mode = 64, 0
    s = Solver(g, sc, device=0)
    info = s.schedule_info()
    assert info["wavefront"] and info["period"] == 2 and info["levels"] == 319
    s.set_state(prim)
    linf, _ = s.explicit_solve(3000)
    launches, ms = s.last_stats()
    assert launches == 1
    out = tmp_path / "gpu.sav"
    write_sav(g, s.get_state(), s.iter, str(out))
    assert out.read_bytes() == open(sav, "rb").read()
    printed = np.array([[float("%.3e" % x) for x in row] for row in linf])
    assert np.array_equal(printed, make_shipped_wedge.residual_columns(res))
    print("3000 iterations, 19200 cells: %.1f ms on the device (%.3g cell-updates/s)"
          % (ms, 19200 * 3000 / (ms * 1e-3)))


MESHES = {
    "ordered_quads": lambda: meshgen.wedge2d(30, 10, 15.0),
    "shuffled_quads": lambda: meshgen.wedge2d(30, 10, 15.0, jitter=0.15, seed=3, shuffle_seed=1,
                                              interior_first=True),
    "adapted": lambda: meshgen.wedge2d_adapted(30, 10, 15.0, refine_frac=0.2, seed=5),
    "tets": lambda: meshgen.wedge3d(10, 5, 3, 12.0, tets=True),
}
SCHEMES = {
    "hllc_dm_vanleer_rk4": dict(flux=3, order=2, limiter=3, lc=1, rk_level=4),
    "ausm_lsq_vanalbada_rk2": dict(flux=1, order=2, limiter=1, lc=1, grad=2, rk_level=2),
    "hll_first_rk1": dict(flux=2, order=1, lc=1, rk_level=1, cfl=0.8),
    "hllc_bj_rk3": dict(flux=3, order=2, limiter=4, lc=1, rk_level=3),
    "ausm_venkat_lsq_rk4": dict(flux=1, order=2, limiter=5, lc=1, grad=2, rk_level=4),
}
PAIRS = [("ordered_quads", "hllc_dm_vanleer_rk4"), ("shuffled_quads", "ausm_lsq_vanalbada_rk2"),
         ("adapted", "hllc_dm_vanleer_rk4"), ("adapted", "hll_first_rk1"), ("tets", "hllc_dm_vanleer_rk4"),
         ("tets", "ausm_venkat_lsq_rk4"), ("ordered_quads", "hllc_bj_rk3")]


@pytest.mark.parametrize("mesh,scheme", PAIRS, ids=["%s-%s" % p for p in PAIRS])
def test_wavefront_equals_level_walk(tmp_path, mesh, scheme):
    m = MESHES[mesh]()
    ckw = dict(SCHEMES[scheme], mach=3.0 if m.dim == 3 else 2.5)
    path, d, name = make_case(tmp_path, m, max_iter=20, **ckw)
    g = Grid.read_fluent(path)
    sc, prim = g.read_case(d, name)
    sc.precision, sc.lc1_mode = 64, 0
    a, b = Solver(g, sc, device=0), Solver(g, sc, device=0)
    b.use_wavefront(False)
    assert a.schedule_info()["wavefront"] and not b.schedule_info()["wavefront"]
    a.set_state(prim)
    b.set_state(prim)
    for n in (1, 6, 2):
        la, ra = a.explicit_solve(n)
        lb, rb = b.explicit_solve(n)
        assert np.array_equal(la, lb)
        np.testing.assert_allclose(ra, rb, rtol=1e-12, atol=0)
        pa, wa = a.get_state(with_w=True)
        pb, wb = b.get_state(with_w=True)
        assert np.array_equal(pa, pb) and np.array_equal(wa, wb)
        assert np.array_equal(a.get("dt"), b.get("dt"))
        if sc.order == 2:
            for k in ("grad_p", "grad_T", "grad_u"):
                assert np.array_equal(a.get(k), b.get(k)), k
        assert np.array_equal(a.get("rho"), b.get("rho"))
    assert a.iter == b.iter


def test_wavefront_matches_oracle_over_long_call(tmp_path):
    """One call of many iterations (the pipeline full for most of the call)
    against the oracle, on the jittered, shuffled mesh."""
    m = MESHES["shuffled_quads"]()
    path, d, name = make_case(tmp_path, m, max_iter=40, flux=3, order=2, limiter=3, lc=1, rk_level=4)
    g = Grid.read_fluent(path)
    sc, prim = g.read_case(d, name)
    s = Solver(g, sc, device=0)
    s.set_state(prim)
    linf, l2 = s.explicit_solve(40)
    o = Oracle(path, d, name)
    olinf, ol2 = o.run(40)
    assert np.array_equal(linf, olinf)
    np.testing.assert_allclose(l2, ol2, rtol=1e-12, atol=0)
    assert np.array_equal(s.get_state(), oracle_prim(o, g.nvol, g.dim))


def test_barrier_wait_that_runs_out_is_reported(tmp_path):
    """With a zero wait bound every CTA that has to wait gives up at once: the
    call fails with PSST_ERR_TIMEOUT, nothing hangs, and after a new state the
    same solver runs the case exactly."""
    m = MESHES["ordered_quads"]()
    path, d, name = make_case(tmp_path, m, max_iter=4, flux=3, order=2, limiter=3, lc=1, rk_level=4)
    g = Grid.read_fluent(path)
    sc, prim = g.read_case(d, name)
    s = Solver(g, sc, device=0)
    assert s.schedule_info()["blocks"] >= 2
    s.set_state(prim)
    s.set_wait_limit(0)
    with pytest.raises(PsstError) as e:
        s.explicit_solve(4)
    assert e.value.status == 7
    s.set_wait_limit(-1)
    s.set_state(prim)
    linf, _ = s.explicit_solve(4)
    o = Oracle(path, d, name)
    olinf, _ = o.run(4)
    assert np.array_equal(linf, olinf)
    assert np.array_equal(s.get_state(), oracle_prim(o, g.nvol, g.dim))
