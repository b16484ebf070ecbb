"""The oracle (C restatement of the reference) pinned against the reference.

* golden fixtures in tests/golden (computed by the reference itself, see
  tests/golden/make_golden.py) -- always run;
* the compiled reference on a matrix of generated cases -- where oracle/_ref
  was built;
* the reference's own shipped outputs (wedge.sav, wedge_residual.dat) -- where
  the reference sources are mounted.
"""
import glob
import json
import os

import numpy as np
import pytest

from conftest import REFERENCE_DIR, make_case, reference_available
from oracle.pyoracle import Oracle, run_reference
from supersonicflowsolver_b200 import meshgen

GOLDEN_DIR = os.path.join(os.path.dirname(__file__), "golden")


def golden_cases():
    return sorted(glob.glob(os.path.join(GOLDEN_DIR, "*.npz")))


def build_golden_inputs(tmp_path, fixture):
    import sys

    sys.path.insert(0, GOLDEN_DIR)
    from make_golden import write_inputs

    z = np.load(fixture)
    prm = json.loads(str(z["params"]))
    mesh, path = write_inputs(str(tmp_path), prm["mesh"], prm["case"], prm["iterations"])
    return z, prm, mesh, path


@pytest.mark.parametrize("fixture", golden_cases(), ids=lambda p: os.path.basename(p)[:-4])
def test_oracle_matches_reference_golden(tmp_path, fixture):
    z, prm, mesh, path = build_golden_inputs(tmp_path, fixture)
    o = Oracle(path, str(tmp_path), "g")
    linf, _ = o.run(prm["iterations"])
    interior = o.get("vol_bc") == 1
    assert np.array_equal(o.get("vol_p")[interior], z["p"])
    assert np.array_equal(o.get("vol_T")[interior], z["T"])
    assert np.array_equal(o.get("vol_u").reshape(-1, mesh.dim)[interior], z["u"])
    # the reference printed its residual columns with 4 significant digits
    printed = np.array([[float("%.3e" % x) for x in row] for row in linf])
    assert np.array_equal(printed, z["residual_columns"])


MATRIX = [
    ("hll_first_order", dict(nx=30, ny=10), dict(flux=2, order=1, lc=1, rk_level=1, cfl=0.8)),
    ("hllc_vanleer_lc1", dict(nx=30, ny=10), dict(flux=3, order=2, limiter=3, lc=1)),
    ("hll_vanalbada_lc2", dict(nx=30, ny=10), dict(flux=2, order=2, limiter=1, lc=2)),
    ("ausm_minmod_uniform", dict(nx=30, ny=10), dict(flux=1, order=2, limiter=2, lc=0, rk_level=2)),
    ("hllc_lsq", dict(nx=30, ny=10), dict(flux=3, order=2, limiter=1, lc=1, grad=2)),
    ("jitter_shuffle_hllc", dict(nx=30, ny=10, jitter=0.15, shuffle_seed=1, interior_first=True),
     dict(flux=3, order=2, limiter=3, lc=1)),
    ("custom_rk_ausm", dict(nx=30, ny=10, jitter=0.15, shuffle_seed=2),
     dict(flux=1, order=2, limiter=1, lc=2, rk_custom=[0.25, 0.5, 1.0])),
]


@pytest.mark.skipif(not reference_available(), reason="compiled reference not built here")
@pytest.mark.parametrize("tag,mkw,ckw", MATRIX, ids=[m[0] for m in MATRIX])
def test_oracle_matches_compiled_reference_2d(tmp_path, tag, mkw, ckw):
    mesh = meshgen.wedge2d(angle_deg=15.0, **mkw)
    _check_vs_reference(tmp_path, mesh, ckw, 4)


@pytest.mark.skipif(not reference_available(), reason="compiled reference not built here")
@pytest.mark.parametrize("tets", [True, False], ids=["tets", "hexes"])
def test_oracle_matches_compiled_reference_3d(tmp_path, tets):
    mesh = meshgen.wedge3d(12, 6, 3, 12.0, tets=tets)
    _check_vs_reference(tmp_path, mesh, dict(flux=3, order=2, limiter=3, lc=1, mach=3.0), 3)


@pytest.mark.skipif(not reference_available(), reason="compiled reference not built here")
@pytest.mark.parametrize("grad", [1, 2], ids=["green_gauss", "least_squares"])
def test_oracle_matches_compiled_reference_adapted(tmp_path, grad):
    """Hanging-node mesh (parent cells and faces, five-face quads)."""
    mesh = meshgen.wedge2d_adapted(24, 8, 15.0, refine_frac=0.25, seed=7)
    _check_vs_reference(tmp_path, mesh, dict(flux=3, order=2, limiter=3, lc=1, grad=grad), 4)


@pytest.mark.skipif(not (reference_available() and os.path.exists(os.path.join(REFERENCE_DIR, "testGrids"))),
                    reason="reference not mounted")
@pytest.mark.parametrize("mesh", ["quad2D_adapted1.msh", "quad2D_adapted2.msh"])
def test_oracle_matches_reference_on_its_adapted_samples(tmp_path, mesh):
    """The reference's own hanging-node samples (testGrids/guads): far-field
    inlet/outlet as 23/26, walls 15/18."""
    src = os.path.join(REFERENCE_DIR, "testGrids", "guads", mesh)
    (tmp_path / "m.msh").write_bytes(open(src, "rb").read().replace(b"\r", b""))
    meshgen.write_case(str(tmp_path), "c", max_iter=4, flux=3, order=2, limiter=3, lc=1, zones=())
    vel = open(tmp_path / "c.par").read().split("\t")[0]
    (tmp_path / "c.bvp").write_text("inlet\t23\t%s\t101325\noutlet\t26\nup\t15\ndown\t15" % vel.replace(" ", "\t"))
    (tmp_path / "c.btq").write_text("inlet\t27\t300\noutlet\t25\nup\t18\ndown\t18")
    _check_vs_reference_files(str(tmp_path / "m.msh"), str(tmp_path), "c", 4)


@pytest.mark.parametrize("tets", [True, False], ids=["tets", "hexes"])
def test_oracle_3d_least_squares_exact_for_linear_fields(tmp_path, tets):
    """The 3D least-squares gradient (corrected restatement: the reference's
    3D branch writes out of bounds) reproduces linear fields to rounding at
    every interior cell, ghosts holding the same field at their face centres."""
    mesh = meshgen.wedge3d(8, 4, 3, 12.0, tets=tets)
    path, d, name = make_case(tmp_path, mesh, max_iter=1, flux=3, order=2, limiter=3, lc=1, grad=2, mach=3.0)
    o = Oracle(path, d, name)
    x = o.get("vol_x").reshape(-1, 3)
    gp, gT = np.array([3.0e3, -2.0e3, 0.5e3]), np.array([10.0, 40.0, -15.0])
    gu = np.array([[5.0, 10.0, 15.0], [20.0, 0.0, 0.0], [0.0, 0.0, -7.0]])
    u = np.array([800.0, 0.0, 0.0]) + x @ gu.T
    o.set_prim(101325.0 + x @ gp, 300.0 + x @ gT, u.ravel())
    o.run(1)
    inner = o.get("vol_bc") == 1
    for key, ref in (("vol_grad_p", gp), ("vol_grad_T", gT)):
        got = o.get(key).reshape(-1, 3)[inner]
        assert np.max(np.abs(got - ref)) <= 1e-12 * np.max(np.abs(ref)) * 100, key
    gotu = o.get("vol_grad_u").reshape(-1, 3, 3)[inner]
    assert np.max(np.abs(gotu - gu)) <= 1e-10


def _check_vs_reference(tmp_path, mesh, ckw, n):
    path, d, name = make_case(tmp_path, mesh, max_iter=n, **ckw)
    _check_vs_reference_files(path, d, name, n)


def _check_vs_reference_files(path, d, name, n):
    ref = run_reference(path, d, name, os.path.join(d, "dump"))
    o = Oracle(path, d, name)
    o.run(n)
    for k in ["vol_p", "vol_T", "vol_rho", "vol_u", "vol_w", "vol_dt", "vol_V", "vol_x", "face_S", "face_n",
              "face_x", "face_c0", "face_c1", "vol_grad_p", "vol_grad_T", "vol_grad_u"]:
        a = ref[k].astype(float)
        b = o.get(k)
        m = np.isfinite(a)  # ghost gradients are S/0 in the reference
        assert a.shape == b.shape, k
        assert np.array_equal(a[m], b[m]), k


@pytest.mark.slow
def test_oracle_reproduces_shipped_wedge_outputs(tmp_path):
    """wedge80_240.msh + wedge.inp (HLL, 1st order, LocalAccTime1, RK1, CFL 2.08,
    3000 iterations): the shipped wedge.sav byte for byte and every residual
    column of the shipped wedge_residual.dat (the reference's files, packed in
    tests/golden/shipped_wedge)."""
    import sys

    sys.path.insert(0, GOLDEN_DIR)
    import make_shipped_wedge

    mesh, sav, res = make_shipped_wedge.unpack(str(tmp_path))
    o = Oracle(mesh, str(tmp_path), "wedge")
    linf, _ = o.run(3000)
    o.write_sav(str(tmp_path / "wedge.sav"))
    assert (tmp_path / "wedge.sav").read_bytes() == open(sav, "rb").read()
    printed = np.array([[float("%.3e" % x) for x in row] for row in linf])
    assert np.array_equal(printed, make_shipped_wedge.residual_columns(res))


@pytest.mark.parametrize("ckw", [dict(flux=2, order=1, lc=1, rk_level=1), dict(flux=3, order=2, limiter=3, lc=2,
                                                                               rk_level=1)],
                         ids=["hll_first", "hllc_vanleer"])
def test_oracle_residual_is_the_one_its_update_consumes(tmp_path, ckw):
    """The exported one-stage residual ("vol_res") is the residual the pinned
    update consumes: after one RK1 iteration, w = prev_w - dt*a*res/V bit for
    bit (psstFiniteVolumeGrid.cpp:324-330) for every interior cell."""
    mesh = meshgen.wedge2d(30, 10, 15.0, jitter=0.15, shuffle_seed=1)
    path, d, name = make_case(tmp_path, mesh, max_iter=2, **ckw)
    o = Oracle(path, d, name)
    o.run(1)
    res = o.convective()
    w0 = o.get("vol_w").reshape(-1, 4)
    o.run(1)
    interior = o.get("vol_bc") == 1
    dt, V = o.get("vol_dt")[interior], o.get("vol_V")[interior]
    w1 = o.get("vol_w").reshape(-1, 4)[interior]
    expect = w0[interior] - dt[:, None] * 1.0 * res[interior] / V[:, None]
    assert np.array_equal(w1, expect)


def test_oracle_extensions_run(tmp_path):
    """Limiters 4/5 and the Jacobi LocalAccTime1 (no reference counterpart)
    stay finite and differ from the sequential evaluation only slightly."""
    mesh = meshgen.wedge2d(30, 10, 15.0)
    path, d, name = make_case(tmp_path, mesh, max_iter=5, flux=3, order=2, limiter=4, lc=1)
    for lim in (4, 5):
        o = Oracle(path, d, name, limiter=lim)
        linf, l2 = o.run(5)
        assert np.all(np.isfinite(linf)) and np.all(np.isfinite(l2))
        assert np.all(o.get("vol_lim").reshape(-1, 4)[o.get("vol_boundary") == 0] <= 1.0 + 1e-12)
    a = Oracle(path, d, name, limiter=4)
    b = Oracle(path, d, name, limiter=4, lc1_jacobi=1)
    a.run(3)
    b.run(3)
    pa, pb = a.get("vol_p"), b.get("vol_p")
    assert not np.array_equal(pa, pb)
    assert np.max(np.abs(pa - pb) / pa) < 1e-2
