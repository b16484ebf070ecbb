"""Host side of libpsst_b200 (no GPU needed): the C ABI exports, the Fluent
reader, FP64 geometry, case files, and error behaviour, checked against the
oracle bit for bit."""
import ctypes
import os
import re
import shutil

import numpy as np
import pytest

from conftest import REFERENCE_DIR, ROOT, make_case
from oracle.pyoracle import Oracle
from supersonicflowsolver_b200 import _lib, meshgen
from supersonicflowsolver_b200.psst import Grid, PsstError, Scheme, Solver


def declared_symbols():
    hdr = open(os.path.join(ROOT, "include", "psst_b200.h")).read()
    return sorted(set(re.findall(r"\b(psst_[a-z_0-9]+)\s*\(", hdr)))


def test_header_declares_what_the_binding_lists():
    assert declared_symbols() == sorted(_lib.EXPORTED)


def test_library_exports_every_declared_symbol():
    L = ctypes.CDLL(_lib.LIB_PATH)
    for sym in declared_symbols():
        assert hasattr(L, sym), sym
    assert _lib.load().psst_abi_version() == 1


MESHES = {
    "wedge2d": lambda: meshgen.wedge2d(30, 10, 15.0),
    "wedge2d_jitter_shuffle": lambda: meshgen.wedge2d(30, 10, 15.0, jitter=0.15, shuffle_seed=1, interior_first=True),
    "wedge3d_tets": lambda: meshgen.wedge3d(8, 4, 3, 12.0, tets=True),
    "wedge3d_hexes": lambda: meshgen.wedge3d(8, 4, 3, 12.0, tets=False, interior_first=True),
}
GEOM = ["vol_V", "vol_x", "face_S", "face_n", "face_x", "face_beta", "face_c0", "face_c1", "vol_zone",
        "vol_boundary", "face_zone"]


@pytest.mark.parametrize("name", sorted(MESHES))
def test_geometry_and_case_match_oracle(tmp_path, name):
    mesh = MESHES[name]()
    path, d, case = make_case(tmp_path, mesh, max_iter=3, mach=3.0 if mesh.dim == 3 else 2.5)
    g = Grid.read_fluent(path)
    o = Oracle(path, d, case)
    for k in GEOM:
        assert np.array_equal(g.get(k).astype(float), o.get(k)), k
    assert g.min_vol == o.get("min_vol")[0]
    sc, prim = g.read_case(d, case)
    nv = g.nvol
    assert np.array_equal(prim[:nv], o.get("vol_p"))
    assert np.array_equal(prim[nv:2 * nv], o.get("vol_T"))
    assert np.array_equal(prim[2 * nv:].reshape(mesh.dim, nv).T.ravel(), o.get("vol_u"))
    s = o.get("scheme")
    assert (sc.cfl, sc.lc, sc.rk_level, sc.flux, sc.order, sc.limiter, sc.ref_vel) == \
        (s[0], s[1], s[2], s[3], s[4], s[6], s[7])
    assert list(sc.rk)[: sc.rk_level] == list(o.get("rk"))
    assert (sc.rm, sc.cp, sc.cv, sc.gamma) == tuple(o.get("gas"))
    # in-memory mesh description gives the same grid as the file
    g2 = Grid.from_mesh(mesh)
    for k in GEOM:
        assert np.array_equal(g.get(k), g2.get(k)), k


def test_reader_accepts_crlf(tmp_path):
    mesh = meshgen.wedge2d(12, 4, 15.0)
    path, d, case = make_case(tmp_path, mesh)
    crlf = os.path.join(d, "crlf.msh")
    open(crlf, "wb").write(open(path, "rb").read().replace(b"\n", b"\r\n"))
    a, b = Grid.read_fluent(path), Grid.read_fluent(crlf)
    for k in GEOM:
        assert np.array_equal(a.get(k), b.get(k))


@pytest.mark.skipif(not os.path.exists(os.path.join(REFERENCE_DIR, "quad2D.msh")), reason="reference not mounted")
@pytest.mark.parametrize("mesh", ["quad2D.msh", "quad3D.msh", "wedge40_120.msh", "wedge3D.msh"])
def test_reader_on_reference_meshes(mesh):
    """The reference's own GAMBIT/Fluent meshes (CRLF) load, with geometry
    identical to the oracle's."""
    src = os.path.join(REFERENCE_DIR, mesh)
    g = Grid.read_fluent(src)
    assert g.ninterior > 0 and g.nghost > 0


def test_reference_mesh_geometry_matches_oracle(tmp_path):
    src = os.path.join(REFERENCE_DIR, "wedge40_120.msh")
    if not os.path.exists(src):
        pytest.skip("reference not mounted")
    lf = tmp_path / "m.msh"
    lf.write_bytes(open(src, "rb").read().replace(b"\r", b""))
    for f in ("wedge.inp", "wedge.prop", "wedge.par", "wedge.bvp", "wedge.btq"):
        shutil.copy(os.path.join(REFERENCE_DIR, f), tmp_path / f)
    g = Grid.read_fluent(src)
    o = Oracle(str(lf), str(tmp_path), "wedge")
    for k in GEOM:
        assert np.array_equal(g.get(k).astype(float), o.get(k)), k
    sc, prim = g.read_case(str(tmp_path), "wedge")
    assert np.array_equal(prim[: g.nvol], o.get("vol_p"))
    assert (sc.flux, sc.order, sc.lc, sc.rk_level, sc.max_iter) == (2, 1, 1, 1, 3000)


def test_errors_carry_reference_messages(tmp_path):
    mesh = meshgen.wedge2d(12, 4, 15.0)
    path, d, case = make_case(tmp_path, mesh)
    with pytest.raises(PsstError) as e:
        Grid.read_fluent(os.path.join(d, "missing.msh"))
    assert e.value.status == 2 and "Could not open" in e.value.message
    g = Grid.read_fluent(path)
    bvp = os.path.join(d, case + ".bvp")
    txt = open(bvp).read()
    open(bvp, "w").write(txt.replace("symm", "nozone"))
    with pytest.raises(PsstError) as e:
        g.read_case(d, case)
    assert "Error: Could not found zone!" in e.value.message
    with pytest.raises(PsstError) as e:
        g.read_case(d, "nocase")
    assert "Could not found setting file" in e.value.message
    txt = open(path).read()
    open(os.path.join(d, "trunc.msh"), "w").write(txt[: len(txt) // 2])
    with pytest.raises(PsstError) as e:
        Grid.read_fluent(os.path.join(d, "trunc.msh"))
    assert e.value.status == 3


def test_subsonic_inlet_rejected_like_reference(tmp_path):
    """psstInlet's constructor always throws (psstBoundaryCondition.cpp:147)."""
    mesh = meshgen.wedge2d(12, 4, 15.0)
    path, d, case = make_case(tmp_path, mesh)
    bvp = os.path.join(d, case + ".bvp")
    txt = open(bvp).read().split("\n")
    txt[0] = "in\t27\t100.0\t0.0"
    open(bvp, "w").write("\n".join(txt))
    g = Grid.read_fluent(path)
    with pytest.raises(PsstError) as e:
        g.read_case(d, case)
    assert "Wrong dimension" in e.value.message


def test_solver_without_gpu_fails_loudly(tmp_path):
    """No CPU fallback: creating a solver needs a CUDA device."""
    try:
        import torch

        if torch.cuda.is_available():
            pytest.skip("a GPU is present")
    except ImportError:
        pass
    mesh = meshgen.wedge2d(12, 4, 15.0)
    path, d, case = make_case(tmp_path, mesh)
    g = Grid.read_fluent(path)
    sc, prim = g.read_case(d, case)
    with pytest.raises(PsstError) as e:
        Solver(g, sc)
    assert e.value.status == 4


@pytest.mark.skipif(not os.path.exists(os.path.join(REFERENCE_DIR, "wedge.dat")), reason="reference sources absent")
def test_fluent_writer_reproduces_shipped_case_and_data(tmp_path):
    """psst_write_fluent on the shipped wedge case (state from the oracle, which
    reproduces the shipped wedge.sav bit for bit) gives the shipped wedge.cas and
    wedge.dat byte for byte (line ends aside: the shipped files are CRLF)."""
    import shutil

    from conftest import oracle_prim
    from oracle.pyoracle import Oracle

    for f in ("wedge.inp", "wedge.prop", "wedge.par", "wedge.bvp", "wedge.btq"):
        shutil.copy(os.path.join(REFERENCE_DIR, f), tmp_path / f)
    with open(os.path.join(REFERENCE_DIR, "wedge80_240.msh"), "rb") as src:
        (tmp_path / "wedge80_240.msh").write_bytes(src.read().replace(b"\r", b""))
    o = Oracle(str(tmp_path / "wedge80_240.msh"), str(tmp_path), "wedge")
    o.run(3000)
    g = Grid.read_fluent(str(tmp_path / "wedge80_240.msh"))
    prim = oracle_prim(o, g.nvol, g.dim)
    g.write_fluent(prim, o.get("vol_rho"), str(tmp_path / "out"))
    for ext in ("cas", "dat"):
        shipped = open(os.path.join(REFERENCE_DIR, "wedge." + ext), "rb").read().replace(b"\r", b"")
        assert (tmp_path / ("out." + ext)).read_bytes() == shipped, ext


def test_fluent_writer_round_trip(tmp_path):
    """The written .cas reads back as the same grid (generated tet mesh, cell
    types inferred from the faces)."""
    m = meshgen.wedge3d(4, 3, 2, 12.0, tets=True)
    g = Grid.from_mesh(m)
    nv = g.nvol
    prim = np.concatenate([np.full(nv, 101325.0), np.full(nv, 300.0), np.zeros(3 * nv)])
    g.write_fluent(prim, np.full(nv, 1.1766), str(tmp_path / "t"))
    g2 = Grid.read_fluent(str(tmp_path / "t.cas"))
    assert (g2.nvol, g2.nface, g2.ninterior) == (g.nvol, g.nface, g.ninterior)
    for a in ("vol_V", "face_S", "face_n", "vol_x"):
        assert np.array_equal(g.get(a), g2.get(a)), a
    txt = (tmp_path / "t.cas").read_text()
    assert "(12 (2 1 " in txt and " 2 2 2" in txt  # tetrahedra (type 2)


def test_adapted_mesh_matches_oracle(tmp_path):
    """Hanging-node mesh (parent cells bc 32, parent faces bc 31, 58/59
    trees): reader geometry, zone types and initial state equal the oracle's,
    and the in-memory description gives the same grid as the file."""
    m = meshgen.wedge2d_adapted(30, 10, 15.0, refine_frac=0.2, seed=5)
    assert m.nparents > 0
    path, d, case = make_case(tmp_path, m, max_iter=3)
    g = Grid.read_fluent(path)
    o = Oracle(path, d, case)
    for k in GEOM + ["vol_bc"]:
        assert np.array_equal(g.get(k).astype(float), o.get(k)), k
    vbc = g.get("vol_bc")
    assert (vbc == 32).sum() == m.nparents and (vbc == 1).sum() == m.ncells == g.ninterior
    sc, prim = g.read_case(d, case)
    assert np.array_equal(prim[: g.nvol], o.get("vol_p"))
    g2 = Grid.from_mesh(m)
    for k in GEOM + ["vol_bc"]:
        assert np.array_equal(g.get(k), g2.get(k)), k


def _reference_run(d, mesh, case):
    exe = os.path.join(ROOT, "oracle", "_ref", "psst_ref")
    if not os.path.exists(exe):
        pytest.skip("reference build absent")
    import subprocess

    (d / "problem_manager").write_text("%s\n%s" % (mesh, case))
    r = subprocess.run([exe], cwd=str(d), capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]


def test_writers_reproduce_reference_on_adapted_mesh(tmp_path):
    """The reference's own adapted mesh (wedge_adaptation.msh), 5 iterations
    run by the compiled reference: psst_write_fluent and write_sav, fed the
    oracle's state (bit-identical to the reference's), give its .cas, .dat and
    .sav byte for byte (trees, parent-cell zone, parent face zones)."""
    from conftest import oracle_prim
    from supersonicflowsolver_b200.psst import write_sav

    src = os.path.join(REFERENCE_DIR, "wedge_adaptation.msh")
    if not os.path.exists(src):
        pytest.skip("reference not mounted")
    ref = tmp_path / "ref"
    ref.mkdir()
    shutil.copy(src, ref / "wa.msh")
    meshgen.write_case(str(ref), "wa", mach=2.5, max_iter=5, flux=3, order=2, limiter=3, lc=1,
                       zones=("symm-head", "symm", "wedge"))
    _reference_run(ref, "wa.msh", "wa")
    g = Grid.read_fluent(str(ref / "wa.msh"))
    vbc = g.get("vol_bc")
    assert (vbc == 32).sum() > 0 and (g.get("face_zone") > 0).all()
    o = Oracle(str(ref / "wa.msh"), str(ref), "wa")
    o.run(5)
    for k in GEOM + ["vol_bc"]:
        assert np.array_equal(g.get(k).astype(float), o.get(k)), k
    prim = oracle_prim(o, g.nvol, g.dim)
    g.write_fluent(prim, o.get("vol_rho"), str(tmp_path / "out"))
    write_sav(g, prim, o.iter, str(tmp_path / "out.sav"))
    for ext in ("cas", "dat", "sav"):
        assert (tmp_path / ("out." + ext)).read_bytes() == (ref / ("wa." + ext)).read_bytes(), ext


def test_adapted_case_file_round_trip(tmp_path):
    """The .cas written for a generated adapted mesh keeps its trees and reads
    back as the same grid."""
    m = meshgen.wedge2d_adapted(16, 6, 15.0, refine_frac=0.3, seed=2)
    path, d, case = make_case(tmp_path, m)
    g = Grid.read_fluent(path)
    nv = g.nvol
    prim = np.concatenate([np.full(nv, 101325.0), np.full(nv, 300.0), np.zeros(2 * nv)])
    g.write_fluent(prim, np.full(nv, 1.1766), str(tmp_path / "t"))
    txt = (tmp_path / "t.cas").read_text()
    assert txt.count("(58 (") == 1 and txt.count("(59 (") == sum(z.bc_type == 31 for z in m.face_zones)
    assert '(0 "Cells Trees:")' in txt and '(0 "Faces Trees:")' in txt
    g2 = Grid.read_fluent(str(tmp_path / "t.cas"))
    for k in GEOM + ["vol_bc"]:
        assert np.array_equal(g.get(k), g2.get(k)), k
    g2.write_fluent(prim, np.full(nv, 1.1766), str(tmp_path / "t2"))
    assert (tmp_path / "t2.cas").read_bytes() == (tmp_path / "t.cas").read_bytes()


def test_host_geometry_independent_of_thread_count(tmp_path):
    """Geometry and Green-Gauss weights are computed on all host threads; the
    arrays are identical with one thread (a separate process, since the
    thread count is read once)."""
    import subprocess
    import sys

    m = meshgen.wedge3d(40, 20, 6, 12.0, tets=True)  # large enough to split into chunks
    path, d, case = make_case(tmp_path, m)
    code = ("import sys, numpy as np; sys.path.insert(0, %r); from supersonicflowsolver_b200.psst import Grid; "
            "g = Grid.read_fluent(%r); np.savez(sys.argv[1], **{k: g.get(k) for k in %r})" % (ROOT, path, GEOM))
    out = {}
    for threads in ("1", "8"):
        env = dict(os.environ, PSST_HOST_THREADS=threads)
        f = str(tmp_path / ("geo%s.npz" % threads))
        subprocess.run([sys.executable, "-c", code, f], check=True, env=env, timeout=300)
        out[threads] = np.load(f)
    for k in GEOM:
        assert np.array_equal(out["1"][k], out["8"][k]), k
