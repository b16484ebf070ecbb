"""psst_convective_residual_static: the residual entry point that allocates no
memory, checked through the C ABI against the solver's own residual
(psst_convective_calculate with first-order reconstruction) and against the
oracle's residual of the same state (the reference's face loop,
psstConvectiveFlow.cpp:289-299).

Callers that cannot allocate device memory -- code under an application or
framework that owns every device allocation, or an embedded solver whose host
forbids growing the device footprint after start-up -- own their inputs and
outputs; the entry point's only scratch is a fixed buffer compiled into the
library. The buffer is shared by all calls and keeps the last call's
contents, so the GPU test makes two calls in a row with different states and
checks both. This file is named so that pytest collects it last.
"""
import ctypes

import numpy as np
import pytest

from conftest import make_case
from oracle.pyoracle import Oracle
from supersonicflowsolver_b200 import _lib, meshgen
from supersonicflowsolver_b200.psst import Grid, PsstError, Solver


def _csr(g, nint):
    """Per interior volume, (face << 1 | side) in the reference's face-loop order."""
    c0, c1 = g.get("face_c0"), g.get("face_c1")
    nf = g.nface
    cells = np.concatenate([c0, c1])
    faces = np.concatenate([np.arange(nf), np.arange(nf)])
    sides = np.concatenate([np.zeros(nf, np.int64), np.ones(nf, np.int64)])
    m = (cells >= 0) & (cells < nint)
    cells, faces, sides = cells[m], faces[m], sides[m]
    order = np.lexsort((faces, cells))
    ent = (faces[order] << 1) | sides[order]
    ptr = np.zeros(nint + 1, np.int64)
    np.cumsum(np.bincount(cells, minlength=nint), out=ptr[1:])
    return ptr.astype(np.int32), ent.astype(np.int32), c0.astype(np.int32), c1.astype(np.int32)


def _call(g, sc, prim_soa, tensors, torch):
    dim, nint, nall, nf = g.dim, g.ninterior, g.nvol, g.nface
    d = {k: torch.from_numpy(np.ascontiguousarray(v)).cuda() for k, v in tensors.items()}
    d["prim"] = torch.from_numpy(np.ascontiguousarray(prim_soa)).cuda()
    out = torch.full(((dim + 2) * nint,), float("nan"), dtype=torch.float64, device="cuda")
    torch.cuda.synchronize()
    st = _lib.load().psst_convective_residual_static(
        dim, sc.flux, nint, nall, nf, d["c0"].data_ptr(), d["c1"].data_ptr(), d["S"].data_ptr(),
        d["n"].data_ptr(), d["ptr"].data_ptr(), d["ent"].data_ptr(), d["prim"].data_ptr(),
        sc.rm, sc.cp, sc.cv, sc.gamma, out.data_ptr(), None)
    _lib.check(st)
    return out.cpu().numpy().reshape(dim + 2, nint).T


def _prim_soa(s, g, sc):
    """p, T, rho, u.. per volume, with rho exactly as the solver holds it: w[rho]
    for interior cells (psstFiniteVolumeGrid.cpp:336) and p/(T R) for ghosts (:364)."""
    prim, w = s.get_state(with_w=True)
    nv, dim = g.nvol, g.dim
    p, T = prim[:nv], prim[nv:2 * nv]
    rho = p / (T * sc.rm)
    interior = g.get("vol_boundary") == 0
    rho[interior] = w.reshape(nv, dim + 2)[interior, dim]
    return np.concatenate([p, T, rho, prim[2 * nv:]])


@pytest.mark.gpu
@pytest.mark.parametrize("mesh,flux", [("jitter2d", 3), ("jitter2d", 1), ("tets3d", 2)],
                         ids=["2d_hllc", "2d_ausm", "3d_hll"])
def test_static_residual_matches_solver_twice(tmp_path, mesh, flux):
    torch = pytest.importorskip("torch")
    m = (meshgen.wedge2d(30, 10, 15.0, jitter=0.15, shuffle_seed=1) if mesh == "jitter2d"
         else meshgen.wedge3d(10, 5, 3, 12.0, tets=True))
    path, d, name = make_case(tmp_path, m, max_iter=3, flux=flux, order=1, lc=2,
                              mach=3.0 if m.dim == 3 else 2.5)
    g = Grid.read_fluent(path)
    sc, prim = g.read_case(d, name)
    nint = g.ninterior
    bnd = g.get("vol_boundary")
    assert not bnd[:nint].any() and bnd[nint:].all()  # interior volumes first, then ghosts
    ptr, ent, c0, c1 = _csr(g, nint)
    tensors = {"c0": c0, "c1": c1, "S": g.get("face_S"),
               "n": g.get("face_n").reshape(g.nface, g.dim).T.copy(), "ptr": ptr, "ent": ent}
    s = Solver(g, sc, device=0)
    s.set_state(prim)
    o = Oracle(path, d, name)
    for call in range(2):  # two calls in a row, on two different states
        s.explicit_solve(1)
        o.run(1)
        s.convective_calculate()
        expect = s.get("residual").reshape(g.nvol, g.dim + 2)[:nint]
        got = _call(g, sc, _prim_soa(s, g, sc), tensors, torch)
        assert np.all(np.isfinite(got))
        assert np.array_equal(got, expect), "call %d" % (call + 1)
        assert np.array_equal(got, o.convective()[:nint]), "call %d vs the oracle" % (call + 1)


def test_static_residual_rejects_meshes_above_its_buffer():
    """Sizes beyond PSST_STATIC_MAX_FACES are rejected before any device work."""
    L = _lib.load()
    too_many = 131072 + 1
    st = L.psst_convective_residual_static(2, 3, 10, 20, too_many, *([None] * 7), 287.0, 1004.5, 717.5, 1.4,
                                           None, None)
    assert st == 1
    assert "PSST_STATIC_MAX_FACES" in L.psst_last_error().decode()
    with pytest.raises(PsstError):
        _lib.check(st)
