import os
import subprocess
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def _reference_dir():
    """The reference checkout (its meshes and shipped outputs), if present:
    PSST_REFERENCE_DIR, else the directory the build compiled the reference
    from (noted by __graft_entry__.build), else none."""
    d = os.environ.get("PSST_REFERENCE_DIR")
    note = os.path.join(ROOT, "oracle", "_build", "reference_dir")
    if not d and os.path.exists(note):
        d = open(note).read().strip()
    return d if d and os.path.isdir(d) else ""


REFERENCE_DIR = _reference_dir()


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200)")
    config.addinivalue_line("markers", "slow: takes more than ~20 s on CPU")


def _ensure_built():
    lib = os.path.join(ROOT, "supersonicflowsolver_b200", "_build", "libpsst_b200.so")
    orc = os.path.join(ROOT, "oracle", "_build", "liboracle.so")
    if not (os.path.exists(lib) and os.path.exists(orc)):
        import __graft_entry__

        __graft_entry__.build()


_ensure_built()


def walls(mesh):
    return [z.name for z in mesh.face_zones if z.bc_type not in (2, 31) and z.name not in ("in", "out", "side")]


def make_case(tmpdir, mesh, name="t", **kw):
    """Writes mesh + case files into tmpdir; returns (mesh_path, dir, name)."""
    from supersonicflowsolver_b200 import meshgen

    d = str(tmpdir)
    path = os.path.join(d, "m.msh")
    meshgen.write_fluent(mesh, path)
    meshgen.write_case(d, name, dim=mesh.dim, zones=walls(mesh), **kw)
    return path, d, name


def oracle_prim(o, nvol, dim):
    """Oracle state in the C ABI's SoA layout (p, T, u0.., u1..)."""
    return np.concatenate([o.get("vol_p"), o.get("vol_T"), o.get("vol_u").reshape(nvol, dim).T.ravel()])


def reference_available():
    from oracle import pyoracle

    return pyoracle.reference_available()


def cuda_available():
    try:
        import torch

        return torch.cuda.is_available()
    except Exception:
        return False
