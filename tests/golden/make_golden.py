"""Generates the golden fixtures in this directory from the reference itself.

Each fixture is the FP64 state after N iterations computed by the PSST
reference (compiled in place from its own sources by oracle/Makefile and run
through oracle/ref_dump) on a seeded synthetic mesh, plus the residual columns
the reference printed. The mesh and case files are regenerated from the stored
parameters, so the fixtures stay small and need no reference files at test time.

Usage (needs oracle/_ref, i.e. the reference sources at build time):
    python tests/golden/make_golden.py [fixture names; default: all]
"""
import json
import os
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from oracle.pyoracle import run_reference  # noqa: E402
from supersonicflowsolver_b200 import meshgen  # noqa: E402

# name -> (mesh builder kwargs, case kwargs, iterations)
GOLDEN = {
    "g2d_hllc_dm_vanleer_rk4": ({"kind": "wedge2d", "nx": 40, "ny": 12, "angle_deg": 15.0},
                                {"flux": 3, "order": 2, "limiter": 3, "grad": 1, "lc": 1, "rk_level": 4,
                                 "cfl": 0.5, "mach": 2.5}, 20),
    "g2d_jitter_ausm_lsq_vanalbada": ({"kind": "wedge2d", "nx": 30, "ny": 10, "angle_deg": 15.0, "jitter": 0.15,
                                       "seed": 0, "shuffle_seed": 1, "interior_first": True},
                                      {"flux": 1, "order": 2, "limiter": 1, "grad": 2, "lc": 2, "rk_level": 3,
                                       "cfl": 0.5, "mach": 2.5}, 20),
    "g3d_tet_hllc_dm_vanleer": ({"kind": "wedge3d", "nx": 10, "ny": 5, "nz": 3, "angle_deg": 12.0, "tets": True},
                                {"flux": 3, "order": 2, "limiter": 3, "grad": 1, "lc": 1, "rk_level": 4,
                                 "cfl": 0.5, "mach": 3.0}, 5),
    "g2d_hll_first_order_rk1": ({"kind": "wedge2d", "nx": 40, "ny": 12, "angle_deg": 15.0},
                                {"flux": 2, "order": 1, "limiter": 3, "grad": 1, "lc": 1, "rk_level": 1,
                                 "cfl": 2.08, "mach": 2.5}, 100),
    # the reference's 2D case at its own size: 120 x 40 quads (the layout of
    # its wedge40_120.msh), HLLC, DM + VanLeer, RK4, CFL 0.5, LocalAccTime1 in
    # its in-loop order, 2000 iterations
    "g2d_c1_120x40_hllc_dm_vanleer_rk4_2000": ({"kind": "wedge2d", "nx": 120, "ny": 40, "angle_deg": 15.0},
                                               {"flux": 3, "order": 2, "limiter": 3, "grad": 1, "lc": 1,
                                                "rk_level": 4, "cfl": 0.5, "mach": 2.5}, 2000),
    # hanging-node mesh: parent cells and faces, quads with five faces
    "g2d_adapted_hllc_lsq_vanleer": ({"kind": "wedge2d_adapted", "nx": 40, "ny": 12, "angle_deg": 15.0,
                                      "refine_frac": 0.2, "seed": 3},
                                     {"flux": 3, "order": 2, "limiter": 3, "grad": 2, "lc": 2, "rk_level": 4,
                                      "cfl": 0.5, "mach": 2.5}, 20),
}


def build_mesh(spec):
    spec = dict(spec)
    kind = spec.pop("kind")
    return getattr(meshgen, kind)(**spec)


def write_inputs(d, mesh_spec, case_kw, n_iter, name="g"):
    mesh = build_mesh(mesh_spec)
    path = os.path.join(d, "m.msh")
    meshgen.write_fluent(mesh, path)
    zones = [z.name for z in mesh.face_zones if z.bc_type not in (2, 31) and z.name not in ("in", "out", "side")]
    meshgen.write_case(d, name, dim=mesh.dim, zones=zones, max_iter=n_iter, **case_kw)
    return mesh, path


def main(names=()):
    for key, (mspec, ckw, n) in GOLDEN.items():
        if names and key not in names:
            continue
        with tempfile.TemporaryDirectory() as d:
            mesh, path = write_inputs(d, mspec, ckw, n)
            out = run_reference(path, d, "g", os.path.join(d, "dump"))
            interior = out["vol_bc"] == 1  # interior cells (not ghosts, not parent cells)
            dim = int(out["dim"][0])
            res = np.loadtxt(os.path.join(d, "g_residual.dat"))
            np.savez_compressed(
                os.path.join(HERE, key + ".npz"),
                params=json.dumps({"mesh": mspec, "case": ckw, "iterations": n}),
                p=out["vol_p"][interior], T=out["vol_T"][interior],
                u=out["vol_u"].reshape(-1, dim)[interior], residual_columns=res[:, 2:])
            print(key, int(interior.sum()), "cells")


if __name__ == "__main__":
    main(sys.argv[1:])
