"""Packs the reference's own published wedge case as a test fixture.

The reference ships one solved case: the mesh wedge80_240.msh (named by its
problem_manager), the setup files wedge.inp/.prop/.par/.bvp/.btq (HLL, first
order, LocalAccTime1, RK1, CFL 2.08, 3000 iterations), and the outputs it
wrote: wedge.sav (state after 3000 iterations) and wedge_residual.dat (the
residual columns of every iteration, with the authors' wall-clock times).

This script copies those files -- data, not source code -- with line endings
normalised to LF (the reference's own reader needs LF meshes) into
tests/golden/shipped_wedge/, xz-compressing the large ones, so that the GPU
tests can check the solver against the reference's published output on a
machine without the reference sources.

    python tests/golden/make_shipped_wedge.py <reference checkout>
"""
import lzma
import os
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
OUT = os.path.join(HERE, "shipped_wedge")

SMALL = ["wedge.inp", "wedge.prop", "wedge.par", "wedge.bvp", "wedge.btq"]
LARGE = ["wedge80_240.msh", "wedge.sav", "wedge_residual.dat"]


def main(ref):
    os.makedirs(OUT, exist_ok=True)
    for name in SMALL + LARGE:
        with open(os.path.join(ref, name), "rb") as f:
            data = f.read().replace(b"\r", b"")
        if name in LARGE:
            with lzma.open(os.path.join(OUT, name + ".xz"), "wb", preset=9) as f:
                f.write(data)
        else:
            with open(os.path.join(OUT, name), "wb") as f:
                f.write(data)


def unpack(dest):
    """Writes the fixture's files (decompressed) into dest; returns the paths
    of the mesh, the shipped .sav and the shipped residual log."""
    for name in SMALL:
        with open(os.path.join(OUT, name), "rb") as f, open(os.path.join(dest, name), "wb") as g:
            g.write(f.read())
    paths = []
    for name in LARGE:
        with lzma.open(os.path.join(OUT, name + ".xz"), "rb") as f:
            data = f.read()
        p = os.path.join(dest, ("shipped_" + name) if name != "wedge80_240.msh" else name)
        with open(p, "wb") as g:
            g.write(data)
        paths.append(p)
    return tuple(paths)


def residual_columns(path):
    """The four residual columns (rho*u, rho*v, rho, rho*E) of a _residual.dat."""
    import numpy as np

    rows = [l.split() for l in open(path).read().splitlines() if l.strip()]
    return np.array([[float(x) for x in r[2:]] for r in rows])


if __name__ == "__main__":
    main(sys.argv[1])
