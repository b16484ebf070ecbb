"""supersonicflowsolver_b200: PSST's explicit finite-volume loop on NVIDIA B200.

The solver itself is libpsst_b200.so (C ABI: include/psst_b200.h): a C++ host
that reads the reference's Fluent meshes and setup files, and hand-written
sm_100a CUDA kernels for gradients, reconstruction/limiters, HLL/HLLC/AUSM
fluxes, local time step, Runge-Kutta update and boundary conditions.
"""
from . import meshgen  # noqa: F401  (pure numpy; no library needed)

__version__ = "0.1.0"


def __getattr__(name):
    # the solver API needs the built library; import it lazily so that mesh
    # generation works on machines that only build.
    if name in ("Grid", "Solver", "GridFV", "Scheme", "PsstError"):
        from . import psst

        return getattr(psst, name)
    raise AttributeError(name)
