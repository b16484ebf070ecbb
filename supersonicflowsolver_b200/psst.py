"""Python host API over libpsst_b200, mirroring the reference's interfaces.

Reference (C++)                                   here
------------------------------------------------  ------------------------------------------
psstAnsysDirector::construct_grid +                Grid.read_fluent(path)
  psstAnsysInputGrid::create_finite_volume_grid
  (psstAnsysGridReader.cpp:688-907, 1308-1317)
psstGridFV::solver_parameters (:36-194)            Grid.read_case(dir, name) -> (Scheme, prim)
psstInterfaceGradientCalc::calculate               Solver.gradient_calculate()
psstInterfaceConvectiveFlow::calculate             Solver.convective_calculate()
LocalTime + RK update + boundary conditions        Solver.stage_update(k)
  (psstFiniteVolumeGrid.cpp:312-366)
psstGridFV::explicit_solve loop (:305-397)         Solver.explicit_solve(n)
main.cpp                                           GridFV (same files in, same files out)

Errors raise PsstError carrying the reference's message where the reference
reports the same condition (e.g. "Error: Could not found zone!").
"""
import ctypes
import os
import time

import numpy as np

from . import _lib, meshgen
from ._lib import PsstError, Scheme, check

__all__ = ["Grid", "Solver", "GridFV", "Scheme", "PsstError"]


def _ptr(a):
    return a.ctypes.data_as(ctypes.c_void_p)


class Grid:
    """Finite-volume grid in the reference's storage order (host memory)."""

    def __init__(self, handle):
        self._h = handle
        self._info = _lib.GridInfo()
        check(_lib.load().psst_grid_get_info(self._h, ctypes.byref(self._info)))

    @classmethod
    def read_fluent(cls, path):
        h = ctypes.c_void_p()
        check(_lib.load().psst_grid_read_fluent(str(path).encode(), ctypes.byref(h)))
        return cls(h)

    @classmethod
    def from_mesh(cls, mesh):
        """From an in-memory meshgen.Mesh (no file round trip)."""
        L = _lib.load()
        fz = mesh.face_zones
        k = [z.nodes.shape[1] for z in fz]
        counts = np.concatenate([np.full(len(z.c0), kk, dtype=np.int64) for z, kk in zip(fz, k)])
        face_ptr = np.zeros(len(counts) + 1, dtype=np.int64)
        np.cumsum(counts, out=face_ptr[1:])
        nodes = np.ascontiguousarray(np.concatenate([z.nodes.ravel() for z in fz]).astype(np.int64))
        c0 = np.ascontiguousarray(np.concatenate([z.c0 for z in fz]).astype(np.int64))
        c1 = np.ascontiguousarray(np.concatenate([z.c1 for z in fz]).astype(np.int64))
        verts = np.ascontiguousarray(mesh.verts, dtype=np.float64)
        zones = (_lib.ZoneDesc * (len(fz) + 2))()
        first = 1
        names = []
        for i, z in enumerate(fz):
            n = len(z.c0)
            names.append(z.name.encode())
            zones[i] = _lib.ZoneDesc(z.zone_id, z.bc_type, first, first + n - 1, names[-1])
            first += n
        names.append(b"fluid")
        zones[len(fz)] = _lib.ZoneDesc(2, 1, 1, mesh.ncells, names[-1])
        nz = len(fz) + 1
        if mesh.nparents:  # adapted mesh: the parent cells' zone (its trees stay with the file form)
            zones[nz] = _lib.ZoneDesc(meshgen.PARENT_CELL_ZONE, 32, mesh.ncells + 1, mesh.ncells + mesh.nparents,
                                      b"")
            nz += 1
        d = _lib.FluentDesc(mesh.dim, len(verts), verts.ctypes.data, len(c0), face_ptr.ctypes.data,
                            nodes.ctypes.data, c0.ctypes.data, c1.ctypes.data, mesh.ncells + mesh.nparents, nz,
                            ctypes.cast(zones, ctypes.POINTER(_lib.ZoneDesc)))
        h = ctypes.c_void_p()
        check(L.psst_grid_from_fluent(ctypes.byref(d), ctypes.byref(h)))
        return cls(h)

    @property
    def dim(self):
        return self._info.dim

    @property
    def nvol(self):
        return self._info.nvol

    @property
    def ninterior(self):
        return self._info.ninterior

    @property
    def nghost(self):
        return self._info.nghost

    @property
    def nface(self):
        return self._info.nface

    @property
    def min_vol(self):
        return self._info.min_vol

    _INT = {"face_c0", "face_c1", "face_zone", "vol_zone", "vol_boundary", "vol_bc"}
    _SIZES = {"vol_V": ("nvol", 1), "vol_x": ("nvol", "dim"), "face_S": ("nface", 1),
              "face_n": ("nface", "dim"), "face_x": ("nface", "dim"), "face_beta": ("nface", 1),
              "face_c0": ("nface", 1), "face_c1": ("nface", 1), "face_zone": ("nface", 1),
              "vol_zone": ("nvol", 1), "vol_boundary": ("nvol", 1),
              "vol_bc": ("nvol", 1)}

    def get(self, name):
        n, w = self._SIZES[name]
        count = getattr(self, n) * (self.dim if w == "dim" else 1)
        out = np.zeros(count, dtype=np.int64 if name in self._INT else np.float64)
        check(_lib.load().psst_grid_get_array(self._h, name.encode(), _ptr(out), count))
        return out

    def read_case(self, directory, name):
        """psstGridFV::solver_parameters: returns (Scheme, prim[(2+dim)*nvol])."""
        sc = Scheme()
        prim = np.zeros((2 + self.dim) * self.nvol)
        check(_lib.load().psst_case_read(self._h, str(directory).encode(), name.encode(), ctypes.byref(sc),
                                         _ptr(prim)))
        return sc, prim

    @classmethod
    def merge(cls, grids):
        """Disjoint union of case grids (each set up by read_case) for batched
        solving; see psst_grid_merge."""
        arr = (ctypes.c_void_p * len(grids))(*[g._h.value for g in grids])
        h = ctypes.c_void_p()
        check(_lib.load().psst_grid_merge(arr, len(grids), ctypes.byref(h)))
        return cls(h)

    def cases(self):
        """Volume offsets of the cases (length ncase + 1)."""
        n = ctypes.c_int32()
        check(_lib.load().psst_grid_case_count(self._h, ctypes.byref(n), None))
        ptr = np.zeros(n.value + 1, dtype=np.int64)
        check(_lib.load().psst_grid_case_count(self._h, ctypes.byref(n), _ptr(ptr)))
        return ptr

    def initial_state(self):
        """The state read by read_case (for a merged grid: all cases')."""
        prim = np.zeros((2 + self.dim) * self.nvol)
        check(_lib.load().psst_grid_initial_state(self._h, _ptr(prim), prim.size))
        return prim

    def write_fluent(self, prim, rho, prefix):
        """<prefix>.cas and <prefix>.dat as PSST's output manager writes them."""
        prim = np.ascontiguousarray(prim, dtype=np.float64)
        rho = np.ascontiguousarray(rho, dtype=np.float64)
        check(_lib.load().psst_write_fluent(self._h, _ptr(prim), _ptr(rho), str(prefix).encode()))

    def set_boundary(self, zone, dyn_id, u=None, p=0.0, therm_id=18, T=0.0):
        ua = np.zeros(3) if u is None else np.ascontiguousarray(u, dtype=np.float64)
        check(_lib.load().psst_grid_set_boundary(self._h, zone.encode(), dyn_id, _ptr(ua), p, therm_id, T))

    def close(self):
        if getattr(self, "_h", None):
            _lib.load().psst_grid_free(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Solver:
    """Device state of one case on one GPU (psst_solver)."""

    def __init__(self, grid, scheme, device=0):
        self.grid = grid
        self.scheme = scheme
        self.dim = grid.dim
        self.nv = grid.dim + 2
        h = ctypes.c_void_p()
        check(_lib.load().psst_solver_create(grid._h, ctypes.byref(scheme), int(device), ctypes.byref(h)))
        self._h = h

    def set_state(self, prim):
        prim = np.ascontiguousarray(prim, dtype=np.float64)
        if prim.size != (2 + self.dim) * self.grid.nvol:
            raise ValueError("prim must hold (2+dim)*nvol values")
        check(_lib.load().psst_solver_set_state(self._h, _ptr(prim)))

    def get_state(self, with_w=False, out=None):
        """prim (and w) in the reference's volume order; `out` (optional, e.g.
        a pinned buffer) receives prim."""
        prim = out if out is not None else np.empty((2 + self.dim) * self.grid.nvol)
        if prim.dtype != np.float64 or prim.size != (2 + self.dim) * self.grid.nvol or not prim.flags.c_contiguous:
            raise ValueError("out must be a contiguous float64 array of (2+dim)*nvol values")
        w = np.zeros(self.nv * self.grid.nvol) if with_w else None
        check(_lib.load().psst_solver_get_state(self._h, _ptr(prim), _ptr(w) if with_w else None))
        return (prim, w) if with_w else prim

    def save_checkpoint(self, path):
        """Full-precision state + iteration counter (exact resume; see
        psst_solver_save_checkpoint)."""
        check(_lib.load().psst_solver_save_checkpoint(self._h, str(path).encode()))

    def load_checkpoint(self, path):
        check(_lib.load().psst_solver_load_checkpoint(self._h, str(path).encode()))

    def gradient_calculate(self):
        check(_lib.load().psst_gradient_calculate(self._h))

    def convective_calculate(self):
        check(_lib.load().psst_convective_calculate(self._h))

    def stage_update(self, k):
        r = np.zeros(self.nv)
        check(_lib.load().psst_stage_update(self._h, int(k), _ptr(r)))
        return r

    def explicit_solve(self, n_iter):
        """n iterations; returns (linf, l2), each (n_iter, dim+2)."""
        linf = np.zeros((n_iter, self.nv))
        l2 = np.zeros((n_iter, self.nv))
        check(_lib.load().psst_explicit_solve(self._h, int(n_iter), _ptr(linf), _ptr(l2)))
        return linf, l2

    _ARR = {"rho": 1, "dt": 1, "residual": "nv", "grad_u": "dd", "grad_p": "d", "grad_T": "d"}

    def get(self, name):
        w = self._ARR[name]
        per = {1: 1, "nv": self.nv, "dd": self.dim * self.dim, "d": self.dim}[w]
        out = np.zeros(per * self.grid.nvol)
        check(_lib.load().psst_solver_get_array(self._h, name.encode(), _ptr(out), out.size))
        return out

    KERNEL_KINDS = ("gradient", "face", "cell", "ghost_update", "norm_finish")

    def profile(self, n_iter):
        """n iterations with a CUDA event pair around every launch; returns
        {kind: (total_ms, launches)}."""
        ms = np.zeros(len(self.KERNEL_KINDS))
        cnt = np.zeros(len(self.KERNEL_KINDS), dtype=np.int64)
        check(_lib.load().psst_solver_profile(self._h, int(n_iter), _ptr(ms), _ptr(cnt)))
        return {k: (float(ms[i]), int(cnt[i])) for i, k in enumerate(self.KERNEL_KINDS)}

    def autotune(self, n_iter=3):
        """Times n_iter iterations at each launch shape (64/128/256 threads per
        block), keeps the fastest per pass and restores the state; returns
        {"gradient": b, "face": b, "cell": b}."""
        out = np.zeros(3, dtype=np.int32)
        check(_lib.load().psst_solver_autotune(self._h, int(n_iter), _ptr(out)))
        return dict(zip(("gradient", "face", "cell"), (int(x) for x in out)))

    def launch_shape(self, gradient=0, face=0, cell=0):
        """Sets the launch shapes (0 keeps one) and returns the current ones."""
        st = np.array([gradient, face, cell], dtype=np.int32)
        out = np.zeros(3, dtype=np.int32)
        check(_lib.load().psst_solver_launch_shape(self._h, _ptr(st), _ptr(out)))
        return dict(zip(("gradient", "face", "cell"), (int(x) for x in out)))

    def use_graphs(self, on=True):
        """Capture each explicit_solve call as a CUDA graph and replay it."""
        check(_lib.load().psst_solver_use_graphs(self._h, int(bool(on))))
        self.graphs_on = bool(on)

    graphs_on = False

    def use_wavefront(self, on=True):
        """Sequential LocalAccTime1 as one persistent launch per call (default
        on) or level by level, stage by stage (off); same results."""
        check(_lib.load().psst_solver_use_wavefront(self._h, int(bool(on))))

    def set_wait_limit(self, nanoseconds):
        """Bound of each device-side wait of the persistent launch (< 0: default)."""
        check(_lib.load().psst_solver_set_wait_limit(self._h, int(nanoseconds)))

    def schedule_info(self):
        """{"wavefront": bool, "period": P, "levels": n, "items": n, "blocks": n}."""
        out = np.zeros(5, dtype=np.int64)
        check(_lib.load().psst_solver_schedule_info(self._h, _ptr(out)))
        return {"wavefront": bool(out[0]), "period": int(out[1]), "levels": int(out[2]), "items": int(out[3]),
                "blocks": int(out[4])}

    def set_active(self, flags):
        """Merged grids: per-case run flags (stopped cases keep their state)."""
        a = np.ascontiguousarray(np.asarray(flags, dtype=np.int32))
        check(_lib.load().psst_solver_set_active(self._h, _ptr(a)))

    def case_residuals(self, n_iter):
        """Merged grids: per-case residual columns of the last explicit_solve,
        shape (n_iter, ncase, dim+2)."""
        ncase = len(self.grid.cases()) - 1
        out = np.zeros((n_iter, ncase, self.nv))
        check(_lib.load().psst_solver_case_residuals(self._h, int(n_iter), _ptr(out)))
        return out

    def set_stop_rule(self, drop, scale_iters=5, scales=None, caps=None):
        """Merged grids: the per-case stop rule evaluated on the device after
        every iteration (drop <= 0 switches it off); see psst_solver_set_stop_rule."""
        ncase = len(self.grid.cases()) - 1
        sc = None if scales is None else np.ascontiguousarray(np.asarray(scales, dtype=np.float64).reshape(ncase, self.nv))
        cp = None if caps is None else np.ascontiguousarray(np.asarray(caps, dtype=np.int32).reshape(ncase))
        check(_lib.load().psst_solver_set_stop_rule(self._h, float(drop), int(scale_iters),
                                                    None if sc is None else _ptr(sc), None if cp is None else _ptr(cp)))

    def run_to_stop(self, max_iter, chunk=100, history=True):
        """Merged grids with a stop rule: iterates until every case has stopped
        (or max_iter iterations) as one CUDA-graph launch whose while-loop node
        the device ends; see psst_solver_run_to_stop. Returns (iterations run,
        linf, l2), the residual columns [n][dim+2] of those iterations (None
        without history)."""
        n = ctypes.c_int64()
        li = np.zeros((int(max_iter), self.nv)) if history else None
        l2 = np.zeros((int(max_iter), self.nv)) if history else None
        check(_lib.load().psst_solver_run_to_stop(self._h, int(max_iter), int(chunk), ctypes.byref(n),
                                                  _ptr(li) if history else None, _ptr(l2) if history else None))
        if not history:
            return n.value, None, None
        k = min(n.value, int(max_iter))
        return n.value, li[:k], l2[:k]

    def case_status(self):
        """Merged grids: {"active", "iterations", "converged_at", "scales"} per case."""
        ncase = len(self.grid.cases()) - 1
        act = np.zeros(ncase, dtype=np.int32)
        its = np.zeros(ncase, dtype=np.int32)
        conv = np.zeros(ncase, dtype=np.int32)
        sc = np.zeros((ncase, self.nv))
        check(_lib.load().psst_solver_case_status(self._h, _ptr(act), _ptr(its), _ptr(conv), _ptr(sc)))
        return {"active": act, "iterations": its, "converged_at": conv, "scales": sc}

    def set_stream(self, stream_ptr):
        check(_lib.load().psst_solver_set_stream(self._h, ctypes.c_void_p(stream_ptr)))

    def last_stats(self):
        n = ctypes.c_int64()
        ms = ctypes.c_double()
        check(_lib.load().psst_solver_last_stats(self._h, ctypes.byref(n), ctypes.byref(ms)))
        return n.value, ms.value

    @property
    def iter(self):
        return _lib.load().psst_solver_iter(self._h)

    def close(self):
        if getattr(self, "_h", None):
            _lib.load().psst_solver_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def write_sav(grid, prim, iteration, path):
    """The .sav restart file of psstGridFV::private_save_solution
    (psstFiniteVolumeGrid.cpp:606-639): the iteration, then per interior zone
    (bc 1, ascending id; parent cells skipped) its id, its size and one line
    p T u v (w) per cell, and a closing 0."""
    nv, dim = grid.nvol, grid.dim
    zone, vbc = grid.get("vol_zone"), grid.get("vol_bc")
    with open(path, "w") as f:
        f.write("%d\n" % iteration)
        v = 0
        while v < nv:
            e = v
            while e < nv and zone[e] == zone[v]:
                e += 1
            if vbc[v] == 1:
                f.write("%d\n%d\n" % (zone[v], e - v))
                for i in range(v, e):
                    f.write("%.11f %.11f " % (prim[i], prim[nv + i]))
                    f.write("".join("%.11f " % prim[(2 + k) * nv + i] for k in range(dim)))
                    f.write("\n")
            v = e
        f.write("0")


class GridFV:
    """The reference's driver flow (main.cpp + psstGridFV) on the GPU.

    >>> fv = GridFV.construct(mesh_path)        # Director/Builder + create_finite_volume_grid
    >>> fv.settings_file_name("wedge")          # psstGridFV::settings_file_name
    >>> fv.solver_parameters(directory)         # reads .inp/.prop/.par|.sav/.bvp/.btq
    >>> fv.explicit_solve()                     # iterates, writes <case>_residual.dat and <case>.sav
    """

    def __init__(self, grid):
        self.grid = grid
        self._name = None
        self.solver = None
        self.scheme = None
        self.directory = "."

    @classmethod
    def construct(cls, mesh_path):
        return cls(Grid.read_fluent(mesh_path))

    def settings_file_name(self, name):
        self._name = name

    def solver_parameters(self, directory=".", precision=64, lc1_mode=0, renumber=1, device=0):
        self.directory = str(directory)
        sc, prim = self.grid.read_case(directory, self._name)
        sc.precision = precision
        sc.lc1_mode = lc1_mode
        sc.renumber = renumber
        self.scheme = sc
        self.solver = Solver(self.grid, sc, device)
        self.solver.set_state(prim)

    def save_solution(self, path, iteration):
        """Writes <case>.cas/<case>.dat (psstOutputManager.cpp) and the .sav
        (psstGridFV::save_data, psstFiniteVolumeGrid.cpp:240-245)."""
        prim = self.solver.get_state()
        self.grid.write_fluent(prim, self.solver.get("rho"), path[:-4] if path.endswith(".sav") else path)
        write_sav(self.grid, prim, iteration, path)

    def explicit_solve(self, chunk=1000):
        sc = self.scheme
        it = sc.iter
        res_path = os.path.join(self.directory, self._name + "_residual.dat")
        sav_path = os.path.join(self.directory, self._name + ".sav")
        t0 = time.monotonic()
        with open(res_path, "w" if sc.iter == 1 else "a") as rf:
            while it <= sc.max_iter:
                n = min(chunk, sc.max_iter - it + 1)
                if sc.iter_step > 0:
                    n = min(n, sc.iter_step - (it - 1) % sc.iter_step)
                linf, _ = self.solver.explicit_solve(n)
                sec = int((time.monotonic() - t0) * 1000) / 1000.0
                for i in range(n):
                    rf.write("%d %.11e " % (it, sec) + "".join(" %.3e" % x for x in linf[i]) + "\n")
                    if sc.iter_step > 0 and it % sc.iter_step == 0:
                        self.save_solution(sav_path, it)
                    it += 1
        self.save_solution(sav_path, self.solver.iter)
