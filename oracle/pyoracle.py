"""ctypes front end for the oracle (TEST INFRASTRUCTURE ONLY).

Only tests/, __graft_entry__.smoke() and bench.py's cpu_baseline leg import
this module. It exposes
  * ``Oracle``: the C restatement in psst_oracle.c (built into _build/), and
  * ``run_reference``: the reference itself, compiled in place from its own
    sources into _ref/ (available only where it was built).
"""
import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
BUILD = os.path.join(HERE, "_build")
REF = os.path.join(HERE, "_ref")

_lib = None


def build(quiet=True):
    """Builds the C restatement (and the compiled reference when its sources exist)."""
    out = subprocess.run(["make", "-C", HERE, "-j8"], capture_output=True, text=True)
    if out.returncode != 0:
        raise RuntimeError("oracle build failed:\n" + out.stdout + out.stderr)
    if not quiet:
        print(out.stdout)


def lib():
    global _lib
    if _lib is None:
        path = os.path.join(BUILD, "liboracle.so")
        if not os.path.exists(path):
            build()
        L = ctypes.CDLL(path)
        L.oracle_open.restype = ctypes.c_void_p
        L.oracle_open.argtypes = [ctypes.c_char_p] * 3 + [ctypes.c_char_p, ctypes.c_int]
        L.oracle_set.argtypes = [ctypes.c_void_p, ctypes.c_char_p, ctypes.c_double]
        L.oracle_run.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p]
        L.oracle_error.restype = ctypes.c_char_p
        L.oracle_error.argtypes = [ctypes.c_void_p]
        for f in ("oracle_dim", "oracle_nvol", "oracle_nface", "oracle_iter"):
            getattr(L, f).argtypes = [ctypes.c_void_p]
        L.oracle_get.restype = ctypes.c_long
        L.oracle_get.argtypes = [ctypes.c_void_p, ctypes.c_char_p, ctypes.c_void_p, ctypes.c_long]
        L.oracle_set_prim.argtypes = [ctypes.c_void_p] * 4
        L.oracle_write_sav.argtypes = [ctypes.c_void_p, ctypes.c_char_p]
        L.oracle_close.argtypes = [ctypes.c_void_p]
        L.oracle_convective.argtypes = [ctypes.c_void_p]
        _lib = L
    return _lib


class OracleError(RuntimeError):
    pass


class Oracle:
    """The C restatement of the reference, opened on one mesh + case."""

    def __init__(self, mesh, case_dir, case_name, **options):
        L = lib()
        err = ctypes.create_string_buffer(512)
        h = L.oracle_open(str(mesh).encode(), str(case_dir).encode(), case_name.encode(), err, 512)
        if not h:
            raise OracleError(err.value.decode())
        self._h = h
        self.dim = L.oracle_dim(h)
        self.nv = self.dim + 2
        for k, v in options.items():
            if L.oracle_set(h, k.encode(), float(v)) != 0:
                raise OracleError(L.oracle_error(h).decode())

    def run(self, n_iter):
        L = lib()
        linf = np.zeros((n_iter, self.nv))
        l2 = np.zeros((n_iter, self.nv))
        if L.oracle_run(self._h, n_iter, linf.ctypes.data, l2.ctypes.data) != 0:
            raise OracleError(L.oracle_error(self._h).decode())
        return linf, l2

    def convective(self):
        """One stage's convective residual of the current state, (nvol, dim+2)
        in the reference's component order; the state is not changed."""
        if lib().oracle_convective(self._h) != 0:
            raise OracleError(lib().oracle_error(self._h).decode())
        return self.get("vol_res").reshape(-1, self.nv)

    def get(self, name):
        L = lib()
        n = L.oracle_get(self._h, name.encode(), None, 0)
        if n < 0:
            raise KeyError(name)
        a = np.zeros(n)
        L.oracle_get(self._h, name.encode(), a.ctypes.data, n)
        return a

    @property
    def iter(self):
        return lib().oracle_iter(self._h)

    def set_prim(self, p, T, u):
        p = np.ascontiguousarray(p, dtype=np.float64)
        T = np.ascontiguousarray(T, dtype=np.float64)
        u = np.ascontiguousarray(u, dtype=np.float64)
        lib().oracle_set_prim(self._h, p.ctypes.data, T.ctypes.data, u.ctypes.data)

    def write_sav(self, path):
        if lib().oracle_write_sav(self._h, str(path).encode()) != 0:
            raise OracleError("cannot write " + str(path))

    def close(self):
        if self._h:
            lib().oracle_close(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def reference_available():
    return os.path.exists(os.path.join(REF, "ref_dump"))


def run_reference(mesh, case_dir, case_name, outdir):
    """Runs the compiled reference (ref_dump) in case_dir; returns its arrays."""
    os.makedirs(outdir, exist_ok=True)
    exe = os.path.join(REF, "ref_dump")
    r = subprocess.run([exe, os.path.abspath(mesh), case_name, os.path.abspath(outdir)],
                       cwd=case_dir, capture_output=True, text=True)
    if r.returncode != 0:
        raise OracleError("reference failed: " + r.stderr[-2000:])
    out = {}
    for f in os.listdir(outdir):
        if f.endswith(".npy"):
            out[f[:-4]] = np.load(os.path.join(outdir, f))
    return out
