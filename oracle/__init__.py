"""TEST INFRASTRUCTURE ONLY: ctypes binding of the CPU oracle.

The oracle (sphdem_oracle.c) is a plain-C FP64 restatement of the
reference ISPH-DEM step.  tests/, __graft_entry__.smoke() and bench.py's
CPU-baseline leg use it as the checker; the engine never calls it.
"""
import ctypes as C
import os
import subprocess

import numpy as np

from fluidized_bed_master_b200.params import DEM, F, INT_FIELDS, SPH, SphdemParams

_HERE = os.path.dirname(os.path.abspath(__file__))
# Where the reference sources lie on a machine that has them (the fixture and
# reference-build recipes read them there).  The one place this path is named
# besides oracle/Makefile's default.
REFERENCE_DIR = os.environ.get("SPHDEM_REFERENCE_DIR", "/root/reference")
LIB_PATH = os.path.join(_HERE, "_build", "liboracle.so")
_lib = None


def build():
    subprocess.run(["make", "-s", "-C", _HERE, "_build/liboracle.so"], check=True)


def lib():
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        build()
    L = C.CDLL(LIB_PATH)
    vp = C.c_void_p
    P = C.POINTER
    L.oracle_create.argtypes = [P(SphdemParams), C.c_int, C.c_int]
    L.oracle_create.restype = vp
    L.oracle_destroy.argtypes = [vp]
    L.oracle_destroy.restype = None
    L.oracle_set_field.argtypes = [vp, C.c_int, C.c_int, vp, C.c_int]
    L.oracle_get_field.argtypes = [vp, C.c_int, C.c_int, vp, C.c_int]
    L.oracle_commit.argtypes = [vp]
    L.oracle_set_domain.argtypes = [vp, P(C.c_double), P(C.c_double), C.c_double]
    L.oracle_set_beds.argtypes = [vp, C.c_int, P(C.c_double)]
    L.oracle_step.argtypes = [vp, C.c_int]
    L.oracle_get_neighbors.argtypes = [vp, P(C.c_int), P(C.c_int), C.c_int]
    L.oracle_get_grid.argtypes = [vp, P(C.c_int), P(C.c_double), P(C.c_double)]
    L.oracle_get_time.argtypes = [vp, P(C.c_double), P(C.c_int)]
    L.oracle_get_history.argtypes = [vp, P(C.c_double), P(C.c_double), C.c_int]
    L.oracle_set_history.argtypes = [vp, P(C.c_double), P(C.c_double), C.c_int]
    L.oracle_set_threads.argtypes = [vp, C.c_int]
    L.oracle_get_ppe.argtypes = [vp, P(C.c_int), P(C.c_double), P(C.c_int)]
    _lib = L
    return L


_BED_KEYS = ("y", "inlet_uz", "inlet_temp", "obc_L1", "obc_L2", "obc_L3", "obc_L4")


class Oracle:
    def __init__(self, params, sph, dem, threads=1, beds=None, domain=None):
        """beds: per-bed rows of 2-D beds in planes y = const (dicts with
        the keys of the engine's BedRow), as Engine(beds=...).  domain:
        (bbox6, h0, ...) fixing the cell grid, as Engine(domain=...)."""
        L = lib()
        self.ns = len(sph["x"]) if sph else 0
        self.nd = len(dem["x"]) if dem else 0
        self.params = params.copy()
        self._h = L.oracle_create(C.byref(self.params), self.ns, self.nd)
        if not self._h:
            raise MemoryError("oracle_create failed")
        L.oracle_set_threads(self._h, int(threads))
        if domain is not None:
            bb = [float(v) for v in domain[0]]
            mins = (C.c_double * 3)(bb[0], bb[2], bb[4])
            maxs = (C.c_double * 3)(bb[1], bb[3], bb[5])
            L.oracle_set_domain(self._h, mins, maxs, float(domain[1]))
        if beds is not None:
            rows = np.ascontiguousarray([[float(r[k]) for k in _BED_KEYS] for r in beds], dtype=np.float64)
            if L.oracle_set_beds(self._h, len(beds), rows.ctypes.data_as(C.POINTER(C.c_double))) != 0:
                raise ValueError("oracle_set_beds")
        for which, d in ((SPH, sph), (DEM, dem)):
            for name, arr in (d or {}).items():
                self._set(which, name, arr)
        if L.oracle_commit(self._h) != 0:
            raise RuntimeError("oracle_commit failed")

    def _set(self, which, name, arr):
        n = self.nd if which == DEM else self.ns
        dt = np.int32 if name in INT_FIELDS else np.float64
        a = np.ascontiguousarray(arr, dtype=dt)
        if lib().oracle_set_field(self._h, which, F[name], a.ctypes.data, n) != 0:
            raise ValueError(f"oracle_set_field({name})")

    def step(self, n=1):
        if lib().oracle_step(self._h, int(n)) != 0:
            raise RuntimeError("oracle_step failed")

    def get(self, which, name):
        n = self.nd if which == DEM else self.ns
        dt = np.int32 if name in INT_FIELDS else np.float64
        a = np.empty(n, dtype=dt)
        if lib().oracle_get_field(self._h, which, F[name], a.ctypes.data, n) != 0:
            raise ValueError(f"oracle_get_field({name})")
        return a

    def neighbors(self, cap=512):
        counts = np.zeros(self.ns, dtype=np.int32)
        lst = np.full((self.ns, cap), -1, dtype=np.int32)
        lib().oracle_get_neighbors(self._h, counts.ctypes.data_as(C.POINTER(C.c_int)),
                                   lst.ctypes.data_as(C.POINTER(C.c_int)), cap)
        return counts, lst

    def grid(self):
        nijk = (C.c_int * 3)()
        bb = (C.c_double * 6)()
        dc = C.c_double()
        lib().oracle_get_grid(self._h, nijk, bb, C.byref(dc))
        return list(nijk), list(bb), dc.value

    def time(self):
        t, c = C.c_double(), C.c_int()
        lib().oracle_get_time(self._h, C.byref(t), C.byref(c))
        return t.value, c.value

    def history(self):
        ct = np.zeros((self.nd, 16))
        ds = np.zeros((self.nd, 16, 3))
        lib().oracle_get_history(self._h, ct.ctypes.data_as(C.POINTER(C.c_double)),
                                 ds.ctypes.data_as(C.POINTER(C.c_double)), self.nd)
        return ct, ds

    def ppe(self):
        """(iterations, relative residual, status) of the last Krylov PPE solve."""
        it, res, st = C.c_int(), C.c_double(), C.c_int()
        lib().oracle_get_ppe(self._h, C.byref(it), C.byref(res), C.byref(st))
        return it.value, res.value, st.value

    def close(self):
        if getattr(self, "_h", None):
            lib().oracle_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
