"""Python binding of the C ABI in include/sphdem.h (libsphdem.so).

Mirrors the reference's per-step operator: ``Engine.step(n)`` advances n
calls of SOPHIA_single_ISPH (ISPH_Calc_seperate.cuh:13-503) plus the host
loop's ``time += dt; count++`` (ISPH_Calc_seperate.cuh:924-925).  There is
no CPU fallback: if the CUDA library is missing or a call fails, an
exception is raised.
"""
import ctypes as C
import os

import numpy as np

from .params import DEM, F, INT_FIELDS, SPH, STATUS, SphdemParams, SphdemStats

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libsphdem.so")
_lib = None


class SphdemError(RuntimeError):
    def __init__(self, status, what):
        super().__init__(f"{what}: {STATUS.get(status, status)} ({status})")
        self.status = status


def lib():
    """Load libsphdem.so (built in-tree by __graft_entry__.build())."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise RuntimeError(f"{LIB_PATH} is missing: the CUDA extension is not built")
    L = C.CDLL(LIB_PATH)
    P = C.POINTER
    vp = C.c_void_p
    L.sphdem_params_default.argtypes = [P(SphdemParams)]
    L.sphdem_read_solv.argtypes = [C.c_char_p, P(SphdemParams)]
    L.sphdem_create.argtypes = [P(SphdemParams), C.c_int32, C.c_int32, P(vp)]
    L.sphdem_create_from_dir.argtypes = [C.c_char_p, P(SphdemParams), P(vp)]
    L.sphdem_create_batch.argtypes = [P(SphdemParams), C.c_int32, P(C.c_int32), P(vp)]
    L.sphdem_batch_offsets.argtypes = [vp, P(C.c_double)]
    L.sphdem_set_field.argtypes = [vp, C.c_int, C.c_int, vp, C.c_size_t]
    L.sphdem_commit_particles.argtypes = [vp]
    L.sphdem_step.argtypes = [vp, C.c_int32]
    L.sphdem_get_field.argtypes = [vp, C.c_int, C.c_int, vp, C.c_size_t]
    L.sphdem_get_stats.argtypes = [vp, P(SphdemStats)]
    L.sphdem_check.argtypes = [vp]
    L.sphdem_get_neighbors.argtypes = [vp, P(C.c_int32), P(C.c_int32), C.c_int32]
    L.sphdem_get_history.argtypes = [vp, P(C.c_int32), P(C.c_double)]
    L.sphdem_write_vtk_dem.argtypes = [vp, C.c_char_p]
    L.sphdem_write_vtk_fluid.argtypes = [vp, C.c_char_p]
    L.sphdem_snapshot.argtypes = [vp]
    L.sphdem_write_snapshot.argtypes = [vp, C.c_char_p, C.c_char_p]
    L.sphdem_set_history.argtypes = [vp, P(C.c_int32), P(C.c_double)]
    L.sphdem_set_timing.argtypes = [vp, C.c_int]
    L.sphdem_set_graphs.argtypes = [vp, C.c_int]
    L.sphdem_set_concurrency.argtypes = [vp, C.c_int]
    L.sphdem_set_timing_only.argtypes = [vp, C.c_int]
    L.sphdem_set_domain.argtypes = [vp, C.POINTER(C.c_double), C.c_double, C.c_double]
    L.sphdem_set_beds.argtypes = [vp, C.c_int32, C.POINTER(BedRow)]
    L.sphdem_set_list_build.argtypes = [vp, C.c_int32]
    L.sphdem_get_list_build.argtypes = [vp, C.POINTER(C.c_int32)]
    L.sphdem_slab_record_bytes.argtypes = [C.c_int]
    dp = C.POINTER(C.c_double)
    L.sphdem_bed_domain.argtypes = [vp, dp, dp, dp, dp, dp, C.c_int32, dp, dp, dp, dp, C.c_int32, dp, dp, dp]
    L.sphdem_slab_select.argtypes = [vp, C.c_int, C.c_int, C.c_int32, C.c_int32, vp, C.c_int32, C.POINTER(C.c_int32)]
    L.sphdem_slab_export.argtypes = [vp, C.c_int, vp, C.c_int32, vp]
    L.sphdem_slab_keep.argtypes = [vp, C.c_int, C.c_int, C.c_int32, C.c_int32]
    L.sphdem_slab_import.argtypes = [vp, C.c_int, vp, C.c_int32]
    L.sphdem_slab_active.argtypes = [vp, C.c_int, C.POINTER(C.c_int32)]
    L.sphdem_collect_timing.argtypes = [vp]
    L.sphdem_get_timing.argtypes = [vp, C.c_int, C.c_char_p, C.c_int, P(C.c_double), P(C.c_int64)]
    L.sphdem_input_counts.argtypes = [C.c_char_p, P(C.c_int32), P(C.c_int32)]
    L.sphdem_input_column.argtypes = [C.c_char_p, C.c_int, C.c_int, vp, C.c_size_t]
    L.sphdem_write_restart.argtypes = [vp, C.c_char_p]
    L.sphdem_get_time.argtypes = [vp, P(C.c_double), P(C.c_int32)]
    L.sphdem_get_counts.argtypes = [vp, P(C.c_int32), P(C.c_int32)]
    L.sphdem_get_stream.argtypes = [vp, P(vp)]
    L.sphdem_get_launch_count.argtypes = [vp, P(C.c_int64)]
    L.sphdem_set_fields.argtypes = [vp, C.c_int, C.c_int32, P(C.c_int32), P(P(C.c_double))]
    L.sphdem_get_fields.argtypes = [vp, C.c_int, C.c_int32, P(C.c_int32), P(P(C.c_double))]
    L.sphdem_get_mlp_state.argtypes = [vp, P(C.c_float), P(C.c_double), P(C.c_int32)]
    L.sphdem_set_mlp_state.argtypes = [vp, P(C.c_float), P(C.c_double), C.c_int32]
    L.sphdem_mlp_param_count.restype = C.c_int32
    L.sphdem_destroy.argtypes = [vp]
    L.sphdem_destroy.restype = None
    L.sphdem_strerror.argtypes = [C.c_int]
    L.sphdem_strerror.restype = C.c_char_p
    L.sphdem_params_size.argtypes = []
    if L.sphdem_params_size() != C.sizeof(SphdemParams):
        raise RuntimeError("SphdemParams layout mismatch between params.py and libsphdem.so")
    _lib = L
    return L


def _chk(status, what):
    if status != 0:
        raise SphdemError(status, what)


def torch_sync():
    """Finish the work torch queued on the current device (before a handle's
    own stream reads a tensor torch wrote)."""
    import torch

    torch.cuda.current_stream().synchronize()


def bed_domain(params, sph, dem):
    """(bbox6, h0, t_ref) that a handle of the whole bed would compute at
    commit (sphdem_bed_domain): the grid every slab of it must share."""
    L = lib()
    dp = C.POINTER(C.c_double)

    def arr(d, k):
        if not d or k not in d:
            return None, None
        a = np.ascontiguousarray(d[k], dtype=np.float64)
        return a, a.ctypes.data_as(dp)

    keep = []
    ptrs = []
    for d, keys in ((sph, ("x", "y", "z", "h", "temp")), (dem, ("x", "y", "z", "h"))):
        for k in keys:
            a, p = arr(d, k)
            keep.append(a)
            ptrs.append(p)
    ns = len(sph["x"]) if sph else 0
    nd = len(dem["x"]) if dem else 0
    bb = (C.c_double * 6)()
    h0, tr = C.c_double(), C.c_double()
    _chk(L.sphdem_bed_domain(C.byref(params), *ptrs[:5], ns, *ptrs[5:], nd, bb, C.byref(h0), C.byref(tr)),
         "sphdem_bed_domain")
    return list(bb), h0.value, tr.value


def default_params():
    p = SphdemParams()
    _chk(lib().sphdem_params_default(C.byref(p)), "sphdem_params_default")
    return p


def read_solv(path, params=None):
    p = params.copy() if params is not None else default_params()
    _chk(lib().sphdem_read_solv(os.fsencode(path), C.byref(p)), "sphdem_read_solv")
    return p


class BedRow(C.Structure):
    """SphdemBedRow: a 2-D bed's plane and open-boundary parameters."""
    _fields_ = [("y", C.c_double), ("inlet_uz", C.c_double), ("inlet_temp", C.c_double),
                ("obc_L1", C.c_double), ("obc_L2", C.c_double), ("obc_L3", C.c_double), ("obc_L4", C.c_double)]


class Engine:
    """One engine handle on the current CUDA device."""

    def __init__(self, params, sph, dem, domain=None, beds=None, list_build=None):
        """params: SphdemParams; sph/dem: dict field-name -> array in input
        order.  domain: (bbox6, h0, t_ref) of a larger bed this one is a slab
        of (sphdem_set_domain; see bed_domain).  beds: rows (dicts with the
        BedRow fields) of several 2-D beds in their own planes y = const
        (sphdem_set_beds; see beds.bed2d_batch).  list_build: the SPH
        list build (sphdem_set_list_build: 1 per particle, 2/4/8 cells per
        block with a warp per cell, None/0 timed at commit)."""
        L = lib()
        ns = len(sph["x"]) if sph else 0
        nd = len(dem["x"]) if dem else 0
        self._h = C.c_void_p()
        _chk(L.sphdem_create(C.byref(params), ns, nd, C.byref(self._h)), "sphdem_create")
        self.params = params.copy()
        self.ns, self.nd = ns, nd
        self._slot_buf = {}
        try:
            if domain is not None:
                bb = (C.c_double * 6)(*[float(v) for v in domain[0]])
                _chk(L.sphdem_set_domain(self._h, bb, float(domain[1]), float(domain[2])), "sphdem_set_domain")
            if list_build is not None:
                _chk(L.sphdem_set_list_build(self._h, int(list_build)), "sphdem_set_list_build")
            if beds is not None:
                rows = (BedRow * len(beds))(*[BedRow(**{k: float(r[k]) for k, _ in BedRow._fields_}) for r in beds])
                _chk(L.sphdem_set_beds(self._h, len(beds), rows), "sphdem_set_beds")
            for which, d in ((SPH, sph), (DEM, dem)):
                for name, arr in (d or {}).items():
                    self._set(which, name, arr)
            _chk(L.sphdem_commit_particles(self._h), "sphdem_commit_particles")
        except Exception:
            self.close()
            raise

    @classmethod
    def batch(cls, params, beds):
        """Several independent 2-D WCSPH beds in one handle
        (sphdem_create_batch): beds is a list of SPH dicts, each in its own
        coordinates.  Rows are the beds concatenated in order; bed_of(pid)
        maps a slot's input row back to its bed."""
        self = cls.__new__(cls)
        L = lib()
        counts = [len(b["x"]) for b in beds]
        arr = (C.c_int32 * len(counts))(*counts)
        self._h = C.c_void_p()
        _chk(L.sphdem_create_batch(C.byref(params), len(counts), arr, C.byref(self._h)), "sphdem_create_batch")
        self.params = params.copy()
        self.ns, self.nd = sum(counts), 0
        self.bed_start = np.concatenate([[0], np.cumsum(counts)]).astype(np.int64)
        try:
            for name in beds[0]:
                self._set(SPH, name, np.concatenate([np.asarray(b[name]) for b in beds]))
            _chk(L.sphdem_commit_particles(self._h), "sphdem_commit_particles")
        except Exception:
            self.close()
            raise
        return self

    def bed_of(self, pid):
        """Bed index of each input row (batch handles)."""
        return np.searchsorted(self.bed_start, np.asarray(pid), side="right") - 1

    def batch_offsets(self):
        off = np.zeros(2 * (len(self.bed_start) - 1))
        _chk(lib().sphdem_batch_offsets(self._h, off.ctypes.data_as(C.POINTER(C.c_double))), "sphdem_batch_offsets")
        return off.reshape(-1, 2)

    @classmethod
    def from_dir(cls, path, precision=0):
        self = cls.__new__(cls)
        L = lib()
        ov = default_params()
        ov.precision = precision
        self._h = C.c_void_p()
        _chk(L.sphdem_create_from_dir(os.fsencode(path), C.byref(ov), C.byref(self._h)), "sphdem_create_from_dir")
        ns, nd = C.c_int32(), C.c_int32()
        L.sphdem_get_counts(self._h, C.byref(ns), C.byref(nd))
        self.ns, self.nd = ns.value, nd.value
        self.params = read_solv(os.path.join(path, "solv.txt"))
        return self

    def _set(self, which, name, arr):
        fid = F[name]
        if name in INT_FIELDS:
            a = np.ascontiguousarray(arr, dtype=np.int32)
        else:
            a = np.ascontiguousarray(arr, dtype=np.float64)
        _chk(lib().sphdem_set_field(self._h, which, fid, a.ctypes.data, a.nbytes), f"sphdem_set_field({name})")

    def step(self, n=1):
        _chk(lib().sphdem_step(self._h, int(n)), "sphdem_step")

    def get(self, which, name):
        n = self.nd if which == DEM else self.ns
        if name in INT_FIELDS:
            a = np.empty(n, dtype=np.int32)
        else:
            a = np.empty(n, dtype=np.float64)
        _chk(lib().sphdem_get_field(self._h, which, F[name], a.ctypes.data, a.nbytes), f"sphdem_get_field({name})")
        return a

    def check(self):
        """sphdem_check: the status code (0, or SPHDEM_E_OVERFLOW / SPHDEM_E_NAN) of the state so far."""
        return int(lib().sphdem_check(self._h))

    def stats(self):
        s = SphdemStats()
        _chk(lib().sphdem_get_stats(self._h, C.byref(s)), "sphdem_get_stats")
        return {k: getattr(s, k) for k, _ in s._fields_}

    def neighbors(self, cap=512):
        counts = np.zeros(self.ns, dtype=np.int32)
        lst = np.full((self.ns, cap), -1, dtype=np.int32)
        _chk(lib().sphdem_get_neighbors(self._h, counts.ctypes.data_as(C.POINTER(C.c_int32)),
                                        lst.ctypes.data_as(C.POINTER(C.c_int32)), cap), "sphdem_get_neighbors")
        return counts, lst

    def history(self, out=None):
        """Contact history (ids (nd, 16) int32, springs (nd, 16, 3) float64);
        out=(ids, springs) fills preallocated arrays."""
        if out is None:
            ids = np.zeros((self.nd, 16), dtype=np.int32)
            sp = np.zeros((self.nd, 16, 3), dtype=np.float64)
        else:
            ids, sp = out
            if (ids.dtype != np.int32 or sp.dtype != np.float64 or not ids.flags["C_CONTIGUOUS"]
                    or not sp.flags["C_CONTIGUOUS"] or ids.size != self.nd * 16 or sp.size != self.nd * 48):
                raise ValueError("history out: contiguous int32 (nd,16) and float64 (nd,16,3) arrays")
        _chk(lib().sphdem_get_history(self._h, ids.ctypes.data_as(C.POINTER(C.c_int32)),
                                      sp.ctypes.data_as(C.POINTER(C.c_double))), "sphdem_get_history")
        return ids, sp

    def set(self, which, name, arr):
        """Upload a state field after commit, in the current slot order."""
        self._set(which, name, arr)

    def _bulk(self, fn, which, arrays, what):
        names = list(arrays)
        n = self.nd if which == DEM else self.ns
        ids = (C.c_int32 * len(names))(*[F[k] for k in names])
        ptrs = (C.POINTER(C.c_double) * len(names))()
        for k, name in enumerate(names):
            a = arrays[name]
            if a.dtype != np.float64 or not a.flags["C_CONTIGUOUS"] or a.shape != (n,):
                raise ValueError(f"{name}: need a contiguous float64 array of {n}")
            ptrs[k] = a.ctypes.data_as(C.POINTER(C.c_double))
        _chk(fn(self._h, which, len(names), ids, ptrs), what)

    def set_fields(self, which, arrays):
        """Upload several state fields at once ({name: float64 array}) after
        commit, in the current slot order (sphdem_set_fields)."""
        self._bulk(lib().sphdem_set_fields, which, arrays, "sphdem_set_fields")

    def get_fields(self, which, arrays):
        """Fill {name: float64 array} with the current values of several
        real fields at once (sphdem_get_fields)."""
        self._bulk(lib().sphdem_get_fields, which, arrays, "sphdem_get_fields")

    def mlp_state(self):
        """(params float32, stats float64, trained steps) of the learned warm start."""
        L = lib()
        p = np.zeros(L.sphdem_mlp_param_count(), dtype=np.float32)
        st = np.zeros(40, dtype=np.float64)
        t = C.c_int32()
        _chk(L.sphdem_get_mlp_state(self._h, p.ctypes.data_as(C.POINTER(C.c_float)),
                                    st.ctypes.data_as(C.POINTER(C.c_double)), C.byref(t)), "sphdem_get_mlp_state")
        return p, st, t.value

    def set_mlp_state(self, params, stats, trained_steps):
        p = np.ascontiguousarray(params, dtype=np.float32)
        st = np.ascontiguousarray(stats, dtype=np.float64)
        _chk(lib().sphdem_set_mlp_state(self._h, p.ctypes.data_as(C.POINTER(C.c_float)),
                                        st.ctypes.data_as(C.POINTER(C.c_double)), int(trained_steps)),
             "sphdem_set_mlp_state")

    def set_history(self, ids, springs):
        ids = np.ascontiguousarray(ids, dtype=np.int32)
        sp = np.ascontiguousarray(springs, dtype=np.float64)
        _chk(lib().sphdem_set_history(self._h, ids.ctypes.data_as(C.POINTER(C.c_int32)),
                                      sp.ctypes.data_as(C.POINTER(C.c_double))), "sphdem_set_history")

    def list_build(self):
        """The SPH list build the handle runs (sphdem_get_list_build)."""
        m = C.c_int32()
        _chk(lib().sphdem_get_list_build(self._h, C.byref(m)), "sphdem_get_list_build")
        return m.value

    def set_timing(self, on):
        _chk(lib().sphdem_set_timing(self._h, int(bool(on))), "sphdem_set_timing")

    def set_graphs(self, on):
        """Step graphs on/off (off: kernel profilers see every launch)."""
        _chk(lib().sphdem_set_graphs(self._h, int(bool(on))), "sphdem_set_graphs")

    def set_timing_only(self, name=None):
        """Time only the named kernel (a key of timing()), or every kernel."""
        k = -1
        if name is not None:
            names = list(self.timing_names())
            k = names.index(name)
        _chk(lib().sphdem_set_timing_only(self._h, k), "sphdem_set_timing_only")

    def timing_names(self):
        out = []
        name = C.create_string_buffer(64)
        ms, n = C.c_double(), C.c_int64()
        while lib().sphdem_get_timing(self._h, len(out), name, 64, C.byref(ms), C.byref(n)) == 0:
            out.append(name.value.decode())
        return out

    def set_concurrency(self, on):
        """DEM branch of the step on its own stream (default) or on the step stream."""
        _chk(lib().sphdem_set_concurrency(self._h, int(bool(on))), "sphdem_set_concurrency")

    def collect_timing(self):
        _chk(lib().sphdem_collect_timing(self._h), "sphdem_collect_timing")

    def timing(self):
        """{kernel name: (total ms, launches)} accumulated by collect_timing."""
        out = {}
        k = 0
        name = C.create_string_buffer(64)
        while True:
            ms, n = C.c_double(), C.c_int64()
            if lib().sphdem_get_timing(self._h, k, name, 64, C.byref(ms), C.byref(n)) != 0:
                break
            out[name.value.decode()] = (ms.value, n.value)
            k += 1
        return out

    # -- slab exchange (sphdem_slab_*): device tensors on the engine's device --
    def _slots(self, which):
        import torch

        n = self.ns if which == SPH else self.nd
        t = self._slot_buf.get(which)
        if t is None:
            t = self._slot_buf[which] = torch.empty(max(n, 1), dtype=torch.int32, device="cuda")
        return t

    def slab_select(self, which, axis, lo, hi):
        """Active slots whose cell layer along axis is in [lo, hi), ascending
        (an int32 CUDA tensor)."""
        buf = self._slots(which)
        cnt = C.c_int32()
        _chk(lib().sphdem_slab_select(self._h, which, axis, int(lo), int(hi), C.c_void_p(buf.data_ptr()),
                                      buf.numel(), C.byref(cnt)), "sphdem_slab_select")
        return buf[:cnt.value]

    def slab_export(self, which, slots):
        """Records of the given slots (a uint8 CUDA tensor), written on the
        engine's stream; the call returns after the copy has finished."""
        import torch

        rb = lib().sphdem_slab_record_bytes(which)
        out = torch.empty(max(slots.numel(), 1) * rb, dtype=torch.uint8, device="cuda")
        _chk(lib().sphdem_slab_export(self._h, which, C.c_void_p(slots.data_ptr()), slots.numel(),
                                      C.c_void_p(out.data_ptr())), "sphdem_slab_export")
        torch.cuda.ExternalStream(self.stream_ptr()).synchronize()
        return out[:slots.numel() * rb]

    def slab_keep(self, which, axis, lo, hi):
        _chk(lib().sphdem_slab_keep(self._h, which, axis, int(lo), int(hi)), "sphdem_slab_keep")

    def slab_import(self, which, records):
        """Unpack records (a uint8 CUDA tensor) into parked slots."""
        rb = lib().sphdem_slab_record_bytes(which)
        n = records.numel() // rb
        if n:
            records = records.contiguous()
            torch_sync()
            _chk(lib().sphdem_slab_import(self._h, which, C.c_void_p(records.data_ptr()), n), "sphdem_slab_import")

    def slab_active(self, which):
        n = C.c_int32()
        _chk(lib().sphdem_slab_active(self._h, which, C.byref(n)), "sphdem_slab_active")
        return n.value

    def time(self):
        t, c = C.c_double(), C.c_int32()
        lib().sphdem_get_time(self._h, C.byref(t), C.byref(c))
        return t.value, c.value

    def stream_ptr(self):
        s = C.c_void_p()
        lib().sphdem_get_stream(self._h, C.byref(s))
        return s.value or 0

    def launches(self):
        n = C.c_int64()
        lib().sphdem_get_launch_count(self._h, C.byref(n))
        return n.value

    def write_vtk_dem(self, path):
        _chk(lib().sphdem_write_vtk_dem(self._h, os.fsencode(path)), "sphdem_write_vtk_dem")

    def write_vtk_fluid(self, path):
        _chk(lib().sphdem_write_vtk_fluid(self._h, os.fsencode(path)), "sphdem_write_vtk_fluid")

    def snapshot(self):
        """sphdem_snapshot: start copying the output fields of this step to the host."""
        _chk(lib().sphdem_snapshot(self._h), "sphdem_snapshot")

    def write_snapshot(self, dem_vtk=None, fluid_vtk=None):
        """sphdem_write_snapshot: wait for the last snapshot and write its VTK files."""
        _chk(lib().sphdem_write_snapshot(self._h, os.fsencode(dem_vtk) if dem_vtk else None,
                                         os.fsencode(fluid_vtk) if fluid_vtk else None), "sphdem_write_snapshot")

    def write_restart(self, path):
        _chk(lib().sphdem_write_restart(self._h, os.fsencode(path)), "sphdem_write_restart")

    def close(self):
        if getattr(self, "_h", None) and self._h.value:
            lib().sphdem_destroy(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()


def read_input_txt(path):
    """Host-only read of an input.txt: returns (sph, dem) dicts of arrays."""
    L = lib()
    ns, nd = C.c_int32(), C.c_int32()
    _chk(L.sphdem_input_counts(os.fsencode(path), C.byref(ns), C.byref(nd)), "sphdem_input_counts")
    out = []
    for which, n in ((SPH, ns.value), (DEM, nd.value)):
        d = {}
        for name in ("x", "y", "z", "ux", "uy", "uz", "m", "h", "temp", "pres", "rho", "flt_s", "rad", "ri",
                     "wx", "wy", "wz", "temp1", "temp2", "temp3", "p_type", "dem_idx"):
            a = np.zeros(n, dtype=np.int32 if name in INT_FIELDS else np.float64)
            _chk(L.sphdem_input_column(os.fsencode(path), which, F[name], a.ctypes.data, a.nbytes),
                 f"sphdem_input_column({name})")
            d[name] = a
        out.append(d)
    return out[0], out[1]
