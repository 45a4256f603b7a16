"""The allocation-free cell sort (sphdem_sort_cells_static).

Some callers cannot allocate device memory inside their time loop -- an
application that owns all device memory through its own pool and fixes its
footprint at start-up, or a coupled solver whose other streams must not
stall on the device-wide synchronisation that cudaMalloc/cudaFree may
imply -- so the library offers one entry
point whose scratch is a file-scope device array instead of cudaMalloc.
This test calls it through the C ABI on device arrays the test owns and
checks, on consecutive calls, that it returns the same sorted order and
cell keys as the engine's own NNPS (the first step of sphdem_step sorts the
input order), and that it rejects sizes above its limit.

The file name keeps it last in pytest's collection order.
"""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

MAX_N = 1 << 18          # SPHDEM_STATIC_MAX_PARTICLES
E_NOMEM = -8


def _grid(p, sph, dem):
    """Cell grid of the engine's commit: bounding box over the rows in file
    order (SPH then DEM) without the last row, dcell = 1.1 kappa h0."""
    x = np.concatenate([sph["x"], dem["x"]])
    y = np.concatenate([sph["y"], dem["y"]])
    z = np.concatenate([sph["z"], dem["z"]])
    bb = np.array([x[:-1].min(), x[:-1].max(), y[:-1].min(), y[:-1].max(), z[:-1].min(), z[:-1].max()])
    dcell = 1.1 * p.kappa * sph["h"][0]
    nijk = np.array([int((bb[1] - bb[0]) / dcell) + 1, int((bb[3] - bb[2]) / dcell) + 1,
                     int((bb[5] - bb[4]) / dcell) + 1], dtype=np.int32)
    return bb, nijk


def _call(lib, pos, bb, nijk):
    import torch

    n = pos.shape[0]
    dev = torch.device("cuda")
    x = torch.tensor(np.ascontiguousarray(pos[:, 0]), dtype=torch.float64, device=dev)
    y = torch.tensor(np.ascontiguousarray(pos[:, 1]), dtype=torch.float64, device=dev)
    z = torch.tensor(np.ascontiguousarray(pos[:, 2]), dtype=torch.float64, device=dev)
    ncell = int(nijk.prod())
    perm = torch.full((max(n, 1),), -7, dtype=torch.int32, device=dev)
    key = torch.full((max(n, 1),), -7, dtype=torch.int32, device=dev)
    start = torch.zeros(ncell, dtype=torch.int32, device=dev)
    end = torch.zeros(ncell, dtype=torch.int32, device=dev)
    bbc = (C.c_double * 6)(*bb.tolist())
    nc = (C.c_int32 * 3)(*nijk.tolist())
    stream = torch.cuda.current_stream().cuda_stream
    rc = lib.sphdem_sort_cells_static(C.c_void_p(x.data_ptr()), C.c_void_p(y.data_ptr()), C.c_void_p(z.data_ptr()),
                                      n, bbc, nc, C.c_void_p(perm.data_ptr()), C.c_void_p(key.data_ptr()),
                                      C.c_void_p(start.data_ptr()), C.c_void_p(end.data_ptr()), C.c_void_p(stream))
    torch.cuda.synchronize()
    return rc, perm.cpu().numpy()[:n], key.cpu().numpy()[:n], start.cpu().numpy(), end.cpu().numpy()


def _bind():
    from fluidized_bed_master_b200.engine import lib

    L = lib()
    L.sphdem_sort_cells_static.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_int32, C.POINTER(C.c_double),
                                           C.POINTER(C.c_int32), C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
                                           C.c_void_p]
    L.sphdem_sort_cells_static.restype = C.c_int
    return L


def _check_bounds(key, start, end):
    n = len(key)
    occupied = np.unique(key)
    assert np.all(start[np.setdiff1d(np.arange(len(start)), occupied)] == -1)
    for c in occupied:
        s, e = start[c], end[c]
        assert 0 <= s < e <= n
        assert np.all(key[s:e] == c)
        assert (s == 0 or key[s - 1] != c) and (e == n or key[e] != c)


def test_static_sort_matches_engine_on_consecutive_calls():
    from fluidized_bed_master_b200.beds import spouted_bed
    from fluidized_bed_master_b200.engine import Engine
    from fluidized_bed_master_b200.params import DEM, SPH

    p, sph, dem = spouted_bed(dx=2.0e-3, n_dem=100000, r_dem=1.0e-3, seed=31, spacing=2.1)
    q = p.copy()
    q.precision = 1
    eng = Engine(q, sph, dem)
    eng.step(1)       # the first step sorts the input order by cell
    want = {SPH: (eng.get(SPH, "pid"), eng.get(SPH, "cell")), DEM: (eng.get(DEM, "pid"), eng.get(DEM, "cell"))}
    eng.close()
    bb, nijk = _grid(p, sph, dem)
    L = _bind()
    pos = {SPH: np.stack([sph["x"], sph["y"], sph["z"]], 1), DEM: np.stack([dem["x"], dem["y"], dem["z"]], 1)}
    for which in (SPH, DEM, SPH):   # consecutive calls share the static scratch
        rc, perm, key, start, end = _call(L, pos[which], bb, nijk)
        assert rc == 0
        assert np.array_equal(perm, want[which][0]), "sorted order differs from the engine's NNPS"
        assert np.array_equal(key, want[which][1]), "cell keys differ from the engine's NNPS"
        _check_bounds(key, start, end)


def test_static_sort_rejects_sizes_above_limit():
    import torch

    L = _bind()
    buf = torch.zeros(16, dtype=torch.float64, device="cuda")
    ib = torch.zeros(16, dtype=torch.int32, device="cuda")
    bbc = (C.c_double * 6)(0, 1, 0, 1, 0, 1)
    nc = (C.c_int32 * 3)(2, 2, 2)
    rc = L.sphdem_sort_cells_static(C.c_void_p(buf.data_ptr()), C.c_void_p(buf.data_ptr()),
                                    C.c_void_p(buf.data_ptr()), MAX_N + 1, bbc, nc, C.c_void_p(ib.data_ptr()),
                                    C.c_void_p(ib.data_ptr()), C.c_void_p(ib.data_ptr()), C.c_void_p(ib.data_ptr()),
                                    None)
    assert rc == E_NOMEM
