"""Analytic and structural checks of the oracle (CPU only)."""
import ctypes as C

import numpy as np
import pytest

from fluidized_bed_master_b200.beds import spouted_bed
from fluidized_bed_master_b200.params import DEM, SPH, reference_params
from oracle import Oracle, lib


def kern(kt, h, r, deriv=0):
    L = lib()
    L.oracle_kernel.restype = C.c_double
    L.oracle_kernel.argtypes = [C.c_int, C.c_int, C.c_double, C.c_double, C.c_int]
    return np.array([L.oracle_kernel(kt, 3, h, float(x), deriv) for x in np.atleast_1d(r)])


@pytest.mark.parametrize("kt", [3, 4, 5])
def test_wendland_normalisation_and_derivative(kt):
    h = 1.0e-3
    r = np.linspace(0, 2 * h, 20001)
    w = kern(kt, h, r)
    integral = np.trapezoid(4 * np.pi * r * r * w, r)
    assert abs(integral - 1.0) < 1e-6, integral   # functions_KNL.cuh:2-32 normalisation
    dw = kern(kt, h, r[1:-1], 1)
    fd = (w[2:] - w[:-2]) / (r[2:] - r[:-2])
    assert np.max(np.abs(dw - fd)) < 1e-5 * np.max(np.abs(dw))
    assert w[-1] == 0.0


def _small_bed(**kw):
    args = dict(dx=2.5e-3, n_dem=40, r_dem=1.0e-3, seed=7)
    args.update(kw)
    return spouted_bed(**args)


def test_sorted_cells_and_symmetric_lists():
    p, sph, dem = _small_bed()
    o = Oracle(p, sph, dem, threads=2)
    o.step(1)
    cell = o.get(SPH, "cell")
    assert np.all(np.diff(cell) >= 0)
    cnt, lst = o.neighbors()
    n = len(cnt)
    pairs = set()
    for i in range(n):
        row = lst[i, : cnt[i]]
        assert i in row                      # self is inside kappa*h
        assert np.all(np.diff(row) > 0)      # reference visit order == ascending slot
        pairs.update((i, int(j)) for j in row)
    assert all((j, i) in pairs for (i, j) in pairs)   # equal h: symmetric


def test_thread_count_does_not_change_results():
    p, sph, dem = _small_bed(spacing=1.9, u_dem=0.05)
    a = Oracle(p, sph, dem, threads=1)
    b = Oracle(p, sph, dem, threads=8)
    a.step(3)
    b.step(3)
    for which, f in ((SPH, "pres"), (SPH, "uz"), (DEM, "ux"), (DEM, "ftotalz")):
        assert np.array_equal(a.get(which, f), b.get(which, f))


def test_two_sphere_head_on_restitution():
    """Hertz-Mindlin with the reference damping constant (e = 0.9 design):
    two equal spheres meeting head-on rebound with 0.8 < e < 0.98."""
    p = reference_params()
    p.fg_solve = 0
    p.open_boundary = 0
    p.dem_wall_mask = 0
    p.xsph_solve = 0
    p.dt = 1.0e-7
    r, v = 1.0e-3, 0.5
    rho = 2500.0
    m = rho * 4 / 3 * np.pi * r ** 3
    dem = dict(x=np.array([-1.001e-3, 1.001e-3]), y=np.zeros(2), z=np.zeros(2),
               ux=np.array([v, -v]), uy=np.zeros(2), uz=np.zeros(2),
               wx=np.zeros(2), wy=np.zeros(2), wz=np.zeros(2), m=np.full(2, m), rho=np.full(2, rho),
               rad=np.full(2, r), ri=np.full(2, 0.4 * m * r * r), h=np.full(2, 1.6e-3),
               temp=np.full(2, 300.0), p_type=np.array([1001, 1001], np.int32), dem_idx=np.array([1, 2], np.int32))
    # gas at rest around the pair: the drag closure divides by the local
    # porosity, which is 0/0 for a sphere with no fluid neighbours
    # (functions_SPH_DEM_COUPLING2.cuh:907, 1105)
    g = (np.arange(-6, 7) + 0.5) * 1.0e-3
    X, Y, Z = np.meshgrid(g, g, g, indexing="ij")
    ns = X.size
    sph = dict(x=X.ravel(), y=Y.ravel(), z=Z.ravel(), h=np.full(ns, 1.6e-3), m=np.full(ns, 1.784e-9),
               rho=np.full(ns, 1.784), temp=np.full(ns, 300.0), flt_s=np.ones(ns), p_type=np.ones(ns, np.int32))
    o = Oracle(p, sph, dem)
    contact_seen = False
    for _ in range(4000):
        o.step(1)
        ct, _ = o.history()
        contact_seen |= bool((ct > 0).any())
        x = o.get(DEM, "x")
        ux = o.get(DEM, "ux")
        ids = o.get(DEM, "dem_idx")
        u = ux[np.argsort(ids)]
        xs = x[np.argsort(ids)]
        if contact_seen and (xs[1] - xs[0]) > 2.0 * r and u[1] > u[0]:
            break
    e = (u[1] - u[0]) / (2 * v)
    assert contact_seen
    assert 0.8 < e < 0.98, e


@pytest.mark.parametrize("mode", [1, 2])
def test_oracle_krylov_ppe_converges(mode):
    """The oracle's Krylov PPE (BiCGStab / PCG, FP64) reaches ppe_tol within
    the iteration cap on a small bed, and differs from the one-sweep
    reference pressure only on solved rows."""
    from fluidized_bed_master_b200.beds import spouted_bed
    from fluidized_bed_master_b200.params import SPH

    p, sph, dem = spouted_bed(dx=2.5e-3, n_dem=200, r_dem=1.0e-3, seed=43)
    p.ppe_mode = mode
    p.ppe_tol = 1e-8
    p.ppe_max_iter = 2000
    if mode == 2:
        p.kgc_solve = 0
    o = Oracle(p, sph, dem, threads=4)
    for _ in range(2):
        o.step(1)
        it, res, st = o.ppe()
        assert st == 0 and res <= 1e-8 and it >= 1, (it, res, st)
    assert np.isfinite(o.get(SPH, "pres")).all()


def test_mlp_oracle_gradient_by_finite_differences():
    """The FP64 oracle's backward pass (without BF16 rounding) against
    central differences of its own loss, every parameter block."""
    from oracle import mlp_oracle as MO

    rng = np.random.default_rng(3)
    p = MO.init_params(3)
    p[MO.OFF_B1:MO.OFF_W2] = 0.1 * rng.standard_normal(MO.N_H)
    x = rng.standard_normal((64, MO.N_IN))
    t = rng.standard_normal(64)
    w = rng.uniform(0.5, 1.0, size=64)
    ws = w.sum()

    def loss(q):
        y, _ = MO.forward(q, x, rounding=False)
        return float((w * (y - t) ** 2).sum() / ws)

    g, _, _ = MO.grad(p, x, t, w, ws, rounding=False)
    idx = np.concatenate([rng.choice(np.arange(a, b), size=min(8, b - a), replace=False)
                          for a, b in ((MO.OFF_W1, MO.OFF_B1), (MO.OFF_B1, MO.OFF_W2), (MO.OFF_W2, MO.OFF_B2),
                                       (MO.OFF_B2, MO.OFF_W3), (MO.OFF_W3, MO.OFF_B3), (MO.OFF_B3, MO.N_PARAM))])
    for k in idx:
        e = np.zeros_like(p)
        e[k] = 1e-6
        fd = (loss(p + e) - loss(p - e)) / 2e-6
        assert abs(fd - g[k]) <= 1e-5 * max(1.0, abs(fd)), (k, fd, g[k])
