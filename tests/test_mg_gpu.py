"""The two-level PCG preconditioner (ppe_mode PCG, ppe_precond TWO_LEVEL).

An engine extension with no counterpart in the reference (which has one
Jacobi sweep per step and no preconditioner), so the oracle does not run
it.  It is pinned instead against the Jacobi-PCG, which the oracle does
run (test_ppe_gpu.py, test_column_gpu.py).  Bar (written into each assert):
* both solves reach the relative residual 1e-6 every step;
* the two-level solve needs at most 0.6 x the Jacobi iterations;
* its pressure agrees with the Jacobi-PCG pressure to rel. L2 <= 2e-5
  after 3 steps: two solutions of the same system, each to 1e-6 of the
  right-hand side;
* the step graph (conditional while node) and the host-driven loop give
  the same iterations and bit-identical pressures (no atomics in the
  preconditioner).
"""
import numpy as np
import pytest

from fluidized_bed_master_b200.beds import box_bed, isph_column
from fluidized_bed_master_b200.params import PPE_PCG, PRECOND_JACOBI, PRECOND_TWO_LEVEL, SPH, WARM_PROJECT
from tests.helpers import by_id, rel_l2

pytestmark = pytest.mark.gpu


def _engine(p, sph, dem, prec, precond):
    from fluidized_bed_master_b200.engine import Engine

    q = p.copy()
    q.precision = prec
    q.ppe_precond = precond
    return Engine(q, sph, dem)


def _column():
    return isph_column(dx=8.0e-3, seed=7)


def _bed():
    p, sph, dem = box_bed(n_fluid=30000, n_dem=3000, seed=6)
    p.ppe_mode = PPE_PCG
    p.kgc_solve = 0
    p.ppe_tol = 1e-6
    p.ppe_max_iter = 2000
    return p, sph, dem


@pytest.mark.parametrize("case", ["column", "bed"])
@pytest.mark.parametrize("prec", [0, 1])
def test_two_level_cuts_iterations_and_agrees_with_jacobi(case, prec):
    p, sph, dem = _column() if case == "column" else _bed()
    a = _engine(p, sph, dem, prec, PRECOND_JACOBI)
    b = _engine(p, sph, dem, prec, PRECOND_TWO_LEVEL)
    ia, ib = [], []
    for _ in range(3):
        a.step(1)
        b.step(1)
        for e, its in ((a, ia), (b, ib)):
            st = e.stats()
            assert st["ppe_status"] == 0 and st["ppe_rel_residual"] <= 1e-6, st
            its.append(st["ppe_iters"])
    assert sum(ib) <= 0.6 * sum(ia), (ia, ib)
    e = rel_l2(by_id(a.get(SPH, "pid"), a.get(SPH, "pres")), by_id(b.get(SPH, "pid"), b.get(SPH, "pres")))
    assert e <= 2e-5, e


def test_two_level_graph_equals_host_driven_loop():
    p, sph, dem = _bed()
    p.warm_start = WARM_PROJECT
    p.warm_hist = 8
    a = _engine(p, sph, dem, 0, PRECOND_TWO_LEVEL)
    b = _engine(p, sph, dem, 0, PRECOND_TWO_LEVEL)
    b.set_graphs(False)
    for _ in range(4):
        a.step(1)
        b.step(1)
        assert a.stats()["ppe_iters"] == b.stats()["ppe_iters"]
    assert np.array_equal(a.get(SPH, "pres"), b.get(SPH, "pres"))


def test_two_level_needs_pcg():
    from fluidized_bed_master_b200.engine import Engine, SphdemError

    p, sph, dem = _bed()
    q = p.copy()
    q.ppe_mode = 1   # BiCGStab
    q.ppe_precond = PRECOND_TWO_LEVEL
    with pytest.raises(SphdemError):
        Engine(q, sph, dem)
