"""Batched 2-D WCSPH beds (sphdem_create_batch) on the GPU.

Several dam breaks of different sizes share one handle and one step graph.
Each bed must evolve as if it ran alone: the same neighbour counts per
particle and, in the FP64 build, the same fields to rel. L2 <= 1e-9 after
20 steps (the beds sit in a different cell grid than when alone, which
changes only the order of the neighbour sums).  x and y come back in each
bed's own coordinates.
"""
import numpy as np
import pytest

from fluidized_bed_master_b200.beds import dam_break_batch
from fluidized_bed_master_b200.params import SPH
from tests.helpers import by_id, rel_l2

pytestmark = pytest.mark.gpu

FIELDS = ["x", "y", "ux", "uy", "rho", "pres", "flt_s", "ftotalx", "ftotaly", "drho"]


def _params(p, prec):
    q = p.copy()
    q.precision = prec
    q.xsph_solve = 1
    q.c_xsph = 0.5
    q.delSPH_solve = 1
    q.w_lanes = 4
    return q


def test_batch_matches_each_bed_alone():
    from fluidized_bed_master_b200.engine import Engine

    p, beds = dam_break_batch(n_beds=4, n_min=1_500, n_max=6_000, seed=3)
    q = _params(p, 1)
    batch = Engine.batch(q, beds)
    batch.step(20)
    pid = batch.get(SPH, "pid")
    bed = batch.bed_of(pid)
    cnt_b, _ = batch.neighbors(cap=1)
    vals = {f: batch.get(SPH, f) for f in FIELDS}
    off = batch.batch_offsets()
    assert np.all(np.abs(off).sum(1)[1:] > 0), "beds were not separated"
    bad = []
    for b, sph in enumerate(beds):
        alone = Engine(q, sph, {})
        alone.step(20)
        sel = bed == b
        local = pid[sel] - batch.bed_start[b]
        ia = alone.get(SPH, "pid")
        ca, _ = alone.neighbors(cap=1)
        assert np.array_equal(by_id(local, cnt_b[sel]), by_id(ia, ca)), f"neighbour counts of bed {b} differ"
        for f in FIELDS:
            e = rel_l2(by_id(local, vals[f][sel]), by_id(ia, alone.get(SPH, f)))
            if not e <= 1e-9:
                bad.append((b, f, e))
        alone.close()
    assert not bad, bad


def test_batch_state_roundtrip_in_bed_coordinates():
    """get_fields/set_fields of x, y on a batch handle use the beds' own
    coordinates: a round trip leaves the run bit-identical."""
    from fluidized_bed_master_b200.engine import Engine

    p, beds = dam_break_batch(n_beds=3, n_min=1_500, n_max=4_000, seed=4)
    q = _params(p, 0)
    a = Engine.batch(q, beds)
    b = Engine.batch(q, beds)
    a.step(3)
    b.step(3)
    x = b.get(SPH, "x")
    pid = b.get(SPH, "pid")
    x_in = np.concatenate([bd["x"] for bd in beds])
    assert np.max(np.abs(x - x_in[pid])) < 0.05, "x is not in the bed's own coordinates"
    st = {f: np.zeros(b.ns) for f in ("x", "y", "ux", "uy", "rho")}
    b.get_fields(SPH, st)
    assert np.array_equal(st["x"], x)
    b.set_fields(SPH, st)
    a.step(2)
    b.step(2)
    for f in ("x", "y", "ux", "uy", "rho", "pres"):
        assert np.array_equal(a.get(SPH, f), b.get(SPH, f)), f
