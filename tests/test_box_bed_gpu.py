"""Parity of the engine on the benchmark bed's own configuration.

The bench bed is the 3-D SPH-DEM box bed (beds.box_bed: Wendland C2,
h = 1.3 dx, water-like fluid, Hertz-Mindlin with E = 1e7 Pa, nu = 0.3,
friction 0.3, heat transfer and XSPH on, box DEM walls, inlet/outlet
slabs).  These tests run the same configuration at reduced size -- a
0.05 x 0.02 m cross-section, 20,000 fluid particles at the bench's
dx = 1.25 mm and 2,000 spheres at the bench's sphere density (d = 2 mm
+-5 %, FCC sites 2.1 mm apart in the lower 0.02 m) -- so that the FP64
oracle runs 100 steps in seconds.

Bar (written into each assert):
* every 10 steps: sorted order, cell keys and every neighbour list
  bit-exact, and the DEM contact partners of every sphere exact;
* FP32 build vs the FP64 oracle after 100 steps: every SPH and DEM field
  within rel. L2 1e-5;
* FP64 build vs the oracle after 10 steps: rel. L2 1e-9 per field, springs
  to rtol 1e-9;
* FP32 build vs the FP64 build of the same kernels after 100 steps: every
  field within rel. L2 1e-5.
"""
import numpy as np
import pytest

from fluidized_bed_master_b200.beds import box_bed
from fluidized_bed_master_b200.params import DEM, SPH
from oracle import Oracle
from tests.helpers import by_id, history_map, rel_l2

pytestmark = pytest.mark.gpu

SPH_ALL = ["x", "y", "z", "ux", "uy", "uz", "m", "rho", "pres", "temp", "DEMpor", "dDEMpor", "flt_s",
           "ftotalx", "ftotaly", "ftotalz", "fpx", "fpy", "fpz", "pgfx", "pgfy", "pgfz", "rho_ref", "dtemp"]
DEM_ALL = ["x", "y", "z", "ux", "uy", "uz", "wx", "wy", "wz", "temp", "DEMpor", "flt_s", "flt_sd", "flt_sd2",
           "Fdx_df", "Fdy_df", "Fdz_df", "ftotalx", "ftotaly", "ftotalz", "torqx", "torqy", "torqz", "dtemp",
           "Q_sd", "temp1", "temp2", "temp3"]
FP32_TOL = 1e-5
FP64_TOL = 1e-9


@pytest.fixture(scope="module")
def small_box_bed():
    return box_bed(n_fluid=20_000, n_dem=2_000, lx=0.05, dem_height=0.02, seed=41)


def _engine(p, sph, dem, prec):
    from fluidized_bed_master_b200.engine import Engine

    q = p.copy()
    q.precision = prec
    return Engine(q, sph, dem)


def _ids(src, which):
    return src.get(which, "pid") if which == SPH else src.get(which, "dem_idx")


def _field_errors(a, b, fields_s, fields_d):
    out = {}
    for which, fields in ((SPH, fields_s), (DEM, fields_d)):
        ia, ib = _ids(a, which), _ids(b, which)
        for f in fields:
            out[("dem" if which else "sph", f)] = rel_l2(by_id(ia, a.get(which, f)), by_id(ib, b.get(which, f)))
    return out


def _partners(src):
    ids, springs = src.history()
    m = history_map(np.asarray(ids, dtype=float), springs)
    dem_ids = _ids(src, DEM)
    return {int(dem_ids[i]): m[i] for i in range(len(dem_ids))}


def _check_lists_and_partners(eng, orc, label):
    for which in (SPH, DEM):
        assert np.array_equal(_ids(eng, which), _ids(orc, which)), f"{label}: sorted order differs"
        assert np.array_equal(eng.get(which, "cell"), orc.get(which, "cell")), f"{label}: cell keys differ"
    ce, le = eng.neighbors()
    co, lo = orc.neighbors()
    assert np.array_equal(ce, co), f"{label}: neighbour counts differ"
    for i in np.flatnonzero(ce):
        assert np.array_equal(le[i, : ce[i]], lo[i, : co[i]]), f"{label}: neighbour list of slot {i} differs"
    pe, po = _partners(eng), _partners(orc)
    for k, v in po.items():
        assert set(pe[k]) == set(v), f"{label}: contact partners of sphere {k} differ"
    return sum(len(v) for v in po.values())


def test_box_bed_fp32_100_steps_vs_oracle(small_box_bed):
    """FP32 build vs the FP64 oracle on the bench configuration: lists and
    partners exact every 10 steps, every field within rel. L2 1e-5 after 100."""
    p, sph, dem = small_box_bed
    eng = _engine(p, sph, dem, 0)
    orc = Oracle(p, sph, dem, threads=16)
    contacts = 0
    for k in range(10):
        eng.step(10)
        orc.step(10)
        contacts = _check_lists_and_partners(eng, orc, f"step {10 * (k + 1)}")
    assert contacts > 100, "the bed formed too few contacts for the history to be exercised"
    err = _field_errors(eng, orc, SPH_ALL, DEM_ALL)
    bad = {k: v for k, v in err.items() if not v <= FP32_TOL}
    assert not bad, sorted(bad.items(), key=lambda kv: -kv[1])


def test_box_bed_fp64_vs_oracle(small_box_bed):
    """FP64 build vs the oracle on the bench configuration after 10 steps."""
    p, sph, dem = small_box_bed
    eng = _engine(p, sph, dem, 1)
    orc = Oracle(p, sph, dem, threads=16)
    eng.step(10)
    orc.step(10)
    _check_lists_and_partners(eng, orc, "step 10")
    err = _field_errors(eng, orc, SPH_ALL, DEM_ALL)
    bad = {k: v for k, v in err.items() if not v <= FP64_TOL}
    assert not bad, sorted(bad.items(), key=lambda kv: -kv[1])
    pe, po = _partners(eng), _partners(orc)
    for k, v in po.items():
        for j, s in v.items():
            assert np.allclose(pe[k][j], s, rtol=1e-9, atol=1e-18), (k, j)


def test_box_bed_fp32_vs_fp64_build_100_steps(small_box_bed):
    """Every field of the FP32 build against the FP64 build of the same
    kernels after 100 steps on the bench configuration."""
    p, sph, dem = small_box_bed
    e32 = _engine(p, sph, dem, 0)
    e64 = _engine(p, sph, dem, 1)
    e32.step(100)
    e64.step(100)
    err = _field_errors(e32, e64, SPH_ALL, DEM_ALL)
    bad = {k: v for k, v in err.items() if not v <= FP32_TOL}
    assert not bad, sorted(bad.items(), key=lambda kv: -kv[1])
