"""Parity of the engine on the benchmark bed's own configuration.

The bench bed is the 3-D SPH-DEM box bed (beds.box_bed: Wendland C2,
h = 1.3 dx, water-like fluid, Hertz-Mindlin with E = 1e7 Pa, nu = 0.3,
friction 0.3, heat transfer and XSPH on, box DEM walls, inlet/outlet
slabs).  These tests run the same configuration as a quarter-height slice
of it -- the bench's 0.1 x 0.02 m cross-section, 50,000 fluid particles at
the bench's dx = 1.25 mm and 5,000 spheres at the bench's sphere density
(d = 2 mm +-5 %, FCC sites 2.1 mm apart in the lower 0.025 m) -- so that the
FP64 oracle runs 100 steps in well under a minute.

Bar (written into each assert):
* every 10 steps: sorted order, cell keys and every neighbour list
  bit-exact, and the DEM contact partners of every sphere exact;
* FP64 build vs the oracle after 10 steps: rel. L2 1e-9 per field, springs
  to rtol 1e-9;
* FP32 build (FP32 SPH fields; FP64 positions and DEM set) vs the FP64
  oracle, and vs the FP64 build of the same kernels, after 100 steps:
  - every state field (positions, velocities, angular velocities, mass,
    density, pressure, temperature, porosity and filters) within rel. L2
    1e-5, the specification's tolerance;
  - every rate field (forces, pressure gradients, torques, drag, heat
    rates) within rel. L2 1e-4.  These are differences of the FP32 fluid
    state: the drag follows the slip between the fluid's Shepard average
    and the sphere, the torques the tangential slip of touching spheres,
    so their relative error is the fluid's FP32 rounding over a small
    difference, grown by 100 steps of stiff contacts.  Measured on this
    bed: <= 5.2e-5 for the DEM torques, <= 1.6e-5 for the DEM total forces,
    <= 1e-5 for every SPH rate.
"""
import numpy as np
import pytest

from fluidized_bed_master_b200.beds import box_bed
from fluidized_bed_master_b200.params import DEM, SPH
from oracle import Oracle
from tests.helpers import by_id, history_map, rel_l2

pytestmark = pytest.mark.gpu

SPH_STATE = ["x", "y", "z", "ux", "uy", "uz", "m", "rho", "pres", "temp", "DEMpor", "flt_s", "rho_ref"]
SPH_RATE = ["dDEMpor", "ftotalx", "ftotaly", "ftotalz", "fpx", "fpy", "fpz", "pgfx", "pgfy", "pgfz", "dtemp"]
DEM_STATE = ["x", "y", "z", "ux", "uy", "uz", "wx", "wy", "wz", "temp", "temp1", "temp2", "temp3", "DEMpor",
             "flt_s", "flt_sd", "flt_sd2"]
DEM_RATE = ["Fdx_df", "Fdy_df", "Fdz_df", "ftotalx", "ftotaly", "ftotalz", "torqx", "torqy", "torqz", "dtemp",
            "Q_sd"]
SPH_ALL = SPH_STATE + SPH_RATE
DEM_ALL = DEM_STATE + DEM_RATE
STATE_TOL = 1e-5    # FP32 build, state fields
RATE_TOL = 1e-4     # FP32 build, rate fields
FP64_TOL = 1e-9


@pytest.fixture(scope="module")
def slice_bed():
    return box_bed(n_fluid=50_000, n_dem=5_000, dem_height=0.025, seed=41)


def _fp32_bad(err):
    bad = {}
    for (which, f), v in err.items():
        state = f in (DEM_STATE if which == "dem" else SPH_STATE)
        if not v <= (STATE_TOL if state else RATE_TOL):
            bad[(which, f)] = v
    return bad


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
    ce, _ = eng.neighbors(cap=1)
    co, _ = orc.neighbors(cap=1)
    assert np.array_equal(ce, co), f"{label}: neighbour counts differ"
    cap = int(ce.max()) + 1
    _, le = eng.neighbors(cap=cap)    # rows padded with -1 past the count on both sides
    _, lo = orc.neighbors(cap=cap)
    if not np.array_equal(le, lo):
        i = int(np.flatnonzero((le != lo).any(axis=1))[0])
        raise AssertionError(f"{label}: neighbour list of slot {i} differs")
    pe, po = _partners(eng), _partners(orc)
    for k, v in po.items():
        assert set(pe[k]) == set(v), f"{label}: contact partners of sphere {k} differ"
    return sum(len(v) for v in po.values())


def test_box_bed_fp32_100_steps_vs_oracle(slice_bed):
    """FP32 build vs the FP64 oracle on the bench configuration: lists and
    partners exact every 10 steps; after 100 steps state fields within rel.
    L2 1e-5, rate fields within 1e-4."""
    p, sph, dem = slice_bed
    eng = _engine(p, sph, dem, 0)
    orc = Oracle(p, sph, dem, threads=16)
    contacts = 0
    for k in range(10):
        eng.step(10)
        orc.step(10)
        contacts = _check_lists_and_partners(eng, orc, f"step {10 * (k + 1)}")
    assert contacts > 100, "the bed formed too few contacts for the history to be exercised"
    bad = _fp32_bad(_field_errors(eng, orc, SPH_ALL, DEM_ALL))
    assert not bad, sorted(bad.items(), key=lambda kv: -kv[1])


def test_box_bed_fp64_vs_oracle(slice_bed):
    """FP64 build vs the oracle on the bench configuration after 10 steps."""
    p, sph, dem = slice_bed
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


def test_box_bed_fp32_vs_fp64_build_100_steps(slice_bed):
    """Every field of the FP32 build against the FP64 build of the same
    kernels after 100 steps on the bench configuration."""
    p, sph, dem = slice_bed
    e32 = _engine(p, sph, dem, 0)
    e64 = _engine(p, sph, dem, 1)
    e32.step(100)
    e64.step(100)
    bad = _fp32_bad(_field_errors(e32, e64, SPH_ALL, DEM_ALL))
    assert not bad, sorted(bad.items(), key=lambda kv: -kv[1])
