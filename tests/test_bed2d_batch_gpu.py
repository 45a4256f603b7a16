"""Several 2-D ISPH-DEM beds in one handle (sphdem_set_beds;
beds.bed2d_batch): each bed in its own plane y = const with its own inlet
velocity and outlet slab, all stepped by the one step graph.

Batch: 5 beds of 1,500 - 6,000 fluid particles (log-uniform, seeded), 10 %
spheres, inlet velocities U(0.1, 0.3).  Bars (in each assert):
* every bed of the batch equals the same bed run alone in a handle of its
  own on the batch's cell grid (sphdem_set_domain), bit for bit, in the
  FP64 and the FP32 build, after 20 steps: no pair crosses two beds, and a
  bed's sums run in the same order;
* the FP64 batch against the oracle on the same beds (oracle_set_beds)
  after 20 steps: neighbour lists and contact partners exact, every field
  within rel. L2 1e-9;
* planes closer than two cells are refused at commit (SPHDEM_E_INPUT),
  empty or non-finite rows and 3-D handles by sphdem_set_beds;
* the bench's 64-bed batch, FP64 against the oracle after 3 steps (its
  sphere count selects the thread-per-sphere DEM passes).
"""
import numpy as np
import pytest

from fluidized_bed_master_b200.beds import bed2d_batch
from fluidized_bed_master_b200.params import DEM, SPH
from oracle import Oracle
from tests.test_box_bed_gpu import DEM_ALL, SPH_ALL, _check_lists_and_partners, _field_errors

pytestmark = pytest.mark.gpu
STEPS = 20


@pytest.fixture(scope="module")
def batch():
    return bed2d_batch(n_beds=5, n_min=1500, n_max=6000, seed=3)


def _engine(p, sph, dem, prec, **kw):
    from fluidized_bed_master_b200.engine import Engine

    q = p.copy()
    q.precision = prec
    return Engine(q, sph, dem, **kw)


def _by_input_row(eng, which, f, lo, n):
    """Field f of the input rows lo .. lo + n - 1, in input order."""
    pid = eng.get(which, "pid")
    m = (pid >= lo) & (pid < lo + n)
    out = np.empty(n)
    out[pid[m] - lo] = eng.get(which, f)[m]
    return out


@pytest.mark.parametrize("prec", [1, 0])
def test_batch_beds_equal_beds_alone(batch, prec):
    from fluidized_bed_master_b200.engine import bed_domain

    p, sph, dem, rows, parts = batch
    dom = bed_domain(p, sph, dem)
    eb = _engine(p, sph, dem, prec, beds=rows)
    eb.step(STEPS)
    s0 = d0 = 0
    for b, (sb, db, rb) in enumerate(parts):
        ea = _engine(p, sb, db, prec, beds=rb, domain=dom)
        ea.step(STEPS)
        for which, lo, src, fields in ((SPH, s0, sb, SPH_ALL), (DEM, d0, db, DEM_ALL)):
            n = len(src["x"])
            for f in fields:
                a = _by_input_row(eb, which, f, lo, n)
                c = _by_input_row(ea, which, f, 0, n)
                assert np.array_equal(a, c), f"bed {b}: {'dem' if which else 'sph'} {f} differs from the bed alone"
        s0 += len(sb["x"])
        d0 += len(db["x"])


def test_batch_fp64_vs_oracle(batch):
    p, sph, dem, rows, parts = batch
    eng = _engine(p, sph, dem, 1, beds=rows)
    orc = Oracle(p, sph, dem, threads=16, beds=rows)
    eng.step(STEPS)
    orc.step(STEPS)
    _check_lists_and_partners(eng, orc, f"step {STEPS}")
    err = _field_errors(eng, orc, SPH_ALL, DEM_ALL)
    bad = {k: v for k, v in err.items() if not v <= 1e-9}
    assert not bad, sorted(bad.items(), key=lambda kv: -kv[1])


def test_close_planes_refused(batch):
    from fluidized_bed_master_b200.engine import SphdemError

    p, sph, dem, rows, parts = batch
    (s0, d0, r0), (s1, d1, r1) = parts[0], parts[1]
    r1 = [dict(r1[0], y=r0[0]["y"] + 1.9 * 1.1 * p.kappa * float(s0["h"][0]))]
    s1 = dict(s1, y=np.full(len(s1["x"]), r1[0]["y"]))
    d1 = dict(d1, y=np.full(len(d1["x"]), r1[0]["y"]))
    sph2 = {k: np.concatenate([s0[k], s1[k]]) for k in s0}
    dem2 = {k: np.concatenate([d0[k], d1[k]]) for k in d0}
    with pytest.raises(SphdemError):
        _engine(p, sph2, dem2, 0, beds=r0 + r1)


def test_large_batch_fp64_vs_oracle():
    """The bench's 64-bed batch (1,029,448 SPH and 94,181 DEM): with more
    than 65,536 spheres on 2-D beds the DEM contact, filter and coupling
    passes take a thread per sphere; FP64 against the oracle after 3 steps,
    lists and partners exact, every field within rel. L2 1e-9."""
    p, sph, dem, rows, parts = bed2d_batch(seed=0)
    assert len(dem["x"]) >= 65536
    eng = _engine(p, sph, dem, 1, beds=rows)
    orc = Oracle(p, sph, dem, threads=16, beds=rows)
    eng.step(3)
    orc.step(3)
    _check_lists_and_partners(eng, orc, "step 3")
    err = _field_errors(eng, orc, SPH_ALL, DEM_ALL)
    bad = {k: v for k, v in err.items() if not v <= 1e-9}
    assert not bad, sorted(bad.items(), key=lambda kv: -kv[1])


def test_set_beds_arguments(batch):
    """sphdem_set_beds refuses what it cannot honour: no rows or a non-finite
    row (SPHDEM_E_ARG), a 3-D handle (SPHDEM_E_UNSUPPORTED)."""
    from fluidized_bed_master_b200.beds import box_bed
    from fluidized_bed_master_b200.engine import SphdemError

    p, sph, dem, rows, parts = batch
    s0, d0, r0 = parts[0]
    with pytest.raises(SphdemError) as e:
        _engine(p, s0, d0, 0, beds=[])
    assert e.value.status == -1
    with pytest.raises(SphdemError) as e:
        _engine(p, s0, d0, 0, beds=[dict(r0[0], inlet_uz=float("nan"))])
    assert e.value.status == -1
    p3, s3, d3 = box_bed(n_fluid=2_000, n_dem=100, dem_height=0.005, seed=1)
    with pytest.raises(SphdemError) as e:
        _engine(p3, s3, d3, 0, beds=r0)
    assert e.value.status == -7
