"""The two-dimensional ISPH-DEM bed (beds.box_bed_2d, dim 2): the engine
against the oracle's restatement of the same 2-D model.

The model (the reference's ISPH step is three-dimensional only): the bed
lies in a plane y = const; 2-D kernel normalisation and SPH volume
(h / h_over_dx)^2; the gradient correction on the x-z block; spheres with
their centres in the plane keep the sphere contact, drag and heat laws,
enter the porosity with the disc area 3.14159 r^2 of the reference's 2-D
coupling prep (functions_PREP2.cuh:2944-3033) and act on the fluid per
unit depth (depth 4 r / 3).  Parity is against the oracle only (no
reference run exists for it).

Bed: 8,000 fluid particles, 80 columns at dx = 1.25 mm, 800 spheres, in
the plane y = 0.0125 m.  Bars (in each assert):
* the state stays in the plane: y, the in-plane normal velocity uy, the
  DEM angular velocity components wx, wz and the torques about x and z
  exactly as set (0);
* FP64 build vs the oracle after 20 and after 100 steps (the spheres
  start apart; the first contacts form after about 40 steps): sorted
  order, neighbour lists and contact partners exact, every field and
  tangential spring within rel. 1e-9 (measured 5.5e-13 at step 100);
* FP32 build vs the oracle over 60 steps: lists and partners exact every
  10 steps; state fields within rel. L2 1e-5, rate fields within 1e-4.
"""
import numpy as np
import pytest

from fluidized_bed_master_b200.beds import box_bed_2d
from fluidized_bed_master_b200.params import DEM, SPH
from oracle import Oracle
from tests.test_box_bed_gpu import (DEM_ALL, SPH_ALL, _check_lists_and_partners, _engine, _field_errors, _fp32_bad,
                                    _partners)

pytestmark = pytest.mark.gpu
Y0 = 0.0125


@pytest.fixture(scope="module")
def bed2d():
    return box_bed_2d(n_fluid=8000, seed=5, y0=Y0)


def _in_plane(src):
    for which in (SPH, DEM):
        assert np.all(src.get(which, "y") == Y0), "a particle left the plane"
        assert np.all(src.get(which, "uy") == 0.0), "an out-of-plane velocity appeared"
    assert np.all(src.get(DEM, "wx") == 0.0) and np.all(src.get(DEM, "wz") == 0.0), "an in-plane spin axis appeared"
    assert np.all(src.get(DEM, "torqx") == 0.0) and np.all(src.get(DEM, "torqz") == 0.0), "a torque left the y axis"


def test_bed2d_fp64_vs_oracle(bed2d):
    p, sph, dem = bed2d
    eng = _engine(p, sph, dem, 1)
    orc = Oracle(p, sph, dem, threads=16)
    eng.step(20)
    orc.step(20)
    _check_lists_and_partners(eng, orc, "step 20")
    err = _field_errors(eng, orc, SPH_ALL, DEM_ALL)
    bad = {k: v for k, v in err.items() if not v <= 1e-9}
    assert not bad, sorted(bad.items(), key=lambda kv: -kv[1])
    eng.step(80)
    orc.step(80)
    contacts = _check_lists_and_partners(eng, orc, "step 100")
    assert contacts > 20, "too few contacts for the history to be exercised"
    _in_plane(eng)
    _in_plane(orc)
    err = _field_errors(eng, orc, SPH_ALL, DEM_ALL)
    bad = {k: v for k, v in err.items() if not v <= 1e-9}
    assert not bad, sorted(bad.items(), key=lambda kv: -kv[1])
    pe, po = _partners(eng), _partners(orc)
    for k, v in po.items():
        for j, s in v.items():
            assert np.allclose(pe[k][j], s, rtol=1e-9, atol=1e-18), (k, j)


def test_bed2d_fp32_vs_oracle(bed2d):
    p, sph, dem = bed2d
    eng = _engine(p, sph, dem, 0)
    orc = Oracle(p, sph, dem, threads=16)
    for k in range(6):
        eng.step(10)
        orc.step(10)
        _check_lists_and_partners(eng, orc, f"step {10 * (k + 1)}")
    _in_plane(eng)
    bad = _fp32_bad(_field_errors(eng, orc, SPH_ALL, DEM_ALL))
    assert not bad, sorted(bad.items(), key=lambda kv: -kv[1])
