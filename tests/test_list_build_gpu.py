"""The SPH list build's modes (sphdem_set_list_build / get): one thread per
particle (1) and one warp per cell with 2, 4 or 8 cells per block, and the
default (0) that times the four at commit and keeps the fastest.  A fixed
mode also fixes the SPH -> DEM list build (1: a thread per particle, 2/4/8:
a warp per cell), so the modes compare both of its kernels too.

Bar: on the 3-D bed slice and on a 2-D bed (FP32 build), every mode gives
the same neighbour lists and, after 5 steps, every field bit for bit equal
to the per-particle mode; the default reports one of the four; an FP64
handle builds per particle; other modes are refused.
"""
import numpy as np
import pytest

from fluidized_bed_master_b200.beds import box_bed, box_bed_2d
from fluidized_bed_master_b200.params import DEM, SPH
from tests.test_box_bed_gpu import DEM_ALL, SPH_ALL

pytestmark = pytest.mark.gpu


def _engine(p, sph, dem, prec, mode):
    from fluidized_bed_master_b200.engine import Engine

    q = p.copy()
    q.precision = prec
    return Engine(q, sph, dem, list_build=mode)


@pytest.mark.parametrize("bed", ["3d", "2d"])
def test_list_modes_agree(bed):
    if bed == "3d":
        p, sph, dem = box_bed(n_fluid=20_000, n_dem=2_000, dem_height=0.01, seed=7)
    else:
        p, sph, dem = box_bed_2d(n_fluid=6_000, seed=7)
    ref = _engine(p, sph, dem, 0, 1)
    ref.step(5)
    cnt0, lst0 = ref.neighbors(cap=256)
    for mode in (2, 4, 8, 0):
        e = _engine(p, sph, dem, 0, mode)
        got = e.list_build()
        assert got == mode if mode else got in (1, 2, 4, 8)
        e.step(5)
        cnt, lst = e.neighbors(cap=256)
        assert np.array_equal(cnt, cnt0) and np.array_equal(lst, lst0), f"mode {mode}: lists differ"
        for which, fields in ((SPH, SPH_ALL), (DEM, DEM_ALL)):
            for f in fields:
                assert np.array_equal(e.get(which, f), ref.get(which, f)), f"mode {mode}: {f} differs"
        e.close()


def test_list_mode_fp64_and_refusals():
    from fluidized_bed_master_b200.engine import SphdemError

    p, sph, dem = box_bed_2d(n_fluid=3_000, seed=8)
    assert _engine(p, sph, dem, 1, 0).list_build() == 1
    with pytest.raises(SphdemError):
        _engine(p, sph, dem, 0, 3)
