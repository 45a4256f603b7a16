"""Failure paths of the engine, driven from the host; none faults or hangs a GPU.

The reference exits the process on a CUDA error (CUDA_CHECK, ISPH.cuh:1-8)
and has no check of its own state.  The engine keeps every kernel in
bounds and reports through status codes instead:
* a NaN put into the state through sphdem_set_field -> sphdem_check
  returns SPHDEM_E_NAN;
* a sphere that meets a 17th contact partner (16 history slots,
  class_Cuda_Particle_Array2.cuh:57-58) -> SPHDEM_E_OVERFLOW; the sphere
  keeps 16 valid partners and the oracle, which also leaves the 17th
  unrecorded, agrees on them;
* neighbour lists that outgrow their capacity (particles squeezed after
  commit) -> SPHDEM_E_OVERFLOW, and the handle still answers;
* a bounded tensor-core wait made to run out (SPHDEM_FAULT_DRILL=mlp_wait
  withholds the MMA that would complete it) -> SPHDEM_E_TIMEOUT, and the
  next call on the same context succeeds with the same output, so the
  kernel freed its tensor memory.
"""
import ctypes as C
import os

import numpy as np
import pytest

from fluidized_bed_master_b200.beds import _dem_arrays, spouted_bed
from fluidized_bed_master_b200.params import DEM, SPH
from oracle import Oracle
from tests.helpers import history_map

pytestmark = pytest.mark.gpu

E_OVERFLOW, E_NAN, E_TIMEOUT = -4, -5, -6


def _engine(p, sph, dem, prec=0):
    from fluidized_bed_master_b200.engine import Engine

    q = p.copy()
    q.precision = prec
    return Engine(q, sph, dem)


@pytest.fixture(scope="module")
def calm_bed():
    return spouted_bed(dx=2.0e-3, n_dem=100000, r_dem=1.0e-3, seed=22, spacing=2.1)


def test_nan_in_state_is_reported(calm_bed):
    p, sph, dem = calm_bed
    eng = _engine(p, sph, dem)
    eng.step(2)
    assert eng.check() == 0
    uz = eng.get(SPH, "uz")
    fluid = np.flatnonzero(eng.get(SPH, "p_type") == 1)
    uz[fluid[len(fluid) // 2]] = np.nan
    eng.set(SPH, "uz", uz)
    eng.step(1)
    assert eng.check() == E_NAN
    assert eng.check() == E_NAN, "the flag must stay set"


def _cluster_bed(n_partners=17):
    """A sphere of radius 1 mm with n_partners spheres of 0.5 mm around it,
    each overlapping it by 1 um and clear of one another (Fibonacci points on
    a 1.499 mm shell), inside the fluid of the spouted bed."""
    p, sph, _ = spouted_bed(dx=2.0e-3, n_dem=1, r_dem=1.0e-3, seed=23)
    c = np.array([0.0, 0.0, 0.004])
    k = np.arange(n_partners) + 0.5
    th = np.arccos(1.0 - 2.0 * k / n_partners)
    ph = np.pi * (1.0 + 5.0 ** 0.5) * k
    d = np.stack([np.sin(th) * np.cos(ph), np.sin(th) * np.sin(ph), np.cos(th)], 1)
    rad = np.concatenate([[1.0e-3], np.full(n_partners, 0.5e-3)])
    pos = np.concatenate([c[None, :], c[None, :] + (1.5e-3 - 1.0e-6) * d])
    gap = np.linalg.norm(pos[1:, None, :] - pos[None, 1:, :], axis=2) + np.eye(n_partners)
    assert gap.min() > 1.0e-3, "partners must not touch one another"
    dem = _dem_arrays(pos, rad, 2500.0, sph["h"][0], 300.0)
    return p, sph, dem


def _partners_of(src, dem_id):
    ids, springs = src.history()
    m = history_map(np.asarray(ids, dtype=float), springs)
    k = int(np.flatnonzero(src.get(DEM, "dem_idx") == dem_id)[0])
    return set(m[k])


def test_seventeenth_contact_partner_is_reported():
    """A new contact takes the first slot free at the start of the step, so
    the 17 partners enter one per step; the 17th finds no slot."""
    p, sph, dem = _cluster_bed(17)
    eng = _engine(p, sph, dem, prec=1)
    orc = Oracle(p, sph, dem, threads=8)
    eng.step(16)
    orc.step(16)
    assert eng.check() == 0
    assert len(_partners_of(eng, 1)) == 16
    eng.step(4)
    orc.step(4)
    assert eng.check() == E_OVERFLOW
    pe, po = _partners_of(eng, 1), _partners_of(orc, 1)
    assert len(pe) == 16 and pe <= set(range(2, 19)), pe
    assert pe == po, "the oracle leaves the same partner out"
    for f in ("x", "y", "z", "ux", "uz"):
        assert np.isfinite(eng.get(DEM, f)).all(), f


def test_neighbour_list_overflow_is_reported(calm_bed):
    """Lists are sized at commit (1.25 x the largest count); squeezing the
    particles toward the bed's centre afterwards roughly doubles the counts.
    The list build keeps the first `capacity` entries and every pass walks
    at most that many, so the step stays in bounds and the handle answers."""
    p, sph, dem = calm_bed
    eng = _engine(p, sph, dem)
    eng.step(1)
    assert eng.check() == 0
    pos = {f: eng.get(SPH, f) for f in ("x", "y", "z")}
    cen = {f: 0.5 * (v.min() + v.max()) for f, v in pos.items()}
    for f, v in pos.items():
        eng.set(SPH, f, cen[f] + 0.75 * (v - cen[f]))
    eng.step(1)
    assert eng.check() == E_OVERFLOW
    counts, _ = eng.neighbors(cap=1)
    assert counts.max() > 0
    assert eng.get(SPH, "pid").shape == (eng.ns,)


def test_mlp_wait_drill_times_out_and_recovers():
    import torch

    from fluidized_bed_master_b200.engine import lib

    L = lib()
    L.sphdem_mlp_param_count.restype = C.c_int32
    L.sphdem_mlp_forward.argtypes = [C.c_void_p, C.c_int32, C.c_void_p, C.c_void_p, C.c_void_p]
    npar = L.sphdem_mlp_param_count()
    g = torch.Generator(device="cpu").manual_seed(7)
    n = 4096
    feat = torch.randn(n, 16, generator=g).to(torch.bfloat16).cuda()
    params = (0.2 * torch.randn(npar, generator=g)).float().cuda()
    out = torch.zeros(n, dtype=torch.float32, device="cuda")
    stream = torch.cuda.current_stream().cuda_stream

    def fwd():
        return L.sphdem_mlp_forward(feat.data_ptr(), n, params.data_ptr(), out.data_ptr(), stream)

    assert fwd() == 0
    ref = out.clone()
    os.environ["SPHDEM_FAULT_DRILL"] = "mlp_wait"
    try:
        assert fwd() == E_TIMEOUT
    finally:
        del os.environ["SPHDEM_FAULT_DRILL"]
    for _ in range(2):
        out.zero_()
        assert fwd() == 0, "the context must stay usable after the drill"
        assert torch.equal(out, ref)
