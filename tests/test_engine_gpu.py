"""Parity of the CUDA engine (through the C ABI) with the CPU oracle.

Bar (written into each assert):
* integer and index work bit-exact: cell keys, sort order, neighbour
  lists, particle types, contact-history partner ids;
* FP64 build vs oracle: rel. L2 <= 1e-9 per field (rounding and FMA only);
* FP32 build vs oracle: rel. L2 <= 1e-5 per field after 100 steps on a
  bed without initial contacts, the tolerance of the specification for
  the FP32 paths.
"""
import os
import tempfile

import numpy as np
import pytest

from fluidized_bed_master_b200.beds import spouted_bed, write_input_dir
from fluidized_bed_master_b200.params import DEM, SPH
from oracle import Oracle
from tests.helpers import by_id, history_map, rel_l2

pytestmark = pytest.mark.gpu

SPH_REAL = ["x", "y", "z", "ux", "uy", "uz", "m", "rho", "pres", "temp", "DEMpor", "dDEMpor", "flt_s",
            "ftotalx", "ftotaly", "ftotalz", "fpx", "fpy", "fpz", "pgfx", "pgfy", "pgfz", "rho_ref"]
DEM_REAL = ["x", "y", "z", "ux", "uy", "uz", "wx", "wy", "wz", "temp", "DEMpor", "flt_s", "flt_sd", "flt_sd2",
            "Fdx_df", "Fdy_df", "Fdz_df", "ftotalx", "ftotaly", "ftotalz", "torqx", "torqy", "torqz"]


def _engine(p, sph, dem, prec):
    from fluidized_bed_master_b200.engine import Engine

    q = p.copy()
    q.precision = prec
    return Engine(q, sph, dem)


def _ids(src, which):
    return src.get(which, "pid") if which == SPH else src.get(which, "dem_idx")


def _compare(eng, orc, fields_s, fields_d, tol, label):
    bad = []
    for which, fields in ((SPH, fields_s), (DEM, fields_d)):
        n = eng.nd if which == DEM else eng.ns
        if n == 0:
            continue
        ie, io = _ids(eng, which), _ids(orc, which)
        for f in fields:
            a = by_id(ie, eng.get(which, f))
            b = by_id(io, orc.get(which, f))
            e = rel_l2(a, b)
            if not (e <= tol):
                bad.append((label, "dem" if which else "sph", f, e))
    return bad


@pytest.fixture(scope="module")
def contact_bed():
    return spouted_bed(dx=2.0e-3, n_dem=100000, r_dem=1.0e-3, seed=21, spacing=1.9, u_dem=0.05)


@pytest.fixture(scope="module")
def calm_bed():
    return spouted_bed(dx=2.0e-3, n_dem=100000, r_dem=1.0e-3, seed=22, spacing=2.1)


@pytest.mark.parametrize("prec", [0, 1])
def test_cells_sort_and_neighbor_lists_bit_exact(contact_bed, prec):
    p, sph, dem = contact_bed
    eng = _engine(p, sph, dem, prec)
    orc = Oracle(p, sph, dem, threads=8)
    for k in range(3):
        eng.step(1)
        orc.step(1)
        for which in (SPH, DEM):
            assert np.array_equal(_ids(eng, which), _ids(orc, which)), "sorted order differs"
            assert np.array_equal(eng.get(which, "cell"), orc.get(which, "cell")), "cell keys differ"
        ce, le = eng.neighbors()
        co, lo = orc.neighbors()
        assert np.array_equal(ce, co), "neighbour counts differ"
        assert ce.max() <= le.shape[1]
        for i in range(eng.ns):
            assert np.array_equal(le[i, : ce[i]], lo[i, : co[i]]), f"neighbour list of slot {i} differs"


def test_fp64_matches_oracle_contact_bed(contact_bed):
    """FP64 build vs oracle: rel. L2 <= 1e-9 per field after 1 and 8 steps."""
    p, sph, dem = contact_bed
    eng = _engine(p, sph, dem, 1)
    orc = Oracle(p, sph, dem, threads=8)
    bad = []
    done = 0
    for cp in (1, 8):
        eng.step(cp - done)
        orc.step(cp - done)
        done = cp
        bad += _compare(eng, orc, SPH_REAL, DEM_REAL, 1e-9, f"step{cp}")
        for f in ("p_type", "i_type", "buffer_type"):
            assert np.array_equal(by_id(_ids(eng, SPH), eng.get(SPH, f)), by_id(_ids(orc, SPH), orc.get(SPH, f)))
        ie, se = eng.history()
        io_, so = orc.history()
        me = history_map(ie.astype(float), se)
        mo = history_map(io_, so)
        ide = _ids(eng, DEM)
        ido = _ids(orc, DEM)
        he = {int(ide[i]): me[i] for i in range(eng.nd)}
        ho = {int(ido[i]): mo[i] for i in range(orc.nd)}
        for k in ho:
            assert set(he[k]) == set(ho[k]), f"contact partners of sphere {k} differ"
            for j in ho[k]:
                assert np.allclose(he[k][j], ho[k][j], rtol=1e-9, atol=1e-18)
        assert sum(len(v) for v in ho.values()) > 0, "the bed has no contacts: the test would be vacuous"
    assert not bad, bad


def test_fp64_matches_oracle_heat(contact_bed):
    p, sph, dem = contact_bed
    q = p.copy()
    q.con_solve = 1
    eng = _engine(q, sph, dem, 1)
    orc = Oracle(q, sph, dem, threads=8)
    eng.step(5)
    orc.step(5)
    bad = _compare(eng, orc, SPH_REAL + ["dtemp"], DEM_REAL + ["dtemp"], 1e-9, "heat")
    assert not bad, bad


def test_fp32_within_1e5_after_100_steps(calm_bed):
    """FP32 build vs the FP64 oracle: rel. L2 <= 1e-5 after 100 steps."""
    p, sph, dem = calm_bed
    eng = _engine(p, sph, dem, 0)
    orc = Oracle(p, sph, dem, threads=8)
    eng.step(100)
    orc.step(100)
    fs = ["x", "y", "z", "ux", "uy", "uz", "m", "rho", "pres", "temp", "DEMpor"]
    fd = ["x", "y", "z", "ux", "uy", "uz", "temp", "DEMpor"]
    bad = _compare(eng, orc, fs, fd, 1e-5, "fp32-100")
    assert not bad, bad


RATE_FIELDS = {"dDEMpor", "ftotalx", "ftotaly", "ftotalz", "fpx", "fpy", "fpz", "pgfx", "pgfy", "pgfz", "Fdx_df",
               "Fdy_df", "Fdz_df", "torqx", "torqy", "torqz", "dtemp"}


def test_fp32_vs_fp64_engine_builds(calm_bed):
    """Every field of the FP32 build against the FP64 build of the same
    kernels after 100 steps: state fields within rel. L2 1e-5, rate fields
    (forces, gradients, torques, heat rates) within 1e-4."""
    p, sph, dem = calm_bed
    e32 = _engine(p, sph, dem, 0)
    e64 = _engine(p, sph, dem, 1)
    e32.step(100)
    e64.step(100)
    bad = {}
    for which, fields in ((SPH, SPH_REAL), (DEM, DEM_REAL)):
        for f in fields:
            e = rel_l2(by_id(_ids(e32, which), e32.get(which, f)), by_id(_ids(e64, which), e64.get(which, f)))
            if not e <= (1e-4 if f in RATE_FIELDS else 1e-5):
                bad[("dem" if which else "sph", f)] = e
    assert not bad, sorted(bad.items(), key=lambda kv: -kv[1])


@pytest.mark.parametrize("prec", [0, 1])
def test_dem_list_cap_walks_stencil_bit_identical(contact_bed, prec):
    """The SPH kernels that sum over DEM spheres walk the per-step SPH -> DEM
    list, or the 27-cell stencil for a particle with more DEM neighbours than
    the list holds.  Both visit the same spheres in the same order, so a cap
    of one entry (nearly every particle in the bed walks its stencil) gives
    the same bits as the auto-sized list."""
    p, sph, dem = contact_bed
    a = _engine(p, sph, dem, prec)
    q = p.copy()
    q.dem_list_cap = 1
    b = _engine(q, sph, dem, prec)
    a.step(5)
    b.step(5)
    for which, fields in ((SPH, SPH_REAL), (DEM, DEM_REAL)):
        assert np.array_equal(_ids(a, which), _ids(b, which))
        for f in fields:
            assert np.array_equal(a.get(which, f), b.get(which, f)), ("dem" if which else "sph", f)


@pytest.mark.parametrize("prec", [0, 1])
def test_dem_branch_concurrency_bit_identical(contact_bed, prec):
    """The DEM kernels that read no SPH pass run on a second stream forked
    from the step stream; run serialised on the step stream
    (sphdem_set_concurrency(h, 0)), the same step gives the same bits, with
    graphs and without, and switching back and forth mid-run changes
    nothing."""
    p, sph, dem = contact_bed
    a = _engine(p, sph, dem, prec)
    b = _engine(p, sph, dem, prec)
    b.set_concurrency(False)
    c = _engine(p, sph, dem, prec)
    c.set_graphs(False)
    a.step(4)
    b.step(4)
    c.step(2)
    c.set_concurrency(False)
    c.step(1)
    c.set_concurrency(True)
    c.step(1)
    for which, fields in ((SPH, SPH_REAL), (DEM, DEM_REAL)):
        for e in (b, c):
            assert np.array_equal(_ids(a, which), _ids(e, which))
            for f in fields:
                assert np.array_equal(a.get(which, f), e.get(which, f)), ("dem" if which else "sph", f)
    ia, sa = a.history()
    for e in (b, c):
        ie, se = e.history()
        assert np.array_equal(ia, ie) and np.array_equal(sa, se)


def test_stats_and_time(calm_bed):
    p, sph, dem = calm_bed
    eng = _engine(p, sph, dem, 0)
    eng.step(3)
    t, c = eng.time()
    assert c == 3 and abs(t - 3 * p.dt) < 1e-15
    s = eng.stats()
    assert s["count"] == 3 and s["overflow_flags"] == 0 and s["nan_flag"] == 0
    orc = Oracle(p, sph, dem, threads=8)
    orc.step(3)
    m = (orc.get(SPH, "p_type") != 0) & (orc.get(SPH, "i_type") < 2)
    assert abs(s["rho_max_sph"] - orc.get(SPH, "rho")[m].max()) <= 1e-5 * orc.get(SPH, "rho")[m].max()
    assert eng.launches() > 0


def test_from_dir_equals_arrays(calm_bed):
    from fluidized_bed_master_b200.engine import Engine

    p, sph, dem = calm_bed
    with tempfile.TemporaryDirectory() as d:
        write_input_dir(d, p, sph, dem)
        e1 = Engine.from_dir(d, precision=1)
        e2 = _engine(p, sph, dem, 1)
        e1.step(2)
        e2.step(2)
        for f in ("pres", "uz", "rho"):
            assert rel_l2(by_id(_ids(e1, SPH), e1.get(SPH, f)), by_id(_ids(e2, SPH), e2.get(SPH, f))) < 1e-12


def test_restart_roundtrip(calm_bed):
    from fluidized_bed_master_b200.engine import Engine, read_input_txt

    p, sph, dem = calm_bed
    e = _engine(p, sph, dem, 1)
    e.step(2)
    with tempfile.TemporaryDirectory() as d:
        path = os.path.join(d, "input.txt")
        e.write_restart(path)
        s2, d2 = read_input_txt(path)
        assert len(s2["x"]) == e.ns and len(d2["x"]) == e.nd
        assert np.allclose(s2["uz"], e.get(SPH, "uz"), rtol=0, atol=1e-12)
        assert np.array_equal(d2["dem_idx"], e.get(DEM, "dem_idx"))


def test_vtk_dem_layout(calm_bed):
    p, sph, dem = calm_bed
    e = _engine(p, sph, dem, 0)
    e.step(1)
    with tempfile.TemporaryDirectory() as d:
        path = os.path.join(d, "dem.vtk")
        e.write_vtk_dem(path)
        raw = open(path, "rb").read()
    assert raw.startswith(b"# vtk DataFile Version 3.0\nPrint out results in vtk format\nBINARY\nDATASET POLYDATA\n")
    n = e.nd
    head = f"POINTS\t{n}\tfloat\n".encode()
    k = raw.index(head) + len(head)
    xyz = np.frombuffer(raw[k:k + 12 * n], dtype=">f4").reshape(n, 3)
    assert np.allclose(xyz[:, 2], e.get(DEM, "z").astype(np.float32))
    for name in (b"itype", b"mag_uijf", b"Euler", b"porosity", b"uz", b"Q_sd", b"ftotal_z",
                 b"temperature_surface", b"rad", b"dtemp_dt"):
        assert name + f"\t1\t{n}\tfloat\n".encode() in raw


def test_kernel_timing_mode(calm_bed):
    """In-graph event timing: every engine kernel of the step reports a time."""
    p, sph, dem = calm_bed
    e = _engine(p, sph, dem, 0)
    e.step(1)
    e.set_timing(True)
    for _ in range(3):
        e.step(1)
        e.collect_timing()
    t = e.timing()
    for k in ("build_list", "passA", "passB", "ppe", "passC", "dem_contact", "dem_coupling", "xsph"):
        ms, n = t[k]
        assert n == 3 and ms > 0, (k, ms, n)
    e.set_timing(False)
    e.step(2)


@pytest.mark.parametrize("prec", [0, 1])
def test_bulk_field_transfer(calm_bed, prec):
    """sphdem_get_fields equals per-field reads; sphdem_set_fields writes what
    sphdem_set_field writes (both convert to the field precision)."""
    p, sph, dem = calm_bed
    e = _engine(p, sph, dem, prec)
    e.step(2)
    for which, names in ((SPH, ["x", "uz", "m", "rho", "pres", "temp", "flt_s"]),
                         (DEM, ["x", "ux", "wz", "temp", "Q_sd", "ftotalz"])):
        n = e.nd if which == DEM else e.ns
        bulk = {f: np.empty(n) for f in names}
        e.get_fields(which, bulk)
        for f in names:
            assert np.array_equal(bulk[f], e.get(which, f)), f
        settable = [f for f in names if f != "ftotalz"]
        rng = np.random.default_rng(5)
        new = {f: bulk[f] * (1.0 + 1e-3 * rng.standard_normal(n)) for f in settable}
        e.set_fields(which, new)
        # the DEM set and positions are FP64 in both builds; SPH fields are
        # FP32 in the FP32 build, and the SPH temperature is stored as
        # T - t_ref with t_ref the FP32-rounded mean input temperature
        t_ref = float(np.float32(np.mean(sph["temp"])))
        for f in settable:
            ref = new[f]
            if prec == 0 and which == SPH and f == "temp":
                ref = (new[f] - t_ref).astype(np.float32).astype(np.float64) + t_ref
            elif prec == 0 and which == SPH and f != "x":
                ref = new[f].astype(np.float32).astype(np.float64)
            assert np.array_equal(e.get(which, f), ref), f
    with pytest.raises(Exception):
        e.set_fields(SPH, {"ftotalx": np.zeros(e.ns)})


@pytest.mark.parametrize("prec", [0, 1])
def test_bulk_transfer_pinned_equals_pageable(contact_bed, prec):
    """Page-locked host arrays are read and written in place by the transfer
    kernels (mapped memory); pageable arrays go through copies.  Both give
    the same bits, for fields and for the contact history."""
    import torch

    p, sph, dem = contact_bed
    e = _engine(p, sph, dem, prec)
    e.step(3)

    def pinned(shape, dt):
        return torch.empty(int(np.prod(shape)), dtype=dt, pin_memory=True).numpy().reshape(shape)

    for which, names in ((SPH, ["x", "uz", "m", "rho", "pres", "temp", "flt_s", "dDEMpor"]),
                         (DEM, ["x", "uy", "wz", "temp", "Fdz_df", "Q_sd", "ftotalz"])):
        n = e.nd if which == DEM else e.ns
        a = {f: np.empty(n) for f in names}
        b = {f: pinned((n,), torch.float64) for f in names}
        e.get_fields(which, a)
        e.get_fields(which, b)
        for f in names:
            assert np.array_equal(a[f], b[f]), f
        settable = [f for f in names if f != "ftotalz"]
        rng = np.random.default_rng(9)
        for f in settable:
            b[f][:] = b[f] * (1.0 + 1e-3 * rng.standard_normal(n))
        e.set_fields(which, {f: b[f] for f in settable})
        after_pinned = {f: e.get(which, f) for f in settable}
        e.set_fields(which, {f: np.array(b[f]) for f in settable})
        for f in settable:
            assert np.array_equal(e.get(which, f), after_pinned[f]), f
    ids, sp = e.history()
    pid, psp = pinned((e.nd, 16), torch.int32), pinned((e.nd, 16, 3), torch.float64)
    e.history(out=(pid, psp))
    assert np.array_equal(ids, pid) and np.array_equal(sp, psp)
    psp[:] = psp * 0.5
    e.set_history(pid, psp)
    got_ids, got_sp = e.history()
    assert np.array_equal(got_ids, ids) and np.array_equal(got_sp, sp * 0.5)


def test_history_roundtrip_keeps_the_run(contact_bed):
    """get_history -> set_history is the identity, and a run continued after
    a round trip of the whole state equals the uninterrupted run."""
    p, sph, dem = contact_bed
    a = _engine(p, sph, dem, 1)
    b = _engine(p, sph, dem, 1)
    a.step(3)
    b.step(3)
    ids, sp = b.history()
    assert (ids > 0).sum() > 0
    b.set_history(np.zeros_like(ids), np.zeros_like(sp))
    assert (b.history()[0] > 0).sum() == 0
    b.set_history(ids, sp)
    i2, s2 = b.history()
    assert np.array_equal(ids, i2) and np.array_equal(sp, s2)
    a.step(3)
    b.step(3)
    for f in ("x", "uz", "wx"):
        assert np.array_equal(a.get(DEM, f), b.get(DEM, f)), f


@pytest.mark.parametrize("case", ["column", "bed"])
@pytest.mark.parametrize("prec", [0, 1])
def test_clamped_particle_takes_the_exact_path(case, prec):
    """The last input row does not enter the bounding box (the reference's
    box skips it), so a last row placed three cells beyond the box is
    clamped into a boundary cell.  The cell-tiled scans (list build, wall
    Neumann pass, SPH -> DEM list) stage coordinates relative to a particle
    of the cell and use the FP32 prefilter only for positions within two
    cell widths of it; this one must take the FP64 predicate.  Bar: sorted
    order, cell keys and neighbour lists bit-exact against the oracle over
    two steps; the FP64 build's SPH fields within rel. L2 1e-9 (a sphere
    that far has no fluid around it, and the reference's drag closure
    turns its own state non-finite, in the oracle and the engine alike)."""
    from fluidized_bed_master_b200.beds import box_bed, isph_column

    if case == "column":
        # the last row is a wall particle of the closed box
        p, sph, dem = isph_column(dx=1.0e-2, seed=9)
        p.ppe_mode = 0
        sph = {k: np.array(v, copy=True) for k, v in sph.items()}
        dcell = 1.1 * p.kappa * sph["h"][0]
        sph["x"][-1] = sph["x"][:-1].max() + 3.0 * dcell
    else:
        # spheres inside the fluid layer; the last row is a sphere
        p, sph, dem = box_bed(n_fluid=8000, n_dem=300, dem_height=0.006, seed=9)
        dem = {k: np.array(v, copy=True) for k, v in dem.items()}
        dcell = 1.1 * p.kappa * sph["h"][0]
        dem["x"][-1] = max(sph["x"].max(), dem["x"][:-1].max()) + 3.0 * dcell
    eng = _engine(p, sph, dem, prec)
    orc = Oracle(p, sph, dem, threads=8)
    for _ in range(2):
        eng.step(1)
        orc.step(1)
        for which in (SPH, DEM):
            if (eng.nd if which == DEM else eng.ns) == 0:
                continue
            assert np.array_equal(_ids(eng, which), _ids(orc, which)), "sorted order differs"
            assert np.array_equal(eng.get(which, "cell"), orc.get(which, "cell")), "cell keys differ"
        ce, le = eng.neighbors()
        co, lo = orc.neighbors()
        assert np.array_equal(ce, co), "neighbour counts differ"
        for i in range(eng.ns):
            assert np.array_equal(le[i, : ce[i]], lo[i, : co[i]]), f"neighbour list of slot {i} differs"
    if prec == 1:
        bad = _compare(eng, orc, SPH_REAL, [], 1e-9, case)
        assert not bad, bad
