"""VTK output of the engine against the reference's own files.

The reference writes a binary legacy-VTK file of the DEM set at the end of
every step with count % freq_output == 0 (save_plot_fluid_vtk_bin_solid_dem,
functions_OUTPUT.cuh:1135-1446, called from ISPH_Calc_seperate.cuh:489), so
its first file holds the state after the first step.  tests/golden/
make_golden.py kept that file (vtk_step0) for each ISPH-DEM fixture.  The
FP64 engine replays the fixture's input for one step and must write the same
bytes: header, point count, every big-endian float of the positions and of
the ten point arrays.

The fluid writer (save_plot_fluid_vtk_bin_fluid_sph, functions_OUTPUT.cuh:
445-651) is not called by the reference's live time loop, so there is no
reference file; its layout is checked against the engine's fields.
"""
import json
import os
import tempfile

import numpy as np
import pytest

from fluidized_bed_master_b200.params import SPH
from tests.helpers import golden_files, load_golden

pytestmark = pytest.mark.gpu

ISPH_GOLD = [p for p in golden_files() if json.loads(np.load(p)["meta"].tobytes()).get("solver", "isph") == "isph"]


def _engine(p, sph, dem, prec):
    from fluidized_bed_master_b200.engine import Engine

    q = p.copy()
    q.precision = prec
    return Engine(q, sph, dem)


@pytest.mark.parametrize("path", ISPH_GOLD, ids=[p.split("/")[-1] for p in ISPH_GOLD])
def test_dem_vtk_bytes_equal_reference(path):
    g, p, sph, dem = load_golden(path)
    assert "vtk_step0" in g.files, "fixture has no reference VTK file"
    ref = g["vtk_step0"].tobytes()
    eng = _engine(p, sph, dem, 1)
    eng.step(1)
    with tempfile.TemporaryDirectory() as d:
        out = os.path.join(d, "dem.vtk")
        eng.write_vtk_dem(out)
        got = open(out, "rb").read()
    assert len(got) == len(ref), (len(got), len(ref))
    if got != ref:
        a = np.frombuffer(got, dtype=np.uint8)
        b = np.frombuffer(ref, dtype=np.uint8)
        bad = np.flatnonzero(a != b)
        raise AssertionError(f"{len(bad)} bytes differ, first at offset {bad[0]}")


def _read_vtk(raw):
    """Parse the legacy-VTK POLYDATA the writers emit: {name: array}."""
    out = {}
    k = 0

    def line():
        nonlocal k
        e = raw.index(b"\n", k)
        s = raw[k:e].decode()
        k = e + 1
        return s

    for _ in range(4):
        line()
    _, n, _ = line().split("\t")
    n = int(n)
    out["points"] = np.frombuffer(raw[k:k + 12 * n], dtype=">f4").reshape(n, 3)
    k += 12 * n
    assert line() == f"POINT_DATA\t{n}"
    nf = int(line().split("\t")[1])
    for _ in range(nf):
        name, _, cnt, typ = line().split("\t")
        dt = ">f4" if typ == "float" else ">i4"
        out[name] = np.frombuffer(raw[k:k + 4 * int(cnt)], dtype=dt)
        k += 4 * int(cnt)
    assert k == len(raw)
    return out


def test_fluid_vtk_layout():
    g, p, sph, dem = load_golden(ISPH_GOLD[0])
    q = p.copy()
    q.con_solve = 1
    eng = _engine(q, sph, dem, 0)
    eng.step(2)
    with tempfile.TemporaryDirectory() as d:
        out = os.path.join(d, "fluid.vtk")
        eng.write_vtk_fluid(out)
        v = _read_vtk(open(out, "rb").read())
    fl = eng.get(SPH, "p_type") == 1
    assert v["points"].shape == (fl.sum(), 3)
    assert np.array_equal(v["points"][:, 2], eng.get(SPH, "z")[fl].astype(np.float32))
    for name, f in (("porosity", "DEMpor"), ("pressure", "pres"), ("dtemp", "dtemp"), ("density", "rho"),
                    ("temperature", "temp"), ("uz", "uz")):
        assert np.array_equal(v[name], eng.get(SPH, f)[fl].astype(np.float32)), name
    assert np.array_equal(v["buffer_type"], eng.get(SPH, "buffer_type")[fl])
    assert not v["conv_rate"].any() and not v["cond_rate"].any()
    assert list(v)[1:] == ["porosity", "conv_rate", "pressure", "cond_rate", "dtemp", "buffer_type", "density",
                           "temperature", "uz"]


def test_snapshot_files_equal_sync_writers():
    """sphdem_snapshot copies the output fields while the next steps run;
    sphdem_write_snapshot then writes the files of the snapshot's step,
    byte-identical to the synchronous writers at that step, and the run
    itself is unchanged by the snapshot."""
    g, p, sph, dem = load_golden(ISPH_GOLD[0])
    q = p.copy()
    q.con_solve = 1
    a = _engine(q, sph, dem, 0)
    b = _engine(q, sph, dem, 0)
    a.step(3)
    a.snapshot()
    a.step(2)                      # runs while the snapshot is copied out
    b.step(3)
    with tempfile.TemporaryDirectory() as d:
        ad, af = os.path.join(d, "a_dem.vtk"), os.path.join(d, "a_fluid.vtk")
        bd, bf = os.path.join(d, "b_dem.vtk"), os.path.join(d, "b_fluid.vtk")
        a.write_snapshot(ad, af)
        b.write_vtk_dem(bd)
        b.write_vtk_fluid(bf)
        for x, y in ((ad, bd), (af, bf)):
            assert open(x, "rb").read() == open(y, "rb").read(), os.path.basename(x)
    b.step(2)
    for f in ("x", "uz", "pres", "temp"):
        assert np.array_equal(a.get(SPH, f), b.get(SPH, f)), f
