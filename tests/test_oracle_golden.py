"""The oracle pinned against the reference itself.

tests/golden/*.npz were produced by tests/golden/make_golden.py: the
unmodified reference kernels (oracle/_ref, compiled from the reference
sources) advanced seeded spouted beds (ISPH-DEM) and 2-D dam breaks
(WCSPH) on a B200 and their state was read back.  Here the CPU oracle replays the same inputs and must agree:
integer fields exactly, contact-history partners exactly, real fields to
rel. L2 <= 1e-9 (FP64 on both sides; only rounding, FMA contraction in
the reference build and summation order differ).
"""
import json

import numpy as np
import pytest

from fluidized_bed_master_b200.params import DEM, SPH
from oracle import Oracle
from tests.helpers import by_id, golden_files, history_map, load_golden, rel_l2

GOLD = golden_files()
TOL = 1e-9

REAL_SPH = ["x", "y", "z", "ux", "uy", "uz", "m", "rho", "pres", "temp", "DEMpor", "dDEMpor", "flt_s",
            "pgfx", "pgfy", "pgfz", "rho_ref", "ftotalx", "ftotaly", "ftotalz", "fpx", "fpy", "fpz"]
REAL_DEM = ["x", "y", "z", "ux", "uy", "uz", "wx", "wy", "wz", "temp", "DEMpor", "flt_s", "flt_sd", "flt_sd2",
            "Fdx_df", "Fdy_df", "Fdz_df", "ftotalx", "ftotaly", "ftotalz", "torqx", "torqy", "torqz", "dtemp"]


def test_fixtures_present():
    assert GOLD, "tests/golden/*.npz missing: run tests/golden/make_golden.py on a GPU machine"


REAL_W = ["x", "y", "ux", "uy", "m", "rho", "pres", "flt_s", "pgfx", "pgfy", "rho_ref", "ftotalx", "ftotaly",
          "ftotal", "drho", "grad_rhox", "grad_rhoy"]


def _meta(path):
    return json.loads(np.load(path)["meta"].tobytes())


ISPH_GOLD = [p for p in GOLD if _meta(p).get("solver", "isph") == "isph"]
WCSPH_GOLD = [p for p in GOLD if _meta(p).get("solver") == "wcsph"]


def test_wcsph_fixtures_present():
    assert WCSPH_GOLD, "tests/golden/dam2d*.npz missing: run tests/golden/make_golden.py on a GPU machine"


@pytest.mark.parametrize("path", WCSPH_GOLD, ids=[p.split("/")[-1] for p in WCSPH_GOLD])
def test_oracle_matches_reference_wcsph2d(path):
    """2-D WCSPH dam breaks: cell-sorted order and types exact, real fields
    rel. L2 <= 1e-9 at every checkpoint (up to 1000 steps)."""
    g, p, sph, dem = load_golden(path)
    meta = json.loads(g["meta"].tobytes())
    orc = Oracle(p, sph, dem, threads=4)
    nijk, _, _ = orc.grid()
    assert list(nijk) == list(g["nijk"]), "cell grid differs from the reference's NI, NJ, NK"
    done = 0
    bad = []
    for cp in g["checkpoints"]:
        orc.step(int(cp) - done)
        done = int(cp)
        pre = f"s{cp}_sph_"
        ref_pid = g[pre + "pid"].astype(np.int64)
        opid = orc.get(SPH, "pid")
        assert np.array_equal(np.sort(ref_pid), np.arange(meta["ns"]))
        assert np.array_equal(ref_pid, opid), f"cell-sorted order differs from the reference at step {cp}"
        for f in ("p_type", "i_type", "buffer_type"):
            assert np.array_equal(g[pre + f].astype(np.int64), orc.get(SPH, f)), f
        for f in REAL_W:
            e = rel_l2(orc.get(SPH, f), g[pre + f])
            if not e <= TOL:
                bad.append((int(cp), f, e))
    moved = np.abs(by_id(ref_pid, g[f"s{done}_sph_y"]) - g["in_sph_y"]).max()
    assert moved > 0, "nothing moved: the comparison would be vacuous"
    assert not bad, bad


@pytest.mark.parametrize("path", ISPH_GOLD, ids=[p.split("/")[-1] for p in ISPH_GOLD])
def test_oracle_matches_reference(path):
    g, p, sph, dem = load_golden(path)
    meta = json.loads(g["meta"].tobytes())
    orc = Oracle(p, sph, dem, threads=4)
    nijk, _, _ = orc.grid()
    assert list(nijk) == list(g["nijk"]), "cell grid differs from the reference's NI, NJ, NK"
    done = 0
    bad = []
    for cp in g["checkpoints"]:
        orc.step(int(cp) - done)
        done = int(cp)
        pre = f"s{cp}_"
        # SPH: identity = input row (reference keeps it in part1::concn)
        ref_pid = g[pre + "sph_pid"].astype(np.int64)
        opid = orc.get(SPH, "pid")
        assert np.array_equal(np.sort(ref_pid), np.arange(meta["ns"]))
        assert np.array_equal(ref_pid, opid), "cell-sorted order differs from the reference"
        for f in ("p_type", "i_type", "buffer_type"):
            assert np.array_equal(g[pre + "sph_" + f].astype(np.int64), orc.get(SPH, f)), f
        for f in REAL_SPH + (["vis_t"] if pre + "sph_vis_t" in g.files else []):
            e = rel_l2(by_id(opid, orc.get(SPH, f)), by_id(ref_pid, g[pre + "sph_" + f]))
            if not e <= TOL:
                bad.append((int(cp), "sph", f, e))
        ref_id = g[pre + "dem_dem_idx"].astype(np.int64)
        oid = orc.get(DEM, "dem_idx")
        for f in REAL_DEM:
            e = rel_l2(by_id(oid, orc.get(DEM, f)), by_id(ref_id, g[pre + "dem_" + f]))
            if not e <= TOL:
                bad.append((int(cp), "dem", f, e))
        # contact history: same partners in every sphere, springs close
        nd = len(ref_id)
        ct = np.stack([g[f"{pre}dem_ct_idx{s}"] for s in range(16)], 1)
        ds = np.stack([np.stack([g[f"{pre}dem_del_s{s}_{c}"] for c in range(3)], 1) for s in range(16)], 1)
        href = {int(ref_id[i]): m for i, m in enumerate(history_map(ct, ds))}
        oct_, ods = orc.history()
        hor = {int(oid[i]): m for i, m in enumerate(history_map(oct_, ods))}
        for k in href:
            assert set(href[k]) == set(hor[k]), f"partners of sphere {k} at step {cp}"
            for j in href[k]:
                # each spring vector to 1e-8 of its own magnitude (a component
                # near zero carries the vector's rounding, not its own)
                a, b = np.asarray(hor[k][j]), np.asarray(href[k][j])
                assert np.abs(a - b).max() <= 1e-8 * np.abs(b).max() + 1e-20, (cp, k, j, a, b)
        assert sum(len(v) for v in href.values()) > 0
    assert not bad, bad
