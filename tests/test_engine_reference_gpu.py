"""The CUDA engine held directly to the reference's own ISPH-DEM run.

tests/golden/contact.npz and heat.npz hold the state of two seeded spouted
beds after 1, 8 and 100 steps of the unmodified reference step function
SOPHIA_single_ISPH (ISPH_Calc_seperate.cuh:13-503), run by
tests/golden/make_golden.py through oracle/_ref.  The engine replays the
same inputs through the C ABI.

Bar (written into each assert):
* sorted order (cell-sorted particle identities) and p_type / i_type /
  buffer_type identical to the reference's at every checkpoint; DEM
  contact partners identical;
* FP64 build: every real field within rel. L2 1e-9 at every checkpoint;
* FP32 build: every real field within rel. L2 1e-5 at the last checkpoint
  (100 steps).
"""
import json

import numpy as np
import pytest

from fluidized_bed_master_b200.params import DEM, SPH
from tests.helpers import by_id, golden_files, history_map, load_golden, rel_l2

pytestmark = pytest.mark.gpu

REAL_SPH = ["x", "y", "z", "ux", "uy", "uz", "m", "rho", "pres", "temp", "DEMpor", "dDEMpor", "flt_s",
            "pgfx", "pgfy", "pgfz", "rho_ref", "ftotalx", "ftotaly", "ftotalz", "fpx", "fpy", "fpz"]
REAL_DEM = ["x", "y", "z", "ux", "uy", "uz", "wx", "wy", "wz", "temp", "DEMpor", "flt_s", "flt_sd", "flt_sd2",
            "Fdx_df", "Fdy_df", "Fdz_df", "ftotalx", "ftotaly", "ftotalz", "torqx", "torqy", "torqz", "dtemp"]

ISPH_GOLD = [p for p in golden_files() if json.loads(np.load(p)["meta"].tobytes()).get("solver", "isph") == "isph"]


def _engine(p, sph, dem, prec):
    from fluidized_bed_master_b200.engine import Engine

    q = p.copy()
    q.precision = prec
    return Engine(q, sph, dem)


def _run_against_fixture(path, prec, tol, last_only):
    g, p, sph, dem = load_golden(path)
    eng = _engine(p, sph, dem, prec)
    done = 0
    bad = []
    cps = [int(c) for c in g["checkpoints"]]
    for cp in cps:
        eng.step(cp - done)
        done = cp
        pre = f"s{cp}_"
        ref_pid = g[pre + "sph_pid"].astype(np.int64)
        epid = eng.get(SPH, "pid")
        assert np.array_equal(ref_pid, epid), f"cell-sorted SPH order differs from the reference at step {cp}"
        for f in ("p_type", "i_type", "buffer_type"):
            assert np.array_equal(g[pre + "sph_" + f].astype(np.int64), eng.get(SPH, f)), (cp, f)
        ref_id = g[pre + "dem_dem_idx"].astype(np.int64)
        eid = eng.get(DEM, "dem_idx")
        assert np.array_equal(ref_id, eid), f"cell-sorted DEM order differs from the reference at step {cp}"
        ct = np.stack([g[f"{pre}dem_ct_idx{s}"] for s in range(16)], 1)
        ds = np.stack([np.stack([g[f"{pre}dem_del_s{s}_{c}"] for c in range(3)], 1) for s in range(16)], 1)
        href = {int(ref_id[i]): m for i, m in enumerate(history_map(ct, ds))}
        ids, springs = eng.history()
        heng = {int(eid[i]): m for i, m in enumerate(history_map(np.asarray(ids, dtype=float), springs))}
        for k, v in href.items():
            assert set(v) == set(heng[k]), f"contact partners of sphere {k} differ at step {cp}"
        if last_only and cp != cps[-1]:
            continue
        for f in REAL_SPH + (["vis_t"] if pre + "sph_vis_t" in g.files else []):
            e = rel_l2(by_id(epid, eng.get(SPH, f)), by_id(ref_pid, g[pre + "sph_" + f]))
            if not e <= tol:
                bad.append((cp, "sph", f, e))
        for f in REAL_DEM:
            e = rel_l2(by_id(eid, eng.get(DEM, f)), by_id(ref_id, g[pre + "dem_" + f]))
            if not e <= tol:
                bad.append((cp, "dem", f, e))
    assert cps[-1] >= 100, "fixture has no 100-step checkpoint: regenerate with tests/golden/make_golden.py"
    return bad


@pytest.mark.parametrize("path", ISPH_GOLD, ids=[p.split("/")[-1] for p in ISPH_GOLD])
def test_fp64_engine_matches_reference_run(path):
    """FP64 build vs the reference's own run: rel. L2 <= 1e-9 per field at 1, 8 and 100 steps."""
    bad = _run_against_fixture(path, 1, 1e-9, last_only=False)
    assert not bad, bad


@pytest.mark.parametrize("path", ISPH_GOLD, ids=[p.split("/")[-1] for p in ISPH_GOLD])
def test_fp32_engine_matches_reference_run_after_100_steps(path):
    """FP32 build vs the reference's own FP64 run: rel. L2 <= 1e-5 per field after 100 steps."""
    bad = _run_against_fixture(path, 0, 1e-5, last_only=True)
    assert not bad, bad
