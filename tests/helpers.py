"""Comparison helpers shared by the parity tests."""
import glob
import json
import os

import numpy as np

from fluidized_bed_master_b200.params import DEM, SPH, SphdemParams

GOLDEN_DIR = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def rel_l2(a, b):
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    den = np.linalg.norm(b)
    num = np.linalg.norm(a - b)
    if den == 0.0:
        return num
    return num / den


def by_id(ids, arr):
    """Reorder arr so that entry k belongs to identity k (ids = 0..n-1 or dem ids)."""
    ids = np.asarray(ids).astype(np.int64)
    out = np.empty_like(np.asarray(arr))
    out[ids - ids.min()] = arr
    return out


def golden_files():
    return sorted(glob.glob(os.path.join(GOLDEN_DIR, "*.npz")))


def load_golden(path):
    g = np.load(path)
    p = SphdemParams.from_dict(json.loads(g["params_json"].tobytes().decode()))
    sph = {k[len("in_sph_"):]: g[k] for k in g.files if k.startswith("in_sph_")}
    dem = {k[len("in_dem_"):]: g[k] for k in g.files if k.startswith("in_dem_")}
    for d in (sph, dem):
        for f in ("p_type", "dem_idx"):
            if f in d:
                d[f] = d[f].astype(np.int32)
    return g, p, sph, dem


def history_map(ct, ds):
    """Per particle: dict partner id -> spring vector, from (n,16) ids and (n,16,3) springs."""
    out = []
    for i in range(ct.shape[0]):
        m = {}
        for s in range(ct.shape[1]):
            if ct[i, s] >= 1:
                m[int(round(ct[i, s]))] = ds[i, s]
        out.append(m)
    return out
