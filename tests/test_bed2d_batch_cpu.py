"""The oracle on several 2-D beds in their own planes (oracle_set_beds,
beds.bed2d_batch): every bed of the batch equals the same bed run alone on
the batch's cell grid, bit for bit, after 10 steps -- the beds never
interact and each keeps its own inlet velocity and outlet slab.  The batch
generator itself: planes more than two cells apart, inlet velocities in
[0.1, 0.3], sphere counts a tenth of the fluid counts, sphere ids unique.
"""
import numpy as np

from fluidized_bed_master_b200.beds import bed2d_batch
from fluidized_bed_master_b200.params import DEM, SPH
from oracle import Oracle


def _domain(sph, dem):
    x = np.concatenate([sph["x"], dem["x"]])
    y = np.concatenate([sph["y"], dem["y"]])
    z = np.concatenate([sph["z"], dem["z"]])
    # the reference's find_minmax stops one row short (function_init.cuh:913-950)
    x, y, z = x[:-1], y[:-1], z[:-1]
    return [x.min(), x.max(), y.min(), y.max(), z.min(), z.max()], float(sph["h"][0])


def test_bed2d_batch_generator():
    p, sph, dem, rows, parts = bed2d_batch(n_beds=6, n_min=1500, n_max=5000, seed=2)
    ys = np.array([r["y"] for r in rows])
    dcell = 1.1 * p.kappa * float(sph["h"][0])
    assert np.all(np.diff(ys) > 2.0 * dcell)
    u = np.array([r["inlet_uz"] for r in rows])
    assert np.all((u >= 0.1) & (u <= 0.3)) and len(set(u)) == len(u)
    for s, d, _ in parts:
        nf = int(np.sum((s["p_type"] == 1) & (s["z"] >= 0)))
        assert len(d["x"]) == nf // 10
    assert len(np.unique(dem["dem_idx"])) == len(dem["dem_idx"])


def test_bed2d_batch_beds_equal_beds_alone():
    p, sph, dem, rows, parts = bed2d_batch(n_beds=4, n_min=1500, n_max=5000, seed=1)
    bb, h0 = _domain(sph, dem)
    ob = Oracle(p, sph, dem, threads=4, beds=rows)
    ob.step(10)
    pid_s, pid_d = ob.get(SPH, "pid"), ob.get(DEM, "pid")
    s0 = d0 = 0
    for b, (sb, db, rb) in enumerate(parts):
        oa = Oracle(p, sb, db, threads=4, beds=rb, domain=(bb, h0))
        oa.step(10)
        for which, lo, src, pid in ((SPH, s0, sb, pid_s), (DEM, d0, db, pid_d)):
            n = len(src["x"])
            m = (pid >= lo) & (pid < lo + n)
            for f in ("x", "z", "ux", "uz", "pres", "rho", "temp", "DEMpor"):
                a = np.empty(n)
                a[pid[m] - lo] = ob.get(which, f)[m]
                c = np.empty(n)
                c[oa.get(which, "pid")] = oa.get(which, f)
                assert np.array_equal(a, c), (b, which, f)
        s0 += len(sb["x"])
        d0 += len(db["x"])
