"""The oracle's two-dimensional ISPH-DEM model (dim 2, a bed in a plane
y = const; beds.box_bed_2d) on the CPU.

* The state stays in the plane over 100 steps: y, uy and the DEM spin
  components wx, wz exactly as set, the contact torques about y only,
  every field finite.
* Known answer for the 2-D porosity of the first step, from the initial
  positions: for every SPH particle,
    eps_i = 1 - sum_a W(r_ia) 3.14159 r_a^2 / (sum_{j fluid} (m_j / rho_j) W(r_ij) + 1e-20)
  with the 2-D Wendland C2 kernel, r = |x_i - x_j| + 1e-20 < kappa h (the
  disc-area form of the reference's KERNEL_clc_prep2D_coupling,
  functions_PREP2.cuh:2944-3033, with the Shepard denominator of the 3-D
  KERNEL_clc_prep3D_coupling_sph, :3190-3364).
"""
import numpy as np
from scipy.spatial import cKDTree

from fluidized_bed_master_b200.beds import box_bed_2d
from fluidized_bed_master_b200.params import DEM, SPH
from oracle import Oracle

Y0 = 0.0125


def _wendland2d(r, h):
    q = r / (2.0 * h)
    tA = 2.228169203286535 / (4.0 * h * h)
    return np.where(q < 1.0, tA * (1.0 - q) ** 4 * (1.0 + 4.0 * q), 0.0)


def test_bed2d_oracle_stays_in_plane():
    p, sph, dem = box_bed_2d(n_fluid=3000, seed=2, y0=Y0)
    o = Oracle(p, sph, dem, threads=4)
    o.step(100)
    for which in (SPH, DEM):
        assert np.all(o.get(which, "y") == Y0)
        assert np.all(o.get(which, "uy") == 0.0)
        for f in ("x", "z", "ux", "uz", "pres", "rho"):
            assert np.all(np.isfinite(o.get(which, f))), f
    assert np.all(o.get(DEM, "wx") == 0.0) and np.all(o.get(DEM, "wz") == 0.0)
    # contact torques turn about y only
    assert np.all(o.get(DEM, "torqx") == 0.0) and np.all(o.get(DEM, "torqz") == 0.0)
    assert np.any(o.get(DEM, "torqy") != 0.0), "no contact torque: the check above means nothing"


def test_bed2d_porosity_known_answer():
    p, sph, dem = box_bed_2d(n_fluid=3000, seed=4, y0=Y0)
    o = Oracle(p, sph, dem, threads=4)
    o.step(1)
    h = float(sph["h"][0])
    R = p.kappa * h
    xs = np.stack([sph["x"], sph["z"]], 1)
    xd = np.stack([dem["x"], dem["z"]], 1)
    vol = np.asarray(sph["m"]) / np.asarray(sph["rho"])
    fluid = np.asarray(sph["p_type"]) == 1
    ts, td = cKDTree(xs), cKDTree(xd)
    eps = np.empty(len(xs))
    for i in range(len(xs)):
        js = np.array(ts.query_ball_point(xs[i], R), dtype=int)
        r = np.linalg.norm(xs[js] - xs[i], axis=1) + 1e-20
        js, r = js[r < R], r[r < R]
        den = np.sum(vol[js] * _wendland2d(r, h) * fluid[js])
        ja = np.array(td.query_ball_point(xs[i], R), dtype=int)
        ra = np.linalg.norm(xd[ja] - xs[i], axis=1) + 1e-20 if len(ja) else np.zeros(0)
        keep = ra < R
        num = np.sum(_wendland2d(ra[keep], h) * 3.14159 * dem["rad"][ja[keep]] ** 2)
        eps[i] = 1.0 - num / (den + 1e-20)
    got = o.get(SPH, "DEMpor")
    want = eps[o.get(SPH, "pid")]
    m = o.get(SPH, "i_type") <= 2
    assert np.any(want[m] < 0.9), "no particle near a sphere: the check means nothing"
    np.testing.assert_allclose(got[m], want[m], rtol=1e-12, atol=1e-12)
