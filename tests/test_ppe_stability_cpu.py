"""Why the converged pressure blows up on the water box beds (FP64 oracle, CPU).

With the PPE solved to a relative residual of 1e-6 (PCG) the box beds grow
without bound after ~100-250 steps, while the reference's single Jacobi
sweep stays bounded.  The oracle -- the FP64 CPU restatement, independent
of the CUDA engine -- does the same, so it is the formulation, not the
engine.  The mechanism is the added-mass instability of an explicit
(staggered) fluid-particle pressure coupling: the sphere velocities of the
previous step set the porosity rate in the PPE source
rho_f (div(eps u*) + 2 d_eps - d_eps_prev) / dt (functions_PPE2.cuh:542-698),
the converged pressure pushes the spheres through the pressure-gradient
force (functions_SPH_DEM_COUPLING2.cuh:886-888), and their new velocities
feed the next source.  The loop gain scales with the fluid/solid density
ratio: water on 2500 kg/m^3 glass (0.4) diverges; the same bed with
spheres ten times denser (0.04) stays calm, as does the reference's air
bed (7e-4), whose PPE hard-wires the air density.  One damped sweep per step
keeps the gain below one.

Bar: on the reduced bench-configuration box bed, max |u| of the fluid after
150 PCG steps exceeds 10 m/s (or is not finite) at the real density ratio,
and stays below 1 m/s with the spheres ten times denser.
"""
import numpy as np

from fluidized_bed_master_b200.beds import box_bed
from fluidized_bed_master_b200.params import SPH
from oracle import Oracle


def _umax_after(steps, sphere_density_scale):
    p, sph, dem = box_bed(n_fluid=20_000, n_dem=2_000, lx=0.05, dem_height=0.02, seed=41)
    p.ppe_mode = 2          # PCG to a tolerance
    p.kgc_solve = 0
    p.ppe_tol = 1e-6
    p.ppe_max_iter = 3000
    dem = dict(dem)
    for f in ("m", "rho", "ri"):
        dem[f] = dem[f] * sphere_density_scale
    orc = Oracle(p, sph, dem, threads=8)
    orc.step(steps)
    u = np.stack([orc.get(SPH, f) for f in ("ux", "uy", "uz")])
    return float(np.abs(u).max()) if np.isfinite(u).all() else float("inf")


def test_converged_pressure_added_mass_instability():
    heavy = _umax_after(150, 10.0)
    assert heavy < 1.0, f"denser spheres should keep the converged-PPE bed calm (max |u| {heavy:.3g} m/s)"
    real = _umax_after(150, 1.0)
    assert real > 10.0, f"the water/glass bed was expected to diverge by step 150 (max |u| {real:.3g} m/s)"
