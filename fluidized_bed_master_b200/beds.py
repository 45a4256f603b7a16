"""Seeded synthetic beds written in the reference's input formats.

The reference's own scenario (input/input.txt) is not shipped, so every
run uses one of these generators.  Two families:

* ``spouted_bed`` -- the geometry the reference hard-wires: a 12.5 mm
  cylinder over a truncated cone (functions_DEM_BC.cuh:254-257, 4237-4243),
  an inlet pipe below z = L2 and an outlet slab above z = L3
  (functions_NNPS.cuh:2-5), gas (argon) properties, dx = h/1.6.  Runs with
  the reference-compat preset and is the case the reference kernels can
  run unmodified.
* ``box_bed`` -- the 3-D fluidized bed of the benchmark: a 0.1 x 0.02 x
  0.4 m box, water-like fluid on a dx = 1.25 mm lattice (first N sites in
  z-major order), Wendland C2 with h = 1.3 dx, DEM spheres of 2 mm +/-5 %
  at density 2500 on random FCC sites in the lower 0.1 m, inlet at the
  bottom, heat transfer on.
* ``isph_column`` -- a 3-D water column with no DEM in a wall box: the
  plain ISPH projection with the PPE solved to 1e-6.
* ``box_bed_2d`` / ``bed2d_batch`` -- the box bed in two dimensions (a bed
  in a plane y = const), and many such beds of uneven size, each in its own
  plane with its own inlet velocity, for one handle.

Lattice positions get seeded uniform jitter of +/-0.01 dx so that no pair
sits exactly on a kernel-support boundary.
"""
import os

import numpy as np

from .params import reference_params

INPUT_LABELS = [1, 2, 3, 4, 5, 6, 7, 8, 9, 10, 11, 12, 26, 27, 28, 29, 30, 31, 32, 33, 34, 35]
_LABEL_FIELD = {1: "x", 2: "y", 3: "z", 4: "ux", 5: "uy", 6: "uz", 7: "m", 8: "p_type", 9: "h", 10: "temp",
                11: "pres", 12: "rho", 26: "flt_s", 27: "rad", 28: "ri", 29: "dem_idx", 30: "wx", 31: "wy",
                32: "wz", 33: "temp1", 34: "temp2", 35: "temp3"}


def _fcc_sites(lo, hi, spacing):
    a = spacing * np.sqrt(2.0)
    base = np.array([[0, 0, 0], [0.5, 0.5, 0], [0.5, 0, 0.5], [0, 0.5, 0.5]]) * a
    n = np.floor((np.asarray(hi) - np.asarray(lo)) / a).astype(int) + 1
    g = np.stack(np.meshgrid(np.arange(n[0]), np.arange(n[1]), np.arange(n[2]), indexing="ij"), -1).reshape(-1, 3) * a
    pts = (g[:, None, :] + base[None, :, :]).reshape(-1, 3) + np.asarray(lo)
    keep = np.all((pts >= lo) & (pts <= hi), axis=1)
    return pts[keep]


def _dem_arrays(pos, rad, rho_s, h, temp, first_id=1):
    nd = len(pos)
    m = rho_s * 4.0 / 3.0 * np.pi * rad ** 3
    return dict(
        x=pos[:, 0].copy(), y=pos[:, 1].copy(), z=pos[:, 2].copy(),
        ux=np.zeros(nd), uy=np.zeros(nd), uz=np.zeros(nd),
        wx=np.zeros(nd), wy=np.zeros(nd), wz=np.zeros(nd),
        m=m, rho=np.full(nd, rho_s), rad=rad, ri=0.4 * m * rad ** 2,
        h=np.full(nd, h), temp=np.full(nd, temp), temp1=np.full(nd, temp), temp2=np.full(nd, temp),
        temp3=np.full(nd, temp), pres=np.zeros(nd), flt_s=np.zeros(nd),
        p_type=np.full(nd, 1001, dtype=np.int32), dem_idx=np.arange(first_id, first_id + nd, dtype=np.int32),
    )


def spouted_bed(dx=0.5e-3, n_dem=4580, r_dem=0.5e-3, seed=0, t_gas=823.0, t_dem=300.0, dem_top=-0.002,
                spacing=2.1, u_dem=0.0):
    """Reference-compat spouted bed.  Returns (params, sph, dem).

    DEM spheres sit on random sites of an FCC lattice whose nearest spacing
    is ``spacing`` x the largest radius (below 2 the neighbours start in
    contact); ``u_dem`` is the amplitude of a seeded uniform initial
    velocity of the spheres."""
    rng = np.random.default_rng(seed)
    p = reference_params()
    h = 1.6 * dx
    R_cyl, r2, h_cone = p.cyl_r, p.cone_r2, p.cone_h
    wall = 3 * dx
    xs = np.arange(-(R_cyl + wall), R_cyl + wall + 1e-12, dx)
    zs = np.arange(-0.02275, 0.01375 + 1e-12, dx)
    X, Y, Z = np.meshgrid(xs, xs, zs, indexing="ij")
    X, Y, Z = X.ravel(), Y.ravel(), Z.ravel()
    r = np.hypot(X, Y)
    # radius of the fluid region at height z: pipe, cone, cylinder
    rz = np.where(Z >= 0.0, R_cyl, np.where(Z >= -h_cone, r2 + (Z + h_cone) * (R_cyl - r2) / h_cone, r2))
    fluid = r < rz
    solid = (~fluid) & (r < rz + wall)
    keep = fluid | solid
    X, Y, Z, fl = X[keep], Y[keep], Z[keep], fluid[keep]
    n = len(X)
    jit = rng.uniform(-0.01 * dx, 0.01 * dx, size=(n, 3))
    X, Y, Z = X + jit[:, 0], Y + jit[:, 1], Z + jit[:, 2]
    ptype = np.where(fl, 1, 0).astype(np.int32)
    vol = (h / p.h_over_dx) ** 3
    sph = dict(x=X, y=Y, z=Z, ux=np.zeros(n), uy=np.zeros(n), uz=np.zeros(n),
               m=np.full(n, p.rho_gas * vol), rho=np.full(n, p.rho_gas), pres=np.zeros(n),
               temp=np.full(n, t_gas), h=np.full(n, h), flt_s=np.ones(n), p_type=ptype,
               rad=np.zeros(n), ri=np.zeros(n))
    # DEM spheres on random FCC sites inside the cone/cylinder, below dem_top
    rmax = 1.05 * r_dem
    sites = _fcc_sites([-R_cyl, -R_cyl, -h_cone], [R_cyl, R_cyl, dem_top], spacing * rmax)
    sr = np.hypot(sites[:, 0], sites[:, 1])
    zz = sites[:, 2]
    rz_s = np.where(zz >= 0.0, R_cyl, r2 + (zz + h_cone) * (R_cyl - r2) / h_cone)
    # clearance from the cone wall measured along the wall normal
    cosang = h_cone / np.hypot(R_cyl - r2, h_cone)
    ok = (sr + 1.3 * rmax / cosang < rz_s) & (zz > -h_cone + 1.3 * rmax)
    sites = sites[ok]
    if len(sites) < n_dem:
        n_dem = len(sites)
    pick = rng.choice(len(sites), size=n_dem, replace=False)
    pos = sites[np.sort(pick)]
    rad = r_dem * rng.uniform(0.95, 1.05, size=n_dem)
    dem = _dem_arrays(pos, rad, 2500.0, h, t_dem)
    if u_dem > 0:
        for f in ("ux", "uy", "uz"):
            dem[f] = rng.uniform(-u_dem, u_dem, size=n_dem)
    return p, sph, dem


def box_bed(n_fluid=200_000, n_dem=20_000, dx=1.25e-3, seed=0, u_in=0.15, t_fluid=300.0, t_dem=350.0,
            lx=0.1, ly=0.02, lz=0.4, dem_height=0.1, d_dem=2.0e-3):
    """Benchmark bed (0.1 x 0.02 x 0.4 m).  Returns (params, sph, dem)."""
    rng = np.random.default_rng(seed)
    p = reference_params()
    h = 1.3 * dx
    p.kernel_type = 3            # Wendland C2
    p.h_over_dx = 1.3
    p.rho_gas = 1000.0           # the p_type 1 fluid: water-like
    p.mu_gas = 1.0e-3
    p.nu_gas = 1.0e-6
    p.dem_shear_modulus = 1.0e7 / (2.0 * 1.3)   # E = 1e7, nu = 0.3
    p.dem_poisson = 0.3
    p.dem_friction_ratio = 0.3
    p.g_sph = 9.81
    p.g_dem = 9.81
    p.con_solve = 1
    p.dt = 1.0e-5
    p.inlet_uz_mirror = u_in
    p.inlet_temp = t_fluid
    p.dem_wall_mask = 2          # box walls only
    nx, ny = int(round(lx / dx)), int(round(ly / dx))
    per_layer = nx * ny
    nz_full = n_fluid // per_layer + (1 if n_fluid % per_layer else 0)
    ii, jj = np.meshgrid(np.arange(nx), np.arange(ny), indexing="ij")
    ii, jj = ii.T.ravel(), jj.T.ravel()        # x fastest, then y
    layers = []
    for k in range(-3, nz_full):               # three inlet layers below z = 0
        z = (k + 0.5) * dx
        layers.append(np.stack([(ii + 0.5) * dx, (jj + 0.5) * dx, np.full(per_layer, z)], 1))
    lat = np.concatenate(layers)
    inlet = lat[: 3 * per_layer]
    fluid = lat[3 * per_layer: 3 * per_layer + n_fluid]
    ztop = fluid[:, 2].max() + 0.5 * dx
    # three wall layers around the sides, from the inlet bottom to the fluid top
    wx = np.arange(-3, nx + 3)
    wy = np.arange(-3, ny + 3)
    wz = np.arange(-3, int(np.ceil(ztop / dx)))
    WI, WJ, WK = np.meshgrid(wx, wy, wz, indexing="ij")
    side = (WI < 0) | (WI >= nx) | (WJ < 0) | (WJ >= ny)
    walls = np.stack([(WI[side] + 0.5) * dx, (WJ[side] + 0.5) * dx, (WK[side] + 0.5) * dx], 1)
    pos = np.concatenate([fluid, inlet, walls])
    ptype = np.concatenate([np.ones(len(fluid) + len(inlet), np.int32), np.zeros(len(walls), np.int32)])
    n = len(pos)
    pos = pos + rng.uniform(-0.01 * dx, 0.01 * dx, size=(n, 3))
    vol = (h / p.h_over_dx) ** 3
    uz = np.where(pos[:, 2] < 0, u_in, 0.0) * (ptype == 1)
    sph = dict(x=pos[:, 0], y=pos[:, 1], z=pos[:, 2], ux=np.zeros(n), uy=np.zeros(n), uz=uz,
               m=np.full(n, p.rho_gas * vol), rho=np.full(n, p.rho_gas), pres=np.zeros(n),
               temp=np.full(n, t_fluid), h=np.full(n, h), flt_s=np.ones(n), p_type=ptype,
               rad=np.zeros(n), ri=np.zeros(n))
    # open-boundary slabs: inlet below z = 0, outlet in the top three fluid layers
    p.obc_L1 = -1.0
    p.obc_L2 = 0.0
    p.obc_L3 = ztop - 3 * dx
    p.obc_L4 = ztop + 1.0
    # DEM on random FCC sites with nearest spacing 2.1 mm in the lower dem_height
    rmax = 0.5 * d_dem * 1.05
    sites = _fcc_sites([rmax * 1.2, rmax * 1.2, rmax * 1.2],
                       [lx - rmax * 1.2, ly - rmax * 1.2, dem_height - rmax], 2.1e-3 * max(1.0, d_dem / 2.0e-3))
    if len(sites) < n_dem:
        n_dem = len(sites)
    pick = rng.choice(len(sites), size=n_dem, replace=False)
    dpos = sites[np.sort(pick)]
    rad = 0.5 * d_dem * rng.uniform(0.95, 1.05, size=n_dem)
    dem = _dem_arrays(dpos, rad, 2500.0, h, t_dem)
    p.box_c[:] = [0.5 * lx, 0.5 * ly, 0.5 * lz]
    p.box_L[:] = [lx, ly, lz]
    return p, sph, dem


def box_bed_2d(n_fluid=25_600, n_dem=None, dx=1.25e-3, seed=0, u_in=0.15, t_fluid=300.0, t_dem=350.0,
               lx=0.1, d_dem=2.0e-3, y0=0.0):
    """The benchmark bed in two dimensions: a bed of width lx in the x-z
    plane y = y0 (the engine's dim-2 ISPH-DEM model), with the materials,
    kernel, inlet and walls of box_bed.  n_fluid particles fill rows of
    lx / dx columns from z = 0 up (the height follows from the count);
    three inlet rows below z = 0 enter at u_in; three wall columns on each
    side reach from the inlet bottom to the fluid top; the outlet slab is
    the top three fluid rows.  n_dem spheres (default 10 % of n_fluid),
    diameter d_dem +- 5 %, density 2500, centres on randomly chosen sites of
    a hexagonal lattice of spacing 2.1 mm that covers the bed below the
    outlet slab, so no two overlap.  At 10 % of the fluid count the discs
    cover about a fifth of the bed's area (the 3-D bed's spheres about 40 %
    of its lower volume): in two dimensions a sphere of d = 2 mm holds about
    two thirds of a kernel's area at h = 1.625 mm, and a denser packing
    drives the porosity-rate source of the pressure equation past what the
    reference's one-sweep pressure step holds.  Returns (params, sph, dem)."""
    rng = np.random.default_rng(seed)
    p, _, _ = box_bed(n_fluid=1000, n_dem=1, dx=dx, seed=seed, u_in=u_in, t_fluid=t_fluid, t_dem=t_dem)
    p.dim = 2
    h = 1.3 * dx
    nx = int(round(lx / dx))
    nz = n_fluid // nx + (1 if n_fluid % nx else 0)
    I, K = np.meshgrid(np.arange(nx), np.arange(-3, nz), indexing="xy")
    I, K = I.ravel(), K.ravel()                  # x fastest, then z
    lat = np.stack([(I + 0.5) * dx, (K + 0.5) * dx], 1)
    inlet = lat[: 3 * nx]
    fluid = lat[3 * nx: 3 * nx + n_fluid]
    ztop = fluid[:, 1].max() + 0.5 * dx
    WI, WK = np.meshgrid(np.r_[np.arange(-3, 0), np.arange(nx, nx + 3)], np.arange(-3, int(np.ceil(ztop / dx))),
                         indexing="xy")
    walls = np.stack([(WI.ravel() + 0.5) * dx, (WK.ravel() + 0.5) * dx], 1)
    pos = np.concatenate([fluid, inlet, walls])
    ptype = np.concatenate([np.ones(len(fluid) + len(inlet), np.int32), np.zeros(len(walls), np.int32)])
    n = len(pos)
    pos = pos + rng.uniform(-0.01 * dx, 0.01 * dx, size=(n, 2))
    vol = (h / p.h_over_dx) ** 2
    uz = np.where(pos[:, 1] < 0, u_in, 0.0) * (ptype == 1)
    sph = dict(x=pos[:, 0], y=np.full(n, float(y0)), z=pos[:, 1], ux=np.zeros(n), uy=np.zeros(n), uz=uz,
               m=np.full(n, p.rho_gas * vol), rho=np.full(n, p.rho_gas), pres=np.zeros(n),
               temp=np.full(n, t_fluid), h=np.full(n, h), flt_s=np.ones(n), p_type=ptype,
               rad=np.zeros(n), ri=np.zeros(n))
    p.obc_L1 = -1.0
    p.obc_L2 = 0.0
    p.obc_L3 = ztop - 3 * dx
    p.obc_L4 = ztop + 1.0
    if n_dem is None:
        n_dem = n_fluid // 10
    rmax = 0.5 * d_dem * 1.05
    s = 2.1e-3 * max(1.0, d_dem / 2.0e-3)
    x0, x1 = rmax * 1.2, lx - rmax * 1.2
    per_row = int(np.floor((x1 - x0) / s)) + 1
    rows = int(np.floor((ztop - 4 * dx - rmax - rmax * 1.2) / (s * np.sqrt(3.0) / 2.0))) + 1
    RI, RK = np.meshgrid(np.arange(per_row), np.arange(max(rows, 0)), indexing="xy")
    sx = x0 + RI.ravel() * s + 0.5 * s * (RK.ravel() % 2)
    sz = rmax * 1.2 + RK.ravel() * s * np.sqrt(3.0) / 2.0
    keep = (sx <= x1) & (sz <= ztop - 4 * dx - rmax)
    sites = np.stack([sx[keep], sz[keep]], 1)
    n_dem = min(n_dem, len(sites))
    pick = np.sort(rng.choice(len(sites), size=n_dem, replace=False))
    dpos = np.stack([sites[pick, 0], np.full(n_dem, float(y0)), sites[pick, 1]], 1)
    rad = 0.5 * d_dem * rng.uniform(0.95, 1.05, size=n_dem)
    dem = _dem_arrays(dpos, rad, 2500.0, h, t_dem)
    # DEM box walls in x and z only: the y extent never binds
    p.box_c[:] = [0.5 * lx, float(y0), 0.5 * (ztop + 1.0)]
    p.box_L[:] = [lx, 1.0, ztop + 1.0]
    return p, sph, dem


def isph_column(dx=4.0e-3, lx=0.2, ly=0.2, hz=0.4, seed=0, u_slosh=0.05, g=9.81, dt=1.0e-4):
    """3-D ISPH column without DEM: a 0.2 x 0.2 x 0.4 m water-like column on
    a dx lattice (50 x 50 x 100 = 250,000 fluid at dx = 4 mm) in a closed
    box of three wall layers, Wendland C2 with h = 1.3 dx.  The box is
    closed because the reference's ISPH has no free-surface condition (its
    p = 0 line for surface particles is commented out,
    functions_PPE2.cuh:533-534), so a PPE solved to a tolerance has no
    pressure datum at an open top.  Initial state: hydrostatic pressure
    rho g (hz - z) and one sloshing roll in the x-z plane,
    psi = A sin(pi x / lx) sin(pi z / hz), scaled so that the largest speed
    is u_slosh; it is divergence-free with no normal velocity at any wall.
    The PPE solves to a relative residual with the Jacobi-preconditioned CG
    (ppe_mode PCG, 1e-6).  Returns (params, sph, dem) with an empty DEM
    set."""
    from .params import PPE_PCG

    rng = np.random.default_rng(seed)
    p = reference_params()
    h = 1.3 * dx
    p.kernel_type = 3
    p.h_over_dx = 1.3
    p.rho_gas = 1000.0           # the p_type 1 fluid: water-like
    p.mu_gas = 1.0e-3
    p.nu_gas = 1.0e-6
    p.g_sph = g
    p.con_solve = 0
    p.open_boundary = 0
    p.xsph_solve = 0
    p.dt = dt
    p.ppe_mode = PPE_PCG
    p.kgc_solve = 0              # the CG needs the uncorrected (M-symmetric) operator
    p.ppe_tol = 1.0e-6
    p.ppe_max_iter = 2000
    p.dem_wall_mask = 0
    nx, ny, nz = int(round(lx / dx)), int(round(ly / dx)), int(round(hz / dx))
    I, J, K = np.meshgrid(np.arange(nx), np.arange(ny), np.arange(nz), indexing="ij")
    fluid = np.stack([(I.T.ravel() + 0.5) * dx, (J.T.ravel() + 0.5) * dx, (K.T.ravel() + 0.5) * dx], 1)
    wx, wy, wz = np.arange(-3, nx + 3), np.arange(-3, ny + 3), np.arange(-3, nz + 3)
    WI, WJ, WK = np.meshgrid(wx, wy, wz, indexing="ij")
    side = (WI < 0) | (WI >= nx) | (WJ < 0) | (WJ >= ny) | (WK < 0) | (WK >= nz)
    walls = np.stack([(WI[side] + 0.5) * dx, (WJ[side] + 0.5) * dx, (WK[side] + 0.5) * dx], 1)
    pos = np.concatenate([fluid, walls])
    ptype = np.concatenate([np.ones(len(fluid), np.int32), np.zeros(len(walls), np.int32)])
    n = len(pos)
    pos = pos + rng.uniform(-0.01 * dx, 0.01 * dx, size=(n, 3))
    kx, kz = np.pi / lx, np.pi / hz
    x, z = pos[:, 0], pos[:, 2]
    ux = kz * np.sin(kx * x) * np.cos(kz * z)
    uz = -kx * np.cos(kx * x) * np.sin(kz * z)
    fl = ptype == 1
    scale = u_slosh / max(np.sqrt(ux[fl] ** 2 + uz[fl] ** 2).max(), 1e-30)
    ux, uz = ux * scale * fl, uz * scale * fl
    vol = (h / p.h_over_dx) ** 3
    pres = p.rho_gas * g * np.clip(hz - pos[:, 2], 0.0, None)
    sph = dict(x=pos[:, 0], y=pos[:, 1], z=pos[:, 2], ux=ux, uy=np.zeros(n), uz=uz,
               m=np.full(n, p.rho_gas * vol), rho=np.full(n, p.rho_gas), pres=pres,
               temp=np.full(n, 300.0), h=np.full(n, h), flt_s=np.ones(n), p_type=ptype,
               rad=np.zeros(n), ri=np.zeros(n))
    return p, sph, {}


def scaled_box_bed(n_fluid=2_000_000, n_dem=200_000, seed=0):
    """The same bed with the x extent scaled by 10 (1.0 x 0.02 x 0.4 m)."""
    return box_bed(n_fluid=n_fluid, n_dem=n_dem, seed=seed, lx=1.0)


def dam_break_2d(dx=5.0e-3, seed=0, tank=(1.6, 1.0), column=(0.4, 0.8), rho0=1000.0, alpha=0.02, g=9.81,
                 mu=1.0e-3, cfl=0.2, reference_compat=False):
    """2-D WCSPH dam break: a 0.4 x 0.8 m water column at the left of a
    1.6 x 1.0 m tank (12,800 fluid particles at dx = 5 mm), three layers of
    fixed wall particles (p_type 0) under and beside the tank, Wendland C2
    with h = 1.3 dx, Tait EOS with gamma 7 and c0 = 10 sqrt(2 g H),
    artificial viscosity, gravity along -y, dt = cfl h / c0.  Continuity
    density, predictor-corrector; no KGC, delta-SPH or XSPH (switch them on
    in the returned params).

    Masses are rho0 (h/1.6)^2, the volume the reference's 2-D reference
    density assumes (rho_ref = m / (h/1.6)^2, functions_PREP2.cuh:1392), so
    that rho_ref = rho0.  ``reference_compat`` uses the constants the
    reference hard-wires instead of alpha, g and mu (artificial viscosity
    0.1, gravity 9.8, viscosity 2e-5 for every p_type).
    Returns (params, sph, {})."""
    rng = np.random.default_rng(seed)
    p = reference_params()
    p.solver_type = 0
    p.dim = 2
    p.open_boundary = 0
    p.kernel_type = 3
    p.h_over_dx = 1.3
    p.kgc_solve = 0
    p.delSPH_solve = 0
    p.xsph_solve = 0
    p.fva_solve = 1
    p.gamma = 7.0
    H = column[1]
    if reference_compat:
        alpha, g, mu = 0.1, 9.8, 2.0e-5
    p.soundspeed = 10.0 * np.sqrt(2.0 * g * H)
    p.rho0_eos = rho0
    p.rho_gas = rho0
    p.mu_gas = mu
    p.g_sph = g
    p.g_dem = g
    p.art_visc_alpha = alpha
    h = 1.3 * dx
    p.dt = float(cfl * h / p.soundspeed)
    p.u_limit = 20.0 * p.soundspeed
    p.freq_filt = 20
    nfx, nfy = int(round(column[0] / dx)), int(round(column[1] / dx))
    ntx, nty = int(round(tank[0] / dx)), int(round(tank[1] / dx))
    ii, jj = np.meshgrid(np.arange(nfx), np.arange(nfy), indexing="ij")
    fluid = np.stack([(ii.T.ravel() + 0.5) * dx, (jj.T.ravel() + 0.5) * dx], 1)   # x fastest
    wi, wj = np.meshgrid(np.arange(-3, ntx + 3), np.arange(-3, nty), indexing="ij")
    wall = (wi < 0) | (wi >= ntx) | (wj < 0)
    walls = np.stack([(wi.T[wall.T] + 0.5) * dx, (wj.T[wall.T] + 0.5) * dx], 1)
    pos = np.concatenate([fluid, walls])
    n = len(pos)
    pos = pos + rng.uniform(-0.01 * dx, 0.01 * dx, size=(n, 2))
    ptype = np.concatenate([np.ones(len(fluid), np.int32), np.zeros(len(walls), np.int32)])
    m = rho0 * (h / 1.6) ** 2
    sph = dict(x=pos[:, 0], y=pos[:, 1], z=np.zeros(n), ux=np.zeros(n), uy=np.zeros(n), uz=np.zeros(n),
               m=np.full(n, m), rho=np.full(n, rho0), pres=np.zeros(n), temp=np.full(n, 300.0),
               h=np.full(n, h), flt_s=np.ones(n), p_type=ptype, rad=np.zeros(n), ri=np.zeros(n))
    return p, sph, {}


# ---------------------------------------------------------------------------
# reference input formats
# ---------------------------------------------------------------------------
def write_input_txt(path, sph, dem):
    """input.txt: tab-separated labels, then one row per particle
    (function_init.cuh:743-891).  SPH rows first, then DEM rows."""
    rows = []
    for d in (sph, dem):
        if not d:
            continue
        n = len(d["x"])
        cols = []
        for lbl in INPUT_LABELS:
            f = _LABEL_FIELD[lbl]
            v = d.get(f)
            cols.append(np.zeros(n) if v is None else np.asarray(v, dtype=np.float64))
        rows.append(np.stack(cols, 1))
    data = np.concatenate(rows)
    with open(path, "w") as fh:
        fh.write("\t".join(str(l) for l in INPUT_LABELS) + "\n")
        int_cols = {INPUT_LABELS.index(8), INPUT_LABELS.index(29)}
        for r in data:
            fh.write("\t".join(str(int(v)) if k in int_cols else repr(float(v)) for k, v in enumerate(r)) + "\n")


_KERNEL_NAME = {0: "Gaussian", 1: "Quintic", 2: "Quartic", 3: "Wendland2", 4: "Wendland4", 5: "Wendland6"}


def write_solv_txt(path, p):
    """solv.txt in the layout of the reference's input/solv.txt."""
    yn = lambda v: "YES" if v else "NO"
    lines = [
        "# SOPHIA Input: Solver Setup\t// standard input",
        "solver_type (WCSPH/ISPH/DFSPH):\t" + {0: "WCSPH", 1: "ISPH", 2: "DFSPH"}[p.solver_type],
        "dimension(1/2/3): \t%d" % p.dim,
        "property_table(YES/NO):\t" + yn(p.prop_table),
        "kernel type (Gaussian/Quartic/Quintic/Wendland[2/4/6]):\t" + _KERNEL_NAME[p.kernel_type],
        "filter type (Shepard/MLS): \tShepard",
        "density calculation (Direct/Continuity): \t" + ("Continuity" if p.rho_type == 1 else "Direct"),
        "time integration (Euler/Predictor_Corrector): \t" + ("Predictor_Corrector" if p.time_type else "Euler"),
        "fluid type (Liquid/Gas): \tLiquid",
        "simulation type (Single_Phase/Two_Phase):\tSingle_Phase",
        "pressure-force solve(YES/NO): \t" + yn(p.fp_solve),
        "viscous-force solve(YES/NO): \t" + yn(p.fv_solve),
        "turbulence-model (Laminar/k-lm/k-e/SPS/HB): " + ("Laminar", "k-lm", "k-e", "SPS", "HB")[p.turbulence_model],
        "artificial-viscous-force solve(YES/NO): \t" + yn(p.fva_solve),
        "gravitational-force solve(YES/NO): \t" + yn(p.fg_solve),
        "surface-tension-force solve(YES/NO): \t" + yn(p.fs_solve),
        "surface-tension-model (Potential/Curvature)\t" + ("Curvature" if p.surf_model == 2 else "Potential"),
        "interface-sharpness-force solve(YES/NO):\t" + yn(p.interface_solve),
        "boundary-force solve(YES/NO):\t" + yn(p.fb_solve),
        "Conduction(YES/NO):\t" + yn(p.con_solve),
        "Boussinesq-natural-convection solve(YES/NO):\t" + yn(p.boussinesq_solve),
        "Concentration-diffusion(YES/NO):\t" + yn(p.concn_solve),
        "XSPH solve(YES/NO): \t" + yn(p.xsph_solve),
        "kernel-gradient-correction solve(NO/KGC/FPM/DFPM/KGF):\t" + ("KGC" if p.kgc_solve == 1 else "NO"),
        "delta-SPH solve(NO/Molteni/Antuono):\t" + {0: "NO", 1: "Molteni", 2: "Antuono"}[p.delSPH_solve],
        "particle-shifting solve(YES/NO):\t" + yn(p.pst_solve),
        "penetration_box solve(YES/NO):           NO",
        "noslip_boundary (YES/NO):                NO",
        "open boundary (OPEN/PERIODIC/NO):\t" + {0: "NO", 1: "OPEN", 2: "PERIODIC"}[p.open_boundary],
        "switch_ptype (YES/NO):          NO",
        "reference-pressure (Pa): \t%r" % p.p_ref,
        "sound-speed:  %r" % p.soundspeed,
        "reference-density-eos: %r" % p.rho0_eos,
        "gamma (for EOS): \t%r" % p.gamma,
        "kappa: \t%r" % p.kappa,
        "XSPH-coefficient:\t%r" % p.c_xsph,
        "Boundary-coefficient:\t%r" % p.c_repulsive,
        "minimum-iteration:\t%d" % p.min_iteration,
        "maximum-iteration:\t%d" % p.max_iteration,
        "pressure-convergence criterion\t%r" % p.dp_th,
        "density-convergence criterion\t%r" % p.drho_th,
        "pressure-relaxation factor\t%r" % p.p_relaxation,
        "time-step (sec): \t%r" % p.dt,
        "start-time (sec):\t%r" % p.time,
        "end-time (sec):\t%r" % p.time_end,
        "cell-initialization frequency: \t%d" % p.freq_cell,
        "z-indexing (YES/NO)\t" + yn(p.flag_z_index),
        "timestep update (YES/NO)\tNO",
        "neighbor cell type (3X3/5X5)\t3X3",
        "filtering frequency: \t%d" % p.freq_filt,
        "density-renormalization frequency: \t%d" % p.freq_mass_sum,
        "temperature-filtering frequency:\t%d" % p.freq_temp,
        "plot-output frequency:\t%d" % p.freq_output,
        "plot-variables:                         3 rho pres p_type",
        "velocity-limit (m/s): \t%r" % p.u_limit,
        "Xmargin(-): \t%r" % p.margin[0],
        "Xmargin(+): \t%r" % p.margin[1],
        "Ymargin(-): \t%r" % p.margin[2],
        "Ymargin(+): \t%r" % p.margin[3],
        "Zmargin(-): \t%r" % p.margin[4],
        "Zmargin(+): \t%r" % p.margin[5],
        "decouple-stride:  %d" % p.decouple_stride,
    ]
    with open(path, "w") as fh:
        fh.write("\n".join(lines) + "\n")


DATA_TXT = """#p_type 0
//T
10, 100, 200, 300, 400
//h
0, 1000, 2000, 3000, 4000
//k
1, 1, 1, 1, 1
//mu
1e-3, 1e-3, 1e-3, 1e-3, 1e-3
#end
"""


def write_input_dir(path, p, sph, dem):
    os.makedirs(path, exist_ok=True)
    write_solv_txt(os.path.join(path, "solv.txt"), p)
    write_input_txt(os.path.join(path, "input.txt"), sph, dem)
    with open(os.path.join(path, "data.txt"), "w") as fh:
        fh.write(DATA_TXT)


def dam_break_batch(n_beds=64, n_min=2_000, n_max=50_000, seed=0, dx=5.0e-3, reference_compat=False):
    """Uneven batch of 2-D dam breaks for sphdem_create_batch: bed b has a
    water column of about N_b fluid particles (N_b drawn log-uniform in
    [n_min, n_max], seeded), twice as high as wide, in a tank 4 columns wide
    and 1.25 columns high, with three wall layers.  The beds share one
    parameter set: the sound speed of the tallest column and its CFL time
    step.  Returns (params, [sph dict per bed])."""
    rng = np.random.default_rng(seed)
    counts = np.exp(rng.uniform(np.log(n_min), np.log(n_max), size=n_beds))
    beds, params = [], None
    hmax = 0.0
    for b, nf in enumerate(counts):
        w = max(4, int(round(np.sqrt(nf / 2.0)))) * dx
        col = (w, 2.0 * w)
        tank = (4.0 * w, 2.5 * w)
        p, sph, _ = dam_break_2d(dx=dx, seed=seed * 1000 + b, tank=tank, column=col,
                                 reference_compat=reference_compat)
        beds.append(sph)
        if col[1] > hmax:
            hmax, params = col[1], p
    return params, beds


def bed2d_batch(n_beds=64, n_min=2_000, n_max=50_000, seed=0, u_range=(0.1, 0.3), dx=1.25e-3, plane_cells=2.05):
    """Uneven batch of 2-D ISPH-DEM beds (box_bed_2d) for one handle: bed b
    has N_b fluid particles (drawn log-uniform in [n_min, n_max], seeded),
    N_b / 10 spheres, an inlet velocity drawn uniformly from u_range, and
    lies in the plane y = b * plane_cells * 1.1 kappa h, so that no
    neighbour pair crosses two beds (sphdem_set_beds wants the planes more
    than two cells apart).  The beds share the bed width, kernel, materials
    and DEM walls; their heights, outlet slabs and inlet velocities differ.

    Returns (params, sph, dem, rows, parts): sph and dem concatenate the
    beds in order (sphere ids renumbered to stay unique), rows are the
    per-bed rows for Engine(beds=rows), parts[b] = (sph_b, dem_b, rows_b) is
    bed b alone, in its own plane, for the same run in a handle of its own."""
    rng = np.random.default_rng(seed)
    counts = np.exp(rng.uniform(np.log(n_min), np.log(n_max), size=n_beds)).astype(int)
    u_in = rng.uniform(u_range[0], u_range[1], size=n_beds)
    params, parts, rows = None, [], []
    id0 = 0
    for b in range(n_beds):
        p, sph, dem = box_bed_2d(n_fluid=int(counts[b]), dx=dx, seed=seed * 1000 + b, u_in=float(u_in[b]))
        gap = plane_cells * 1.1 * p.kappa * float(sph["h"][0])
        y0 = b * gap
        sph["y"] = np.full(len(sph["x"]), y0)
        dem["y"] = np.full(len(dem["x"]), y0)
        dem["dem_idx"] = dem["dem_idx"] + id0
        id0 += len(dem["x"])
        row = dict(y=y0, inlet_uz=float(u_in[b]), inlet_temp=p.inlet_temp, obc_L1=p.obc_L1, obc_L2=p.obc_L2,
                   obc_L3=p.obc_L3, obc_L4=p.obc_L4)
        rows.append(row)
        parts.append((sph, dem, [row]))
        if params is None or p.box_L[2] > params.box_L[2]:
            params = p
    params = params.copy()
    params.box_c[1] = 0.5 * rows[-1]["y"]
    params.box_L[1] = rows[-1]["y"] + 1.0      # the DEM walls' y extent never binds
    sph = {k: np.concatenate([pt[0][k] for pt in parts]) for k in parts[0][0]}
    dem = {k: np.concatenate([pt[1][k] for pt in parts]) for k in parts[0][1]}
    return params, sph, dem, rows, parts


GENERATORS = {"spouted_bed": spouted_bed, "box_bed": box_bed, "scaled_box_bed": scaled_box_bed,
              "isph_column": isph_column, "dam_break_2d": dam_break_2d, "box_bed_2d": box_bed_2d}


def _cli(argv=None):
    """Write one seeded bed as a reference input directory:

        python -m fluidized_bed_master_b200.beds box_bed --out input --seed 3 --set n_fluid=50000 dx=2e-3

    input.txt, solv.txt and data.txt in the reference's formats, plus
    params.json with every SphdemParams field (the engine extensions such as
    ppe_mode are not solv.txt keys; pass them to sphdem_create_from_dir)."""
    import argparse
    import ast
    import json

    ap = argparse.ArgumentParser(prog="python -m fluidized_bed_master_b200.beds", description=_cli.__doc__,
                                 formatter_class=argparse.RawDescriptionHelpFormatter)
    ap.add_argument("bed", choices=sorted(GENERATORS))
    ap.add_argument("--out", required=True, help="input directory to write")
    ap.add_argument("--seed", type=int, default=0)
    ap.add_argument("--set", nargs="*", default=[], metavar="KEY=VALUE",
                    help="generator arguments, e.g. n_fluid=50000 dx=2e-3 (Python literals)")
    a = ap.parse_args(argv)
    kw = {"seed": a.seed}
    for item in a.set:
        k, _, v = item.partition("=")
        if not k or not _:
            ap.error(f"--set wants KEY=VALUE, got {item!r}")
        kw[k] = ast.literal_eval(v)
    p, sph, dem = GENERATORS[a.bed](**kw)
    write_input_dir(a.out, p, sph, dem)
    with open(os.path.join(a.out, "params.json"), "w") as fh:
        json.dump(p.as_dict(), fh, indent=1)
    print(f"{a.bed}: {len(sph['x'])} SPH + {len(dem['x']) if dem else 0} DEM -> {a.out}")
    return 0


if __name__ == "__main__":
    raise SystemExit(_cli())
