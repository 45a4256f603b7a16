"""ctypes mirror of ``SphdemParams`` (include/sphdem.h).

The field order and types must match the C declaration exactly;
``check_layout`` compares ``ctypes.sizeof`` with ``sphdem_params_size()``
exported by the library.
"""
import ctypes as C

_I32 = [
    "solver_type", "dim", "prop_table", "kernel_type", "flt_type", "rho_type",
    "time_type", "fluid_type", "open_boundary", "simulation_type", "freq_cell",
    "flag_z_index", "flag_timestep_update", "nb_cell_type", "freq_filt",
    "freq_mass_sum", "freq_temp", "freq_output", "fp_solve", "fv_solve",
    "fva_solve", "fg_solve", "fs_solve", "fb_solve", "con_solve",
    "boussinesq_solve", "interface_solve", "surf_model", "xsph_solve",
    "kgc_solve", "delSPH_solve", "delSPH_model", "pst_solve",
    "turbulence_model", "concn_solve", "min_iteration", "max_iteration",
    "penetration_solve", "switch_ptype", "noslip_bc", "decouple_stride",
    "ppe_mode", "warm_start", "ppe_max_iter", "precision", "dem_wall_mask",
    "mlp_train_steps", "mlp_updates", "mlp_seed", "warm_hist", "warm_fit", "w_lanes",
    "dem_list_cap", "ppe_precond",
]
_F64_A = [
    "kappa", "p_ref", "gamma", "dt", "time", "time_end",
]
_F64_B = [
    "u_limit", "c_xsph", "c_repulsive", "drho_th", "dp_th", "p_relaxation",
    "soundspeed", "rho0_eos", "ball_vel", "ppe_tol",
    "rho_gas", "rho_liquid", "mu_gas", "mu_liquid", "g_sph", "g_dem",
    "h_over_dx", "k_sph", "cp_sph", "k_dem", "cp_dem", "dem_shear_modulus",
    "dem_poisson", "dem_damp_coef", "dem_friction_ratio", "dem_contact_range",
    "dem_search_range", "nu_gas", "inlet_uz_mirror", "inlet_temp",
    "obc_L1", "obc_L2", "obc_L3", "obc_L4", "cyl_cx", "cyl_cy", "cyl_r",
]
_F64_C = ["cone_r1", "cone_r2", "cone_h", "wall_rest_n", "wall_rest_s", "wall_mu_s", "wall_mu_rs"]

_fields = [(n, C.c_int32) for n in _I32]
_fields += [(n, C.c_double) for n in _F64_A]
_fields += [("margin", C.c_double * 6)]
_fields += [(n, C.c_double) for n in _F64_B]
_fields += [("box_c", C.c_double * 3), ("box_L", C.c_double * 3), ("cone_c", C.c_double * 3)]
_fields += [(n, C.c_double) for n in _F64_C]
_fields += [("mlp_lr", C.c_double), ("art_visc_alpha", C.c_double), ("art_visc_beta", C.c_double),
            ("delta_sph", C.c_double), ("reserved_d", C.c_double * 4)]


class SphdemParams(C.Structure):
    _fields_ = _fields

    def copy(self):
        other = SphdemParams()
        C.memmove(C.byref(other), C.byref(self), C.sizeof(self))
        return other

    def as_dict(self):
        out = {}
        for name, typ in self._fields_:
            v = getattr(self, name)
            out[name] = list(v) if hasattr(v, "__len__") else v
        return out

    @classmethod
    def from_dict(cls, d):
        """Inverse of as_dict; fields missing from d stay zero."""
        p = cls()
        for name, typ in cls._fields_:
            if name not in d:
                continue
            v = d[name]
            if hasattr(v, "__len__"):
                arr = getattr(p, name)
                for k, x in enumerate(v):
                    arr[k] = x
            else:
                setattr(p, name, v)
        return p


class SphdemStats(C.Structure):
    _fields_ = [
        ("rho_max_sph", C.c_double), ("u_max_sph", C.c_double), ("ftotal_max_sph", C.c_double),
        ("rho_max_dem", C.c_double), ("u_max_dem", C.c_double), ("ftotal_max_dem", C.c_double),
        ("count", C.c_int32), ("ppe_iters", C.c_int32), ("time", C.c_double),
        ("ppe_rel_residual", C.c_double), ("ppe_ms", C.c_double),
        ("overflow_flags", C.c_int32), ("nan_flag", C.c_int32),
        ("ppe_status", C.c_int32), ("mlp_phase", C.c_int32), ("mlp_loss", C.c_double),
        ("mlp_trained_steps", C.c_int32), ("reserved_stats", C.c_int32),
        ("ppe_initial_residual", C.c_double),
        ("ppe_warm_gain", C.c_double), ("ppe_warm_dirs", C.c_int32), ("w_lanes", C.c_int32),
    ]


# PPE modes and warm starts (SPHDEM_PPE_*, SPHDEM_WARM_*)
PPE_REFERENCE, PPE_KRYLOV, PPE_PCG = 0, 1, 2
PRECOND_JACOBI, PRECOND_TWO_LEVEL = 0, 1
WCSPH, ISPH = 0, 1
WARM_PREVIOUS, WARM_MLP, WARM_EXTRAPOLATE, WARM_PROJECT = 0, 1, 2, 3
WARM_HIST_MAX = 8
FIT_RESIDUAL, FIT_AFFINE = 1, 2


# field ids (enum SphdemField)
F = dict(
    x=0, y=1, z=2, ux=3, uy=4, uz=5, wx=6, wy=7, wz=8, m=9, rho=10, pres=11, temp=12,
    h=13, rad=14, ri=15, DEMpor=16, dDEMpor=17, flt_s=18, flt_sd=19, flt_sd2=20,
    ftotalx=21, ftotaly=22, ftotalz=23, fpx=24, fpy=25, fpz=26, pgfx=27, pgfy=28, pgfz=29,
    Fdx_df=30, Fdy_df=31, Fdz_df=32, torqx=33, torqy=34, torqz=35, rho_ref=36,
    temp1=37, temp2=38, temp3=39, dtemp=40, Q_sd=41, ftotal=42, drho=43, grad_rhox=44, grad_rhoy=45,
    vis_t=46,
    p_type=64, i_type=65, buffer_type=66, dem_idx=67, pid=68, cell=69,
)
INT_FIELDS = {"p_type", "i_type", "buffer_type", "dem_idx", "pid", "cell"}

SPH, DEM = 0, 1

STATUS = {
    0: "ok", -1: "invalid argument", -2: "CUDA runtime error", -3: "malformed input",
    -4: "neighbour list or contact history overflow", -5: "non-finite value",
    -6: "bounded device wait timed out", -7: "switch combination not supported",
    -8: "out of memory or size above limit",
}


def reference_params():
    """The reference-compat preset: the reference's own input/solv.txt and
    every constant it hard-wires (same values as sphdem_params_default)."""
    p = SphdemParams()
    p.solver_type = 1
    p.dim = 3
    p.kernel_type = 5
    p.rho_type = 1
    p.time_type = 1
    p.open_boundary = 1
    p.simulation_type = 1
    p.freq_cell = 1
    p.freq_filt = 40
    p.freq_mass_sum = 1
    p.freq_temp = 10
    p.freq_output = 10000
    p.fp_solve = 1
    p.fv_solve = 1
    p.fg_solve = 1
    p.surf_model = 1
    p.xsph_solve = 1
    p.kgc_solve = 1
    p.delSPH_solve = 2
    p.min_iteration = 3
    p.max_iteration = 10
    p.decouple_stride = 1
    p.ppe_max_iter = 500
    p.mlp_train_steps = 500
    p.warm_hist = 8
    p.mlp_updates = 4
    p.mlp_lr = 3e-4
    p.art_visc_alpha = 0.1
    p.art_visc_beta = 0.02
    p.delta_sph = 0.1
    p.dem_wall_mask = 7
    p.kappa = 2.0
    p.gamma = 1.0
    p.dt = 5.0e-7
    p.time_end = 5.0
    p.u_limit = 40.0
    p.c_xsph = 0.1
    p.c_repulsive = 0.00005
    p.drho_th = 0.005
    p.dp_th = 10.0
    p.p_relaxation = 1.0
    p.soundspeed = 200.0
    p.rho0_eos = 1.784
    p.ppe_tol = 1e-6
    p.rho_gas = 1.784
    p.rho_liquid = 1000.0
    p.mu_gas = 2.0e-5
    p.mu_liquid = 1.0e-3
    p.g_sph = 9.8
    p.g_dem = 9.8
    p.h_over_dx = 1.6
    p.k_sph = 0.0518
    p.cp_sph = 1006.4
    p.k_dem = 2.5
    p.cp_dem = 1068.0
    p.dem_shear_modulus = 8.3e8
    p.dem_poisson = 0.23
    p.dem_damp_coef = 0.0535184
    p.dem_friction_ratio = 0.5
    p.dem_contact_range = 2.01
    p.dem_search_range = 3.5
    p.nu_gas = 2.0e-5 / 1.784
    p.inlet_uz_mirror = 24.045
    p.inlet_temp = 823.0
    p.obc_L1, p.obc_L2, p.obc_L3, p.obc_L4 = -10.505, -0.021, 0.006, 10.25
    p.cyl_cx, p.cyl_cy, p.cyl_r = 0.0, 0.0, 0.0125
    p.box_c[:] = [0.0, 0.0, -0.00176647182]
    p.box_L[:] = [1.15, 1.015, 0.03353294364]
    p.cone_c[:] = [0.0, 0.0, 0.0]
    p.cone_r1, p.cone_r2, p.cone_h = 0.0125, 0.0018, 0.01853294364
    p.wall_rest_n, p.wall_rest_s, p.wall_mu_s, p.wall_mu_rs = 0.9, -0.9, 0.10, 0.2
    return p
