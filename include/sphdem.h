/*
 * sphdem.h -- C ABI of the B200 SPH-DEM step engine.
 *
 * The engine replaces the per-step kernel sequence that SOPHIA_gpu's time
 * loop calls once per iteration:
 *   SOPHIA_single_ISPH(...)   ISPH_Calc_seperate.cuh:13-503  (ISPH + DEM)
 * driven by the host loop at ISPH_Calc_seperate.cuh:905-975 (time += dt,
 * count++ after every step).  The reference passes ~40 raw device pointers
 * and reads solver switches from __constant__ k_vii/k_vif
 * (SOPHIA_gpu.cu:47-56, function_init.cuh:1-213).  Here the same switches
 * travel in SphdemParams and the particle state lives behind an opaque
 * handle; every entry point returns an int status (0 = ok, <0 = error) and
 * never exits the process (the reference's CUDA_CHECK calls exit(),
 * ISPH.cuh:1-8).
 *
 * Threading: one handle per device and host thread (the reference runs one
 * pthread per GPU, ISPH.cuh:178-181).  A handle must not be used from two
 * host threads at the same time.  Steps run asynchronously on the handle's
 * CUDA stream; sphdem_get_* synchronise.
 */
#ifndef SPHDEM_H
#define SPHDEM_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes ---------------------------------------------------- */
#define SPHDEM_OK              0
#define SPHDEM_E_ARG          -1   /* bad argument / null pointer            */
#define SPHDEM_E_CUDA         -2   /* a CUDA runtime call failed             */
#define SPHDEM_E_INPUT        -3   /* malformed solv.txt / input.txt / data  */
#define SPHDEM_E_OVERFLOW     -4   /* neighbour list or contact history full */
#define SPHDEM_E_NAN          -5   /* non-finite value detected in the state */
#define SPHDEM_E_TIMEOUT      -6   /* a bounded device wait gave up          */
#define SPHDEM_E_UNSUPPORTED  -7   /* switch combination not implemented     */
#define SPHDEM_E_NOMEM        -8   /* allocation failed / size above limit   */

/* ---- solver switches (values of solv.txt, function_init.cuh:216-615) -- */
#define SPHDEM_WCSPH 0
#define SPHDEM_ISPH  1
#define SPHDEM_DFSPH 2

/* kernel_type (Parameters.cuh) */
#define SPHDEM_KERNEL_GAUSSIAN  0
#define SPHDEM_KERNEL_QUINTIC   1
#define SPHDEM_KERNEL_QUARTIC   2
#define SPHDEM_KERNEL_WENDLAND2 3
#define SPHDEM_KERNEL_WENDLAND4 4
#define SPHDEM_KERNEL_WENDLAND6 5

/* PPE solution method.  REFERENCE = one Jacobi sweep per step with the
 * previous pressure as iterate (functions_PPE2.cuh:542-698, 868-878).
 * KRYLOV = Jacobi-preconditioned BiCGStab on the same operator to a
 * relative residual ppe_tol; PCG = conjugate gradients in the m-weighted
 * inner product sum m_i x_i y_i, in which the operator is self-adjoint
 * without gradient correction (set kgc_solve 0; unequal masses are fine),
 * preconditioned by its diagonal or, with ppe_precond TWO_LEVEL, by the
 * diagonal plus a cell-level coarse correction.  Neither has a reference
 * counterpart; one Jacobi sweep of either operator from the previous
 * pressure is the reference update. */
#define SPHDEM_PPE_REFERENCE 0
#define SPHDEM_PPE_KRYLOV    1
#define SPHDEM_PPE_PCG       2

/* Initial iterate of the KRYLOV/PCG modes.
 *   PREVIOUS:    the previous pressure.
 *   EXTRAPOLATE: the previous pressure plus its last change.
 *   PROJECT:     the best combination of the directions {previous
 *                pressure, its one-sweep Jacobi increment, the last
 *                warm_hist pressure changes}: A-norm optimal (Galerkin)
 *                for PCG, minimal residual for KRYLOV.  Never worse than
 *                PREVIOUS in that norm.
 *   MLP:         PROJECT plus one more direction, the learned MLP's
 *                prediction of what PROJECT misses (x - x0).  The network
 *                trains on the solver's own solutions during the first
 *                mlp_train_steps steps (which use PROJECT).
 * The solver still converges to ppe_tol from any of them, so results do
 * not depend on the initial iterate beyond that tolerance. */
#define SPHDEM_WARM_PREVIOUS    0
#define SPHDEM_WARM_MLP         1
#define SPHDEM_WARM_EXTRAPOLATE 2
#define SPHDEM_WARM_PROJECT     3
#define SPHDEM_WARM_HIST_MAX    8   /* largest warm_hist */
/* warm_fit: how the projected initial iterate weighs its directions.
 * RESIDUAL: least squares on the residual (default: A-norm, Galerkin);
 * AFFINE: the previous pressure keeps coefficient 1 and only the other
 * directions are fitted (to r0 = b - A p_prev). */
#define SPHDEM_FIT_RESIDUAL     1
#define SPHDEM_FIT_AFFINE       2

/* ppe_precond (PCG only): the diagonal of the operator, or the diagonal plus
 * a coarse correction on the NNPS cells (cell aggregates of the solved
 * particles, Galerkin 27-point operators on the cell grid and on 2x2x2
 * aggregates of it, one damped-Jacobi V-cycle, the last level by Cholesky).
 * An engine extension; the reference has no preconditioner. */
#define SPHDEM_PRECOND_JACOBI 0
#define SPHDEM_PRECOND_TWO_LEVEL 1

/* Precision of the non-position fields inside the engine. */
#define SPHDEM_PREC_FP32 0
#define SPHDEM_PREC_FP64 1

typedef struct SphdemParams {
    /* -- integer switches: vii[] of function_init.cuh:2-58 -- */
    int32_t solver_type;        /* vii[0]  */
    int32_t dim;                /* vii[1]  */
    int32_t prop_table;         /* vii[2]  */
    int32_t kernel_type;        /* vii[3]  */
    int32_t flt_type;           /* vii[4]  */
    int32_t rho_type;           /* vii[5]  0 Direct, 1 Continuity */
    int32_t time_type;          /* vii[6]  0 Euler, 1 Predictor_Corrector */
    int32_t fluid_type;         /* vii[7]  */
    int32_t open_boundary;      /* vii[8]  0 NO, 1 OPEN, 2 PERIODIC */
    int32_t simulation_type;    /* vii[9]  */
    int32_t freq_cell;          /* vii[10] */
    int32_t flag_z_index;       /* vii[11] */
    int32_t flag_timestep_update; /* vii[12] */
    int32_t nb_cell_type;       /* vii[13] */
    int32_t freq_filt;          /* vii[14] */
    int32_t freq_mass_sum;      /* vii[15] */
    int32_t freq_temp;          /* vii[16] */
    int32_t freq_output;        /* vii[17] */
    int32_t fp_solve;           /* vii[18] */
    int32_t fv_solve;           /* vii[19] */
    int32_t fva_solve;          /* vii[20] */
    int32_t fg_solve;           /* vii[21] */
    int32_t fs_solve;           /* vii[22] */
    int32_t fb_solve;           /* vii[23] */
    int32_t con_solve;          /* vii[24] */
    int32_t boussinesq_solve;   /* vii[25] */
    int32_t interface_solve;    /* vii[26] */
    int32_t surf_model;         /* vii[27] */
    int32_t xsph_solve;         /* vii[28] */
    int32_t kgc_solve;          /* vii[29] 0 NO, 1 KGC */
    int32_t delSPH_solve;       /* vii[30] 0 NO, 1 Molteni, 2 Antuono */
    int32_t delSPH_model;       /* vii[31] */
    int32_t pst_solve;          /* vii[32] */
    int32_t turbulence_model;   /* vii[33] */
    int32_t concn_solve;        /* vii[34] */
    int32_t min_iteration;      /* vii[35] */
    int32_t max_iteration;      /* vii[36] */
    int32_t penetration_solve;  /* vii[49] */
    int32_t switch_ptype;       /* vii[50] */
    int32_t noslip_bc;          /* vii[51] */
    int32_t decouple_stride;    /* vii[57] */
    int32_t ppe_mode;           /* SPHDEM_PPE_*  (engine extension)      */
    int32_t warm_start;         /* SPHDEM_WARM_* (engine extension)      */
    int32_t ppe_max_iter;       /* KRYLOV iteration cap                  */
    int32_t precision;          /* SPHDEM_PREC_* (engine extension)      */
    int32_t dem_wall_mask;      /* bit0 cylinder_z, bit1 box_z, bit2 truncated_cone_z */
    int32_t mlp_train_steps;    /* WARM_MLP: steps that train the network (projected warm start) */
    int32_t mlp_updates;        /* WARM_MLP: Adam steps per training step */
    int32_t mlp_seed;           /* WARM_MLP: initialisation seed */
    int32_t warm_hist;          /* WARM_PROJECT/MLP: previous pressure changes used (0..SPHDEM_WARM_HIST_MAX) */
    int32_t warm_fit;           /* WARM_PROJECT/MLP: SPHDEM_FIT_* bits */
    int32_t w_lanes;            /* 2-D WCSPH: lanes per particle of the gathers (1,2,4,8,16); 0 = timed at commit */
    int32_t dem_list_cap;       /* ISPH-DEM: SPH -> DEM list entries per particle; 0 = sized at commit from an
                                   exact count.  A particle with more DEM neighbours walks its stencil instead
                                   (same sums, same order). */
    int32_t ppe_precond;        /* PCG: SPHDEM_PRECOND_JACOBI (0) or SPHDEM_PRECOND_TWO_LEVEL (1) */

    /* -- real switches: vif[] of function_init.cuh:59-100 -- */
    double kappa;               /* vif[0]  */
    double p_ref;               /* vif[1]  */
    double gamma;               /* vif[2]  */
    double dt;                  /* vif[3]  */
    double time;                /* vif[4]  start time */
    double time_end;            /* vif[5]  */
    double margin[6];           /* vif[6..11] X-,X+,Y-,Y+,Z-,Z+ */
    double u_limit;             /* vif[12] */
    double c_xsph;              /* vif[13] */
    double c_repulsive;         /* vif[14] */
    double drho_th;             /* vif[15] */
    double dp_th;               /* vif[16] */
    double p_relaxation;        /* vif[17] */
    double soundspeed;          /* vif[25] */
    double rho0_eos;            /* vif[26] */
    double ball_vel;            /* vif[30] */
    double ppe_tol;             /* KRYLOV relative residual target */

    /* -- constants the reference hard-wires with #define; the
     *    reference-compat preset reproduces them exactly. -- */
    double rho_gas;             /* DENSITY_AIR 1.784 (Parameters.cuh:59) */
    double rho_liquid;          /* DENSITY_WATER 1000 (Parameters.cuh:58) */
    double mu_gas;              /* VISCOSITY_AIR 2e-5 (Parameters.cuh:62) */
    double mu_liquid;           /* VISCOSITY_WATER 1e-3 (Parameters.cuh:61) */
    double g_sph;               /* Gravitational_CONST 9.8 (Parameters.cuh:81) */
    double g_dem;               /* 9.8 (functions_DEM_INTERACTION2.cuh:1702) */
    double h_over_dx;           /* 1.6 (functions_MASS.cuh:33) */
    double k_sph;               /* SPH conductivity 0.0518 (functions_PROP.cuh:271) */
    double cp_sph;              /* SPH heat capacity 1006.4 (functions_PROP.cuh:409) */
    double k_dem;               /* DEM conductivity 2.5 (functions_PROP.cuh:258-268) */
    double cp_dem;              /* DEM heat capacity 1068 (functions_PROP.cuh:401) */
    double dem_shear_modulus;   /* 8.3e8 (functions_PROP.cuh:507) */
    double dem_poisson;         /* 0.23 (functions_PROP.cuh:491) */
    double dem_damp_coef;       /* 0.0535184 (e=0.9) (functions_DEM_INTERACTION2.cuh:1471) */
    double dem_friction_ratio;  /* 0.5 (functions_DEM_INTERACTION2.cuh:1528-1530) */
    double dem_contact_range;   /* 2.01 x radius (functions_DEM_INTERACTION2.cuh:1083) */
    double dem_search_range;    /* 3.5 x radius (functions_DEM_INTERACTION2.cuh:1038) */
    double nu_gas;              /* mu/rho used by the drag Reynolds number */
    double inlet_uz_mirror;     /* 24.045 (functions_BC.cuh:962) */
    double inlet_temp;          /* 823 (functions_BC.cuh:966) */
    double obc_L1, obc_L2, obc_L3, obc_L4;  /* functions_NNPS.cuh:2-5 */
    double cyl_cx, cyl_cy, cyl_r;           /* functions_DEM_BC.cuh:254-257 */
    double box_c[3], box_L[3];              /* functions_DEM_BC.cuh:1503-1509 */
    double cone_c[3], cone_r1, cone_r2, cone_h; /* functions_DEM_BC.cuh:723-725,4237-4243 */
    double wall_rest_n, wall_rest_s, wall_mu_s, wall_mu_rs; /* functions_DEM_BC.cuh:1-5 */
    double mlp_lr;              /* WARM_MLP: Adam learning rate */
    double art_visc_alpha;      /* WCSPH artificial viscosity alpha, Alpha 0.1 (Parameters.cuh:83) */
    double art_visc_beta;       /* WCSPH artificial viscosity beta, Beta 0.02 (Parameters.cuh:84) */
    double delta_sph;           /* WCSPH delta-SPH coefficient, delta 0.1 (Parameters.cuh:92) */
    double reserved_d[4];
} SphdemParams;

/* Particle fields addressable through get/set.  Values cross the ABI as
 * double (or int32 for the integer fields), in the engine's current
 * (cell-sorted) order; SPHDEM_F_PID gives the input row of each slot. */
typedef enum SphdemField {
    SPHDEM_F_X = 0, SPHDEM_F_Y, SPHDEM_F_Z,
    SPHDEM_F_UX, SPHDEM_F_UY, SPHDEM_F_UZ,
    SPHDEM_F_WX, SPHDEM_F_WY, SPHDEM_F_WZ,
    SPHDEM_F_M, SPHDEM_F_RHO, SPHDEM_F_PRES, SPHDEM_F_TEMP,
    SPHDEM_F_H, SPHDEM_F_RAD, SPHDEM_F_RI,
    SPHDEM_F_DEMPOR, SPHDEM_F_DDEMPOR, SPHDEM_F_FLT_S,
    SPHDEM_F_FLT_SD, SPHDEM_F_FLT_SD2,
    SPHDEM_F_FTOTALX, SPHDEM_F_FTOTALY, SPHDEM_F_FTOTALZ,
    SPHDEM_F_FPX, SPHDEM_F_FPY, SPHDEM_F_FPZ,
    SPHDEM_F_PGFX, SPHDEM_F_PGFY, SPHDEM_F_PGFZ,
    SPHDEM_F_FDX_DF, SPHDEM_F_FDY_DF, SPHDEM_F_FDZ_DF,
    SPHDEM_F_TORQX, SPHDEM_F_TORQY, SPHDEM_F_TORQZ,
    SPHDEM_F_RHO_REF, SPHDEM_F_TEMP1, SPHDEM_F_TEMP2, SPHDEM_F_TEMP3,
    SPHDEM_F_DTEMP, SPHDEM_F_Q_SD,
    SPHDEM_F_FTOTAL, SPHDEM_F_DRHO, SPHDEM_F_GRAD_RHOX, SPHDEM_F_GRAD_RHOY,
    SPHDEM_F_VIS_T,             /* SPS eddy viscosity of the step (P3.vis_t; 0 unless fv_solve with SPS) */
    /* integer fields (int32 buffers) */
    SPHDEM_F_PTYPE = 64, SPHDEM_F_ITYPE, SPHDEM_F_BUFFER_TYPE,
    SPHDEM_F_DEM_IDX, SPHDEM_F_PID, SPHDEM_F_CELL
} SphdemField;

#define SPHDEM_SPH 0
#define SPHDEM_DEM 1

typedef struct SphdemStats {
    double rho_max_sph, u_max_sph, ftotal_max_sph;   /* ISPH_Calc_seperate.cuh:928-968 */
    double rho_max_dem, u_max_dem, ftotal_max_dem;
    int32_t count;              /* step counter (vii[43])                 */
    int32_t ppe_iters;          /* iterations of the last PPE solve       */
    double  time;               /* simulated time (vif[4])                */
    double  ppe_rel_residual;   /* last PPE relative residual (KRYLOV)    */
    double  ppe_ms;             /* device time of the last PPE solve      */
    int32_t overflow_flags;     /* bit0 SPH list, bit1 DEM history        */
    int32_t nan_flag;
    int32_t ppe_status;         /* 0 converged, 1 iteration cap, 2 breakdown */
    int32_t mlp_phase;          /* learned warm start: 0 off, 1 training, 2 in use */
    double  mlp_loss;           /* MSE of the last training pass (scaled pressure change) */
    int32_t mlp_trained_steps;  /* training steps taken */
    int32_t reserved_stats;
    double  ppe_initial_residual;  /* ||b - A x0|| / ||b|| of the last solve's initial iterate */
    double  ppe_warm_gain;      /* WARM_PROJECT/MLP: c.h of the last fit, the drop of the squared
                                   error norm that the fit achieves (larger is better; comparable
                                   between runs on the same state with the same warm_fit) */
    int32_t ppe_warm_dirs;      /* directions the last fit kept */
    int32_t w_lanes;            /* 2-D WCSPH: lanes per particle in use (w_lanes or the commit-time choice) */
} SphdemStats;

typedef struct SphdemHandle SphdemHandle;

/* Reference-compat preset: the switches of the reference's own
 * input/solv.txt and every hard-wired constant listed above. */
int sphdem_params_default(SphdemParams* p);

/* Keyword parser for solv.txt (function_init.cuh:216-615).  Fields not
 * named in the file keep the values already in *p. */
int sphdem_read_solv(const char* path, SphdemParams* p);

/* Host-only reader of input.txt (function_init.cuh:743-891): particle
 * counts after the SPH/DEM split (p_type <= 1000 is SPH), then one column
 * per call in input order within the set.  No GPU is touched. */
int sphdem_input_counts(const char* input_txt, int32_t* n_sph, int32_t* n_dem);
int sphdem_input_column(const char* input_txt, int which, int field,
                        void* host_dst, size_t bytes);

/* Batch of independent 2-D WCSPH beds in one handle (engine extension;
 * the reference runs one bed per process and time loop, WCSPH_Calc.cuh:
 * 767-1143).  Rows bed_start..bed_start+n_per_bed[b]-1 of the SPH input
 * are bed b, beds in order; sphdem_set_field before commit takes the
 * concatenated beds, each in its own coordinates, which the engine keeps.
 * At commit each bed gets a placement shift for the cell computation only:
 * shifted, the beds sit side by side on shelves of one cell grid with gaps
 * wider than the search stencil, so no neighbour pair crosses beds, and
 * every sphdem_step advances all beds in one graph launch.  SPHDEM_F_PID
 * (the input row) tells the bed of a slot.  All beds share SphdemParams
 * (dt, kernel, EOS, forces).  solver_type WCSPH, dim 2 only. */
int sphdem_create_batch(const SphdemParams* p, int32_t nbeds, const int32_t* n_per_bed,
                        SphdemHandle** out);
/* The placement shift of every bed's cell computation after commit:
 * offsets[2b], offsets[2b+1] (x, y) for bed b (2 nbeds doubles). */
int sphdem_batch_offsets(SphdemHandle* h, double* offsets);

/* Create an engine for n_sph SPH and n_dem DEM particles on the current
 * CUDA device.  Particle data is then uploaded with sphdem_set_field and
 * sphdem_commit_particles. */
int sphdem_create(const SphdemParams* p, int32_t n_sph, int32_t n_dem,
                  SphdemHandle** out);

/* Read input_dir/solv.txt, input_dir/data.txt and input_dir/input.txt
 * (function_init.cuh:216-1182, ISPH.cuh:55-113) and create an engine.
 * ov may be NULL; when given, its non-switch engine extensions
 * (precision, ppe_mode, warm_start, ppe_tol, ppe_max_iter, warm_hist, warm_fit, w_lanes, dem_list_cap,
 * ppe_precond,
 * mlp_train_steps, mlp_updates, mlp_seed, mlp_lr) override the defaults. */
int sphdem_create_from_dir(const char* input_dir, const SphdemParams* ov,
                           SphdemHandle** out);

/* Upload one field for the SPH (which=0) or DEM (which=1) set from host
 * memory.  Before sphdem_commit_particles: input order, any field.  After
 * it: the engine's current slot order (the order sphdem_get_field
 * returns), state fields only (positions, velocities, m, rho, pres, temp,
 * dDEMpor, flt_s, Fd*_df, Q_sd, temp1-3; for a 2-D WCSPH handle x, y,
 * ux, uy, m, rho, pres, temp, flt_s and the last step's ftotalx/y and
 * drho, which its next predictor reads).  bytes = n * 8 (real fields) or
 * n * 4 (int). */
int sphdem_set_field(SphdemHandle* h, int which, int field,
                     const void* host_src, size_t bytes);

/* Bulk transfer of up to SPHDEM_BULK_MAX_FIELDS real fields of one set
 * after sphdem_commit_particles, in the current slot order: host_src[k]
 * (host_dst[k]) holds n doubles of field fields[k].  The doubles are
 * staged through one device buffer and converted on the GPU; the call
 * returns after one stream synchronisation, so pinned host buffers reach
 * full link bandwidth.  set: the state fields sphdem_set_field accepts
 * after commit; get: any real field.  These are the per-step calls of a
 * host that owns the particle state (the copies SOPHIA_gpu makes around
 * its output, ISPH_Calc_seperate.cuh:928-968, for every field). */
#define SPHDEM_BULK_MAX_FIELDS 32
/* (sphdem_set_fields / sphdem_get_fields: page-locked host arrays, such as
 * those of cudaHostAlloc, are read or written in place by the conversion
 * kernel through their mapped device addresses; pageable arrays go through
 * a device staging buffer.  Either way the call returns when the transfer
 * is complete.) */
int sphdem_set_fields(SphdemHandle* h, int which, int32_t nfields,
                      const int32_t* fields, const double* const* host_src);
int sphdem_get_fields(SphdemHandle* h, int which, int32_t nfields,
                      const int32_t* fields, double* const* host_dst);

/* Learned PPE warm start network (engine extension; no reference
 * counterpart): 16 -> 64 -> 64 -> 1 per-particle MLP with ReLU, BF16
 * weights and activations, FP32 accumulation, on tcgen05 tensor cores.
 * Parameters are one flattened FP32 vector of sphdem_mlp_param_count()
 * values: W1[64][16] | b1[64] | W2[64][64] | b2[64] | w3[64] | b3.
 * These two entries run the network on caller-owned DEVICE arrays (rows
 * of 16 BF16 features, row-major) on the given stream and synchronise it:
 *   forward: out[i] = MLP(feat[i]);
 *   grad:    grad[0..P) = dL/dparams of L = sum_i w_i (y_i - t_i)^2 /
 *            weight_sum, grad[P] = sum_i w_i (y_i - t_i)^2, grad[P+1] =
 *            sum_i w_i. */
/* Every wait of these kernels on the tensor cores is bounded (0.2 s); when
 * one runs out the kernel stops issuing work, frees its tensor memory and
 * the call returns SPHDEM_E_TIMEOUT, leaving the context usable.  Failure
 * drill: with SPHDEM_FAULT_DRILL=mlp_wait in the environment,
 * sphdem_mlp_forward withholds its first MMA group, so that wait runs out
 * and the call must return SPHDEM_E_TIMEOUT (no fault, no hang). */
int32_t sphdem_mlp_param_count(void);
int sphdem_mlp_forward(const void* feat_bf16, int32_t n, const float* params,
                       float* out, void* stream);
int sphdem_mlp_grad(const void* feat_bf16, const float* target,
                    const float* weight, int32_t n, const float* params,
                    double weight_sum, float* grad, void* stream);

/* Device time (CUDA events on the call's stream) of the network kernel of
 * the last successful sphdem_mlp_forward / sphdem_mlp_grad call of this
 * host thread (the gradient kernel only, without its reduction), in ms;
 * either pointer may be NULL. */
int sphdem_mlp_last_ms(double* forward_ms, double* grad_ms);

/* State of the learned warm start of a handle (warm_start = WARM_MLP):
 * the flattened FP32 parameters (sphdem_mlp_param_count() values), the
 * feature statistics (SPHDEM_MLP_STATS doubles: feature means[16] and
 * variances[16], pressure scale, rows, training steps seen, Adam step,
 * reserved) and the number of training steps taken.  Setting them lets a
 * trained network move between handles or runs; set trained_steps >=
 * mlp_train_steps to skip training. */
#define SPHDEM_MLP_STATS 40
int sphdem_get_mlp_state(SphdemHandle* h, float* params, double* stats, int32_t* trained_steps);
int sphdem_set_mlp_state(SphdemHandle* h, const float* params, const double* stats, int32_t trained_steps);

/* Finish the particle upload: bounding box, cell grid, buffer tags
 * (ISPH.cuh:104-113, functions_NNPS.cuh:60-200).  Must be called once
 * after the last sphdem_set_field and before the first step. */
int sphdem_commit_particles(SphdemHandle* h);

/* Advance nsteps time steps (one SOPHIA_single_ISPH + time/count update
 * each).  Asynchronous on the handle's stream. */
int sphdem_step(SphdemHandle* h, int32_t nsteps);

/* Copy a field back to host memory (synchronises). */
int sphdem_get_field(SphdemHandle* h, int which, int field,
                     void* host_dst, size_t bytes);

/* Maxima printed by the reference every freq_output/10 steps, plus PPE
 * statistics (synchronises). */
int sphdem_get_stats(SphdemHandle* h, SphdemStats* out);

/* Health check after the steps enqueued so far (synchronises).  Scans the
 * current state for non-finite velocities or densities and reads the
 * status words the kernels set.  Returns SPHDEM_E_OVERFLOW when a
 * neighbour list ran past its capacity or a sphere met more than 16 contact
 * partners (the kernels stay in bounds: a list keeps its first `capacity`
 * entries, and a 17th partner takes slot 0), SPHDEM_E_NAN when the state
 * holds a NaN or inf, else SPHDEM_OK.  The flags stay set for the life of
 * the handle.  The reference has no such check: it exits the process on a
 * CUDA error (CUDA_CHECK, ISPH.cuh:1-8) and only prints maxima every
 * freq_output/10 steps (ISPH_Calc_seperate.cuh:928-968). */
int sphdem_check(SphdemHandle* h);

/* Cell-sorted neighbour list of the SPH set as built for the current
 * step: counts[n_sph] and, for each particle, its neighbours within
 * kappa*h in the reference's visit order (27 cells z,y,x; ascending
 * slot), as slot indices.  cap = row capacity of dst (ints per row). */
int sphdem_get_neighbors(SphdemHandle* h, int32_t* counts, int32_t* dst,
                         int32_t cap);

/* Tangential contact history of the DEM set (16 slots per sphere,
 * class_Cuda_Particle_Array2.cuh:57-58): partner dem_idx (0 = free) as
 * ids[n*16] and spring vectors as springs[n*16*3], particle-major, in the
 * current sorted order. */
int sphdem_get_history(SphdemHandle* h, int32_t* ids, double* springs);

/* Upload a contact history in the layout of sphdem_get_history. */
int sphdem_set_history(SphdemHandle* h, const int32_t* ids, const double* springs);

/* Per-kernel device timing.  While enabled, every step records a CUDA
 * event pair around each engine kernel on the stream it runs on (inside the
 * captured step graph); sphdem_collect_timing synchronises and adds the
 * elapsed times of the last step to per-kernel totals, which
 * sphdem_get_timing reports (kernel k = 0..n-1, name, total ms, count).
 * With the DEM branch concurrent, a kernel's time includes the SMs it
 * shares with the other branch. */
int sphdem_set_timing(SphdemHandle* h, int on);
int sphdem_collect_timing(SphdemHandle* h);

/* Restrict the per-kernel timing to kernel k (the index of
 * sphdem_get_timing), or -1 for every kernel (the default).  Each timed
 * kernel adds two event records to the step graph; timing one kernel keeps
 * the step's own time within a few microseconds of the untimed step. */
int sphdem_set_timing_only(SphdemHandle* h, int k);

/* The ISPH-DEM step runs the DEM kernels that read no SPH pass (DEM NNPS,
 * contact, filters, corrector) on a second stream, forked from and joined
 * to the handle's stream inside the step (on by default).  Off, every
 * kernel runs on the handle's stream, one after another, in the same
 * order; results are identical either way. */
int sphdem_set_concurrency(SphdemHandle* h, int on);

/* Step graphs on (default) or off.  Off, every step launches its kernels
 * one by one and the KRYLOV/PCG iterations are driven from the host (one
 * status read per iteration): slower, but visible to kernel profilers,
 * which cannot see inside graphs with conditional nodes. */
int sphdem_set_graphs(SphdemHandle* h, int on);
int sphdem_get_timing(SphdemHandle* h, int k, char* name, int name_cap,
                      double* total_ms, int64_t* launches);

/* Binary legacy-VTK POLYDATA of the DEM set, the format of
 * save_plot_fluid_vtk_bin_solid_dem (functions_OUTPUT.cuh:1135-1446). */
int sphdem_write_vtk_dem(SphdemHandle* h, const char* path);

/* Binary legacy-VTK POLYDATA of the fluid particles (p_type 1) of the SPH
 * set, the format of save_plot_fluid_vtk_bin_fluid_sph
 * (functions_OUTPUT.cuh:445-651): positions, porosity, conv_rate,
 * pressure, cond_rate, dtemp, buffer_type, density, temperature, uz.  The
 * reference's conv_rate/cond_rate print fields no compiled kernel sets
 * (zero), and are zero here. */
int sphdem_write_vtk_fluid(SphdemHandle* h, const char* path);

/* Output off the critical path.  sphdem_snapshot enqueues, on the handle's
 * stream after the steps enqueued so far, copies of the fields of the DEM
 * and fluid VTK files into a device buffer, and their copy into pinned host
 * memory on a second stream; it returns without waiting, and the next
 * sphdem_step calls run on the GPU while that copy is in flight (the
 * reference copies P1/P2/P3 to the host synchronously inside its step,
 * ISPH_Calc_seperate.cuh:468-490).  sphdem_write_snapshot waits for the copy
 * and writes the files of the snapshot's step (either path may be NULL);
 * they are byte-identical to sphdem_write_vtk_dem / sphdem_write_vtk_fluid
 * at that step.  A new snapshot first waits for the previous copy and
 * replaces it. */
int sphdem_snapshot(SphdemHandle* h);
int sphdem_write_snapshot(SphdemHandle* h, const char* dem_vtk_path, const char* fluid_vtk_path);

/* ---------------------------------------------------------------------
 * Spatially sharded beds (one handle per slab of cell layers along one
 * axis, one GPU each).  The reference shards only its WCSPH step, in x
 * slabs with a halo copied between GPUs every step (SOPHIA_multi,
 * WCSPH_Calc.cuh:368-738, functions_NNPS.cuh:202-303); these calls carry
 * the same idea to the ISPH-DEM step.  A slab handle holds its own cell
 * layers plus a ghost band of G layers on each side and spare slots parked
 * with i_type 3 (outside every cell: skipped by every kernel, sorted behind
 * all cells).  Between steps, each slab sends the particles of its own
 * layers that lie in a neighbour's ghost band, parks everything outside its
 * own layers, and imports what its neighbours sent.  With G at least the
 * number of dependent neighbour passes of one step plus one, the particles
 * of a slab's own layers step exactly as in the unsharded bed (up to the
 * summation order inside a cell).  fluidized_bed_master_b200/slabs.py
 * drives this over torch.distributed (NCCL between GPUs).
 * All device pointers below are on the handle's device; the calls enqueue
 * on the handle's stream after the steps so far.
 * --------------------------------------------------------------------- */

/* The domain a handle of the whole bed (SPH and DEM arrays in input order)
 * would compute at commit: box with margins, h0, temperature offset. */
int sphdem_bed_domain(const SphdemParams* p, const double* sx, const double* sy, const double* sz,
                      const double* sh, const double* stemp, int32_t ns, const double* dx, const double* dy,
                      const double* dz, const double* dh, int32_t nd, double* bbox6, double* h0,
                      double* t_ref);

/* Before commit: the whole bed's bounding box (xmin, xmax, ymin, ymax, zmin,
 * zmax, margins applied), its h0 (cell edge 1.1 kappa h0) and the SPH
 * temperature offset (rounded to FP32), so that every slab has the same
 * cell grid and stores temperatures alike.  The per-wall and per-buffer
 * passes of a slab get headroom for particles that enter its layers. */
int sphdem_set_domain(SphdemHandle* h, const double* bbox6, double h0, double t_ref);

/* Several two-dimensional ISPH-DEM beds in one handle (dim 2): each bed lies
 * in its own plane y = const, and planes more than two cells
 * (2 x 1.1 kappa h) apart share no neighbour pair, so the one handle steps
 * all beds in every launch of its step graph.  A row gives a bed's plane
 * and the open-boundary parameters that differ from bed to bed (they take
 * the place of SphdemParams' inlet_uz_mirror, inlet_temp and obc_L1..L4 for
 * the particles of that bed, the particles in the row's plane: the row
 * with the nearest y).  Replaces what KERNEL_open_boundary_extrapolation3D
 * (functions_BC.cuh:787-984) reads from k_vif and the slab tags of
 * c_initial_inner_outer_particle_single (functions_NNPS.cuh:60-200). */
/* The SPH neighbour-list build of the step (KERNEL_index_particle_to_cell
 * + the list walk of every gather pass, functions_NNPS.cuh): 1 = one thread
 * per particle; 2, 4, 8 = one warp per cell, that many cells per block (FP32
 * build); 0 (the default) = timed at commit on the committed state, the
 * fastest kept.  Every mode writes the same lists in the same order, so the
 * choice changes only the speed.  FP64 handles build one thread per
 * particle.  The SPH -> DEM list of the coupling passes is picked the same
 * way (a thread per particle or a warp per cell); a fixed mode fixes it
 * too (1: per particle, 2/4/8: per cell).  Set before
 * sphdem_commit_particles; read after it. */
int sphdem_set_list_build(SphdemHandle* h, int32_t mode);
int sphdem_get_list_build(SphdemHandle* h, int32_t* mode);

#define SPHDEM_MAX_BEDS 4096
typedef struct {
    double y;                                 /* the bed's plane */
    double inlet_uz, inlet_temp;              /* inlet velocity and temperature */
    double obc_L1, obc_L2, obc_L3, obc_L4;    /* inlet slab [L1, L2), outlet slab [L3, L4) */
} SphdemBedRow;
/* Before sphdem_commit_particles, dim-2 ISPH handles only; nbeds in
 * [1, SPHDEM_MAX_BEDS], planes more than two cells apart (checked at
 * commit: SPHDEM_E_INPUT). */
int sphdem_set_beds(SphdemHandle* h, int32_t nbeds, const SphdemBedRow* rows);

/* Bytes of one particle record of sphdem_slab_export/import (which: SPH or
 * DEM); every real value as a double, the DEM record with its contact
 * history. */
int sphdem_slab_record_bytes(int which);

/* The active (not parked) slots whose cell layer along axis (0 x, 1 y, 2 z)
 * is in [lo, hi), ascending, into d_slots[0, cap); synchronises and returns
 * their number in *count (which may exceed cap). */
int sphdem_slab_select(SphdemHandle* h, int which, int axis, int32_t lo, int32_t hi, int32_t* d_slots,
                       int32_t cap, int32_t* count);

/* Pack the current state of n slots into n records at d_buf. */
int sphdem_slab_export(SphdemHandle* h, int which, const int32_t* d_slots, int32_t n, void* d_buf);

/* Park the active particles whose layer along axis is outside [lo, hi). */
int sphdem_slab_keep(SphdemHandle* h, int which, int axis, int32_t lo, int32_t hi);

/* Unpack n records into the first n parked slots (SPHDEM_E_NOMEM when
 * fewer are parked); synchronises. */
int sphdem_slab_import(SphdemHandle* h, int which, const void* d_buf, int32_t n);

/* Number of active (not parked) particles of one set; synchronises. */
int sphdem_slab_active(SphdemHandle* h, int which, int32_t* n_active);

/* Restart file in input.txt format: tab-separated column labels then one
 * row per particle with all columns (fixes save_restart,
 * functions_OUTPUT.cuh:1926-1955). */
int sphdem_write_restart(SphdemHandle* h, const char* path);

/* Simulated time and step count of the handle. */
int sphdem_get_time(SphdemHandle* h, double* time, int32_t* count);

/* Static particle counts of the handle. */
int sphdem_get_counts(SphdemHandle* h, int32_t* n_sph, int32_t* n_dem);

/* The CUDA stream the handle launches on (as an opaque pointer). */
int sphdem_get_stream(SphdemHandle* h, void** stream);

/* Number of engine kernels launched by the last sphdem_step call. */
int sphdem_get_launch_count(SphdemHandle* h, int64_t* launches);

/* sizeof(SphdemParams) as compiled into the library (binding check). */
int sphdem_params_size(void);

/* Allocation-free cell sort.  No counterpart in the reference: an extra
 * entry point for callers that cannot allocate device memory once their
 * time loop runs (an application that hands out all device memory from its
 * own pool and fixes its footprint at start-up, or a coupled solver whose
 * other streams must not stall on the device-wide synchronisation that
 * cudaMalloc/cudaFree may imply).  It does the engine's NNPS
 * step on caller-owned device arrays: cell key of every particle
 * (functions_NNPS.cuh:762-821), stable sort by cell, cell start/end
 * (functions_NNPS.cuh:670-730).  Inputs: x, y, z (n doubles, device), the
 * grid bbox[6] = xmin,xmax,ymin,ymax,zmin,zmax and nijk[3] = NI,NJ,NK on the
 * host.  Outputs (device, caller-allocated): perm[n] (input index of each
 * sorted slot), cell_key[n] (sorted cell keys), cell_start/cell_end
 * [NI*NJ*NK] (-1 start for an empty cell; cell_end of an empty cell is
 * not written and keeps what the caller's array held).  Work is enqueued
 * on stream.
 * Its scratch is a file-scope __device__ array of
 * SPHDEM_STATIC_SCRATCH_BYTES that every GPU loading the library keeps
 * until exit; n above SPHDEM_STATIC_MAX_PARTICLES returns SPHDEM_E_NOMEM.
 * The first call on a device resolves the array's device address
 * (cudaGetSymbolAddress), so make that first call before any stream
 * capture.  Calls share the array: calls that overlap on the GPU race. */
#define SPHDEM_STATIC_MAX_PARTICLES (1 << 18)
#define SPHDEM_STATIC_SCRATCH_BYTES (8u << 20)
int sphdem_sort_cells_static(const double* x, const double* y, const double* z, int32_t n,
                             const double* bbox, const int32_t* nijk, int32_t* perm,
                             int32_t* cell_key, int32_t* cell_start, int32_t* cell_end,
                             void* stream);

void sphdem_destroy(SphdemHandle* h);

/* Human-readable text of a status code. */
const char* sphdem_strerror(int status);

#ifdef __cplusplus
}
#endif
#endif /* SPHDEM_H */
