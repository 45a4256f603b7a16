/*
 * sphdem_oracle.c -- TEST INFRASTRUCTURE ONLY (see sphdem_oracle.h).
 *
 * A plain-C FP64 restatement of the reference ISPH-DEM step.  Each
 * function below is one reference kernel, written as a serial (or
 * OpenMP) loop over particles with the reference's neighbour visit order
 * (27 cells in z,y,x order, ascending sorted slot inside a cell) and the
 * reference's expression order, so that sums agree with the reference
 * to rounding.  Quirks of the reference are kept on purpose and marked
 * "quirk:".  Positions, fields and accumulators are all double.
 */
#include "sphdem_oracle.h"

#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

/* ---------------------------------------------------------------------- */
/* field storage                                                          */
/* ---------------------------------------------------------------------- */
#define OR_DFIELDS(X)                                                       \
    X(x) X(y) X(z) X(x_star) X(y_star) X(z_star) X(ux) X(uy) X(uz)          \
    X(wx) X(wy) X(wz) X(m) X(ri) X(rad) X(h) X(temp) X(temp1) X(temp2)      \
    X(temp3) X(pres) X(rho) X(flt_s) X(flt_sd) X(flt_sd_2) X(grad_rhox)     \
    X(grad_rhoy) X(grad_rhoz) X(pgf_x) X(pgf_y) X(pgf_z) X(Fdx_b) X(Fdy_b)  \
    X(Fdz_b) X(Fdx_df) X(Fdy_df) X(Fdz_df) X(Fdx_da) X(Fdy_da) X(Fdz_da)    \
    X(DEMpor) X(dDEMpor) X(dDEMpor_prev) X(Q_sd) X(cond) X(vol0) X(vol)     \
    X(elix) X(eliy) X(eliz) X(PPE1) X(PPE2) X(PPE3) X(PPE4) X(XSPH_ux)      \
    X(XSPH_uy) X(XSPH_uz) X(XSPH_temp) X(rho_ref) X(x0) X(y0) X(z0) X(ux0)  \
    X(uy0) X(uz0) X(rho0) X(temp0)
/* per-step scratch (part3 of class_Cuda_Particle_Array2.cuh:108-167) */
#define OR_SFIELDS(X)                                                       \
    X(ftotalx) X(ftotaly) X(ftotalz) X(ftotal) X(fpx) X(fpy) X(fpz)         \
    X(torqx) X(torqy) X(torqz) X(dtemp) X(dtemp1) X(dtemp2) X(dtemp3)       \
    X(drad) X(drho) X(vis_t)
#define OR_IFIELDS(X) X(p_type) X(i_type) X(buffer_type) X(dem_idx) X(pid)

#define NSLOT 16

typedef struct OSet {
    int n;
#define DECL(f) double* f;
    OR_DFIELDS(DECL) OR_SFIELDS(DECL)
#undef DECL
#define DECLI(f) int* f;
    OR_IFIELDS(DECLI)
#undef DECLI
    double* Cm;       /* n*9   */
    double* ct_idx;   /* n*16  contact partner dem_idx, stored as Real */
    double* del_s;    /* n*48  tangential spring, [slot][3]            */
    double* ct_idx_new;
    double* del_s_new;
    int* g_idx;       /* cell of each slot                              */
    int* g_str;       /* num_cells, -1 = empty                          */
    int* g_end;
    int* perm;
} OSet;

struct OracleState {
    SphdemParams p;
    OSet s, d;             /* SPH and DEM sets */
    int NI, NJ, NK, num_cells;
    double xmin, xmax, ymin, ymax, zmin, zmax, dcell, h0;
    int domain_fixed;
    double time;
    int count;
    int committed;
    int nthreads;
    int* nb_cnt;           /* SPH neighbour list of the last step */
    int* nb_list;
    int nb_cap;
    int ppe_iters;         /* last PPE solve (Krylov modes) */
    double ppe_res;
    int ppe_status;
    int nbeds;             /* 2-D beds in planes y = const: rows of */
    double* beds;          /* {y, inlet_uz, inlet_temp, L1, L2, L3, L4} */
};

/* The row of the bed whose plane is nearest y (NULL: the global values). */
static const double* bed_row(const OracleState* S, double y) {
    if (S->nbeds <= 0) return NULL;
    int best = 0;
    for (int b = 1; b < S->nbeds; b++)
        if (fabs(S->beds[7 * b] - y) < fabs(S->beds[7 * best] - y)) best = b;
    return S->beds + 7 * best;
}

static void* xcalloc(size_t n, size_t sz) {
    void* p = calloc(n ? n : 1, sz);
    return p;
}

static int oset_alloc(OSet* o, int n) {
    memset(o, 0, sizeof(*o));
    o->n = n;
#define AL(f) o->f = (double*)xcalloc((size_t)n, sizeof(double)); if (!o->f) return -1;
    OR_DFIELDS(AL) OR_SFIELDS(AL)
#undef AL
#define ALI(f) o->f = (int*)xcalloc((size_t)n, sizeof(int)); if (!o->f) return -1;
    OR_IFIELDS(ALI)
#undef ALI
    o->Cm = (double*)xcalloc((size_t)n * 9, sizeof(double));
    o->ct_idx = (double*)xcalloc((size_t)n * NSLOT, sizeof(double));
    o->del_s = (double*)xcalloc((size_t)n * NSLOT * 3, sizeof(double));
    o->ct_idx_new = (double*)xcalloc((size_t)n * NSLOT, sizeof(double));
    o->del_s_new = (double*)xcalloc((size_t)n * NSLOT * 3, sizeof(double));
    o->g_idx = (int*)xcalloc((size_t)n, sizeof(int));
    o->perm = (int*)xcalloc((size_t)n, sizeof(int));
    for (int i = 0; i < n; i++) o->pid[i] = i;
    return 0;
}

static void oset_free(OSet* o) {
#define FR(f) free(o->f);
    OR_DFIELDS(FR) OR_SFIELDS(FR) OR_IFIELDS(FR)
#undef FR
    free(o->Cm); free(o->ct_idx); free(o->del_s); free(o->ct_idx_new);
    free(o->del_s_new); free(o->g_idx); free(o->g_str); free(o->g_end);
    free(o->perm);
}

/* ---------------------------------------------------------------------- */
/* property functions: functions_PROP.cuh                                  */
/* ---------------------------------------------------------------------- */
/* viscosity(): functions_PROP.cuh:228-246 -- VISCOSITY_AIR for every type
 * when no property table is used. */
static double prop_viscosity(const SphdemParams* p) { return p->mu_gas; }
/* conductivity(): functions_PROP.cuh:248-277 */
static double prop_conductivity(const SphdemParams* p, int ptype) {
    return (abs(ptype) > 1000) ? p->k_dem : p->k_sph;
}
/* heat_capacity(): functions_PROP.cuh:395-417 (argument is p_type). */
static double prop_heat_capacity(const SphdemParams* p, int ptype) {
    return (abs(ptype) > 1000) ? p->cp_dem : p->cp_sph;
}
/* emissivity(): functions_PROP.cuh:418-440 */
static double prop_emissivity(double temp, int ptype) {
    double em;
    if (abs(ptype) > 1000) {
        if (temp >= 700.0)
            em = 0.505586 + 7.92943e-4 * temp - 5.228643e-7 * temp * temp +
                 1.10479e-10 * temp * temp * temp;
        else
            em = 0.842337;
    } else {
        em = 0.54731;
    }
    return em;
}
/* conductivity_1 / diffusivity_1 for DEM: functions_PROP.cuh:279-341 */
static double prop_conductivity_1(int material) { return material == 1 ? 55.0 : 0.84; }
static double prop_diffusivity_1(int material) { return material == 1 ? 1.77e-5 : 2.5e-6; }

/* ---------------------------------------------------------------------- */
/* SPH kernels: functions_KNL.cuh:2-144                                    */
/* ---------------------------------------------------------------------- */
#define REF_PI 3.141592653 /* Parameters.cuh:78 */

/* calc_tmpA: functions_KNL.cuh:2-32 */
static double knl_tmpA(int kt, int dim, double tH) {
    double tA = 0.0;
    if (kt == SPHDEM_KERNEL_GAUSSIAN) {
        if (dim == 2) tA = 1.0 / (REF_PI * pow(tH, 2));
        else if (dim == 3) tA = 1.0 / (pow(REF_PI, 1.5) * pow(tH, 3));
    } else if (kt == SPHDEM_KERNEL_QUINTIC) {
        if (dim == 2) tA = 7.0 / (478.0 * REF_PI * pow(tH, 2));
        else if (dim == 3) tA = 3.0 / (359.0 * REF_PI * pow(tH, 3));
    } else if (kt == SPHDEM_KERNEL_QUARTIC) {
        if (dim == 2) tA = 15.0 / (7.0 * REF_PI * pow(tH, 2));
        else if (dim == 3) tA = 315.0 / (208.0 * REF_PI * pow(tH, 3));
    } else if (kt == SPHDEM_KERNEL_WENDLAND2) {
        if (dim == 2) tA = 2.228169203286535 / (4 * tH * tH);
        else if (dim == 3) tA = 3.342253804929802 / (8 * tH * tH * tH);
    } else if (kt == SPHDEM_KERNEL_WENDLAND4) {
        if (dim == 2) tA = 2.864788975654116 / (4 * tH * tH);
        else if (dim == 3) tA = 4.923856051905513 / (8 * tH * tH * tH);
    } else if (kt == SPHDEM_KERNEL_WENDLAND6) {
        if (dim == 2) tA = 3.546881588905096 / (4 * tH * tH);
        else if (dim == 3) tA = 6.788953041263660 / (8 * tH * tH * tH);
    }
    return tA;
}

/* calc_kernel_wij: functions_KNL.cuh:47-80 */
static double knl_w(int kt, double tA, double tH, double rr) {
    double tR, w = 0.0;
    if (kt == SPHDEM_KERNEL_GAUSSIAN) {
        tR = rr / tH;
        w = tA * exp(-pow(tR, 2));
    } else if (kt == SPHDEM_KERNEL_QUINTIC) {
        tR = rr / tH;
        if (tR < 1) w = tA * (pow(3.0 - tR, 5) - 6.0 * pow(2.0 - tR, 5) + 15.0 * pow(1.0 - tR, 5));
        else if (1 <= tR && tR < 2) w = tA * (pow(3.0 - tR, 5) - 6.0 * pow(2.0 - tR, 5));
        else if (2 <= tR && tR < 3) w = tA * (pow(3.0 - tR, 5));
    } else if (kt == SPHDEM_KERNEL_QUARTIC) {
        tR = rr / tH;
        w = (tR < 2) * tA * (2.0 / 3.0 - 9.0 / 8.0 * pow(tR, 2) + 19.0 / 24.0 * pow(tR, 3) - 5.0 / 32.0 * pow(tR, 4));
    } else if (kt == SPHDEM_KERNEL_WENDLAND2) {
        tR = rr / tH * 0.5;
        w = (tR < 1) * tA * (1 - tR) * (1 - tR) * (1 - tR) * (1 - tR) * (1 + 4 * tR);
    } else if (kt == SPHDEM_KERNEL_WENDLAND4) {
        tR = rr / tH * 0.5;
        w = (tR < 1) * tA * (1 - tR) * (1 - tR) * (1 - tR) * (1 - tR) * (1 - tR) * (1 - tR) *
            (1 + 6 * tR + 11.666666666666666 * tR * tR);
    } else if (kt == SPHDEM_KERNEL_WENDLAND6) {
        tR = rr / tH * 0.5;
        w = (tR < 1) * tA * (1 - tR) * (1 - tR) * (1 - tR) * (1 - tR) * (1 - tR) * (1 - tR) * (1 - tR) *
            (1 - tR) * (1 + 8 * tR + 25 * tR * tR + 32 * tR * tR * tR);
    }
    return w;
}

/* calc_kernel_dwij: functions_KNL.cuh:111-144 */
static double knl_dw(int kt, double tA, double tH, double rr) {
    double tR, dw = 0.0;
    if (kt == SPHDEM_KERNEL_GAUSSIAN) {
        tR = rr / tH;
        dw = (1.0 / tH) * tA * (-2.0) * tR * exp(-pow(tR, 2));
    } else if (kt == SPHDEM_KERNEL_QUINTIC) {
        tR = rr / tH;
        if (tR < 1) dw = (1.0 / tH) * tA * (pow(3.0 - tR, 5) + 30.0 * pow(2.0 - tR, 4) - 75.0 * pow(1.0 - tR, 4));
        else if (1 <= tR && tR < 2) dw = (1.0 / tH) * tA * (-5.0 * pow(3.0 - tR, 4) + 30.0 * pow(2.0 - tR, 4));
        else if (2 <= tR && tR < 3) dw = (1.0 / tH) * tA * (-5.0 * pow(3.0 - tR, 4));
    } else if (kt == SPHDEM_KERNEL_QUARTIC) {
        tR = rr / tH;
        dw = (tR < 2) * (1.0 / tH) * tA * (-9.0 / 8.0 * 2 * tR + 19.0 / 24.0 * 3.0 * pow(tR, 2) - 5.0 / 32.0 * 4.0 * pow(tR, 3));
    } else if (kt == SPHDEM_KERNEL_WENDLAND2) {
        tR = rr / tH * 0.5;
        dw = (tR < 1) * (1 / (2 * tH)) * tA * (-20 * tR * (1 - tR) * (1 - tR) * (1 - tR));
    } else if (kt == SPHDEM_KERNEL_WENDLAND4) {
        tR = rr / tH * 0.5;
        dw = (tR < 1) * (1 / (2 * tH)) * tA *
             (-18.666666666666668 * tR * (1 - tR) * (1 - tR) * (1 - tR) * (1 - tR) * (1 - tR) * (5 * tR + 1));
    } else if (kt == SPHDEM_KERNEL_WENDLAND6) {
        tR = rr / tH * 0.5;
        dw = (tR < 1) * (1 / (2 * tH)) * tA *
             (-22 * tR * (1 - tR) * (1 - tR) * (1 - tR) * (1 - tR) * (1 - tR) * (1 - tR) * (1 - tR) *
              (16 * tR * tR + 7 * tR + 1));
    }
    return dw;
}

/* apply_gradient_correction_3D (KGC branch): functions_KNL.cuh:763-770 */
static inline void kgc_apply(const SphdemParams* p, const double* Cm, double* dx, double* dy, double* dz) {
    if (p->kgc_solve == 1) {
        double a = *dx, b = *dy, c = *dz;
        *dx = Cm[0] * a + Cm[1] * b + Cm[2] * c;
        *dy = Cm[3] * a + Cm[4] * b + Cm[5] * c;
        *dz = Cm[6] * a + Cm[7] * b + Cm[8] * c;
    }
}

/* ---------------------------------------------------------------------- */
/* cell index: functions_NNPS.cuh:378-390, 762-821                         */
/* ---------------------------------------------------------------------- */
static inline int cell_coord(double v, double vmin, double vmax, int N) {
    /* min(floor((v-vmin)/(vmax-vmin)*N), N-1) through the min() macro,
     * then clamp at 0 (functions_NNPS.cuh:774-784). */
    if (vmax == vmin) return 0;
    double f = floor((v - vmin) / (vmax - vmin) * N);
    double r = (f < (double)(N - 1)) ? f : (double)(N - 1);
    int c = (int)r;
    if (c < 0) c = 0;
    return c;
}

static inline void cell_ijk(const OracleState* S, double x, double y, double z, int* ic, int* jc, int* kc) {
    *ic = cell_coord(x, S->xmin, S->xmax, S->NI);
    *jc = cell_coord(y, S->ymin, S->ymax, S->NJ);
    *kc = cell_coord(z, S->zmin, S->zmax, S->NK);
}

static inline double dist3(double xi, double yi, double zi, double xj, double yj, double zj) {
    return sqrt((xi - xj) * (xi - xj) + (yi - yj) * (yi - yj) + (zi - zj) * (zi - zj));
}

/* Iterate the 27-cell stencil of (ic,jc,kc) in the reference order.  The
 * body sees the neighbour slot j. */
#define FOR_NEIGHBOR_CELLS(S, O, ic, jc, kc, j)                                         \
    for (int zz_ = -1; zz_ <= 1; zz_++)                                                 \
        for (int yy_ = -1; yy_ <= 1; yy_++)                                             \
            for (int xx_ = -1; xx_ <= 1; xx_++)                                         \
                if (!(((ic) + xx_) < 0 || ((ic) + xx_) > (S)->NI - 1 || ((jc) + yy_) < 0 || \
                      ((jc) + yy_) > (S)->NJ - 1 || ((kc) + zz_) < 0 || ((kc) + zz_) > (S)->NK - 1)) \
                    for (int kcell_ = ((ic) + xx_) + (S)->NI * ((jc) + yy_) +                 \
                                      (S)->NI * (S)->NJ * ((kc) + zz_),                       \
                             once_ = 1;                                                       \
                         once_ && (O)->g_str[kcell_] != -1; once_ = 0)                        \
                        for (int j = (O)->g_str[kcell_], jend_ = (O)->g_end[kcell_]; j < jend_; j++)

/* ---------------------------------------------------------------------- */
/* NNPS: hash, stable sort, reorder (functions_NNPS.cuh:639-821)           */
/* ---------------------------------------------------------------------- */
static int cmp_pair(const void* a, const void* b) {
    const int64_t* x = (const int64_t*)a;
    const int64_t* y = (const int64_t*)b;
    return (*x > *y) - (*x < *y);
}

static void permute_d(double* f, const int* perm, int n, double* tmp) {
    for (int i = 0; i < n; i++) tmp[i] = f[perm[i]];
    memcpy(f, tmp, sizeof(double) * (size_t)n);
}
static void permute_i(int* f, const int* perm, int n, int* tmp) {
    for (int i = 0; i < n; i++) tmp[i] = f[perm[i]];
    memcpy(f, tmp, sizeof(int) * (size_t)n);
}
static void permute_blk(double* f, const int* perm, int n, int w, double* tmp) {
    if (n <= 0 || w <= 0) return;
    for (int i = 0; i < n; i++) memcpy(tmp + (size_t)i * w, f + (size_t)perm[i] * w, sizeof(double) * (size_t)w);
    memcpy(f, tmp, sizeof(double) * (size_t)n * w);
}

/* KERNEL_index_particle_to_cell_* (NNPS:762-821), cub SortPairs
 * (ISPH_Calc_seperate.cuh:83-85, a stable radix sort -> same permutation as
 * a stable sort on the key), KERNEL_reorder_* (NNPS:670-730) and the
 * memset of part3 (ISPH_Calc_seperate.cuh:102-105). */
static void nnps(OracleState* S, OSet* o) {
    int n = o->n;
    for (int i = 0; i < S->num_cells; i++) o->g_str[i] = -1;  /* cu_memset */
    if (n == 0) return;
    int64_t* keys = (int64_t*)malloc(sizeof(int64_t) * (size_t)n);
    for (int i = 0; i < n; i++) {
        int key;
        if (o->i_type[i] == 3) key = S->num_cells;
        else {
            int ic, jc, kc;
            cell_ijk(S, o->x[i], o->y[i], o->z[i], &ic, &jc, &kc);
            key = ic + S->NI * jc + S->NI * S->NJ * kc;
        }
        keys[i] = ((int64_t)key << 32) | (int64_t)i;  /* stable: ties by index */
    }
    qsort(keys, (size_t)n, sizeof(int64_t), cmp_pair);
    for (int i = 0; i < n; i++) {
        o->perm[i] = (int)(keys[i] & 0xffffffff);
        o->g_idx[i] = (int)(keys[i] >> 32);
    }
    free(keys);
    /* cell start/end */
    for (int i = 0; i < n; i++) {
        int hsh = o->g_idx[i];
        if (i == 0 || hsh != o->g_idx[i - 1]) {
            if (hsh < S->num_cells) o->g_str[hsh] = i;
            if (i > 0 && o->g_idx[i - 1] < S->num_cells) o->g_end[o->g_idx[i - 1]] = i;
        }
        if (i == n - 1 && hsh < S->num_cells) o->g_end[hsh] = i + 1;
    }
    /* reorder every persistent field */
    double* tmp = (double*)malloc(sizeof(double) * (size_t)n * NSLOT * 3);
    int* itmp = (int*)malloc(sizeof(int) * (size_t)n);
#define PD(f) permute_d(o->f, o->perm, n, tmp);
    OR_DFIELDS(PD)
#undef PD
#define PI_(f) permute_i(o->f, o->perm, n, itmp);
    OR_IFIELDS(PI_)
#undef PI_
    permute_blk(o->ct_idx, o->perm, n, NSLOT, tmp);
    permute_blk(o->del_s, o->perm, n, NSLOT * 3, tmp);
    free(tmp);
    free(itmp);
    /* memset(P3, 0) */
#define ZS(f) memset(o->f, 0, sizeof(double) * (size_t)n);
    OR_SFIELDS(ZS)
#undef ZS
    memset(o->Cm, 0, sizeof(double) * (size_t)n * 9);
    /* TP1 = copy of SP1 for the contact history */
    memcpy(o->ct_idx_new, o->ct_idx, sizeof(double) * (size_t)n * NSLOT);
    memcpy(o->del_s_new, o->del_s, sizeof(double) * (size_t)n * NSLOT * 3);
}

/* Neighbour list of the SPH set with the loop of every SPH gather kernel
 * (e.g. functions_PPE2.cuh:609-681): kappa*h_i, self included. */
static void build_sph_list(OracleState* S) {
    OSet* o = &S->s;
    int n = o->n, cap = S->nb_cap;
    for (int i = 0; i < n; i++) {
        int ic, jc, kc, c = 0;
        cell_ijk(S, o->x[i], o->y[i], o->z[i], &ic, &jc, &kc);
        double R = S->p.kappa * o->h[i];
        FOR_NEIGHBOR_CELLS(S, o, ic, jc, kc, j) {
            double d = dist3(o->x[i], o->y[i], o->z[i], o->x[j], o->y[j], o->z[j]) + 1e-20;
            if (d < R) {
                if (c < cap) S->nb_list[(size_t)i * cap + c] = j;
                c++;
            }
        }
        S->nb_cnt[i] = c;
    }
}

/* ---------------------------------------------------------------------- */
/* per-particle prep kernels                                               */
/* ---------------------------------------------------------------------- */
/* KERNEL_set_alpha_{sph,dem}: functions_ALE.cuh:26-69 */
static void k_set_alpha(OSet* o) {
    for (int i = 0; i < o->n; i++) {
        if (o->i_type[i] == 3) continue;
        double v = (o->p_type[i] <= 1000) ? 0.0 : 1.0;
        o->elix[i] = o->eliy[i] = o->eliz[i] = v;
    }
}

/* Two-dimensional ISPH-DEM beds (dim 2) lie in a plane y = const and use
 * the three-dimensional step with these changes (the reference's ISPH step
 * is three-dimensional only; its one two-dimensional coupling kernel,
 * KERNEL_clc_prep2D_coupling, functions_PREP2.cuh:2944-3033, gives the
 * porosity form):
 *  - kernel normalisation and SPH particle volume (h / h_over_dx)^2;
 *  - the gradient correction inverts the x-z block of the moment matrix;
 *  - a DEM sphere (centre in the plane; contact, drag and heat as for a
 *    sphere) enters the porosity with its equatorial disc, 3.14159 r^2, as
 *    the reference's 2-D coupling prep does: its volume spread over a depth
 *    4 r / 3, and its drag and heat act on the fluid per unit depth, i.e.
 *    divided by that depth. */
static double sph_volume(int dim, double th, double hd) {
    return dim == 2 ? (th / hd) * (th / hd) : (th / hd) * (th / hd) * (th / hd);
}

/* KERNEL_clc_mass_init_sph: functions_MASS.cuh:24-43 */
static void k_mass_init(OracleState* S) {
    OSet* o = &S->s;
    for (int i = 0; i < o->n; i++) {
        if (o->p_type[i] > 1000) continue;
        if (o->i_type[i] > 2) continue;
        o->vol0[i] = pow(o->h[i] / S->p.h_over_dx, S->p.dim);
        o->vol[i] = o->vol0[i];
        o->rho0[i] = o->rho[i];
        o->cond[i] = prop_conductivity(&S->p, o->p_type[i]);
    }
}

/* KERNEL_clc_correction_KGC_3D_sph: functions_PREP2.cuh:452-568 */
static void k_kgc(OracleState* S) {
    OSet* o = &S->s;
    const SphdemParams* P = &S->p;
#pragma omp parallel for schedule(dynamic, 64) num_threads(S->nthreads)
    for (int i = 0; i < o->n; i++) {
        if (o->i_type[i] > 2 || o->p_type[i] > 1000) continue;
        double th = o->h[i], tA = knl_tmpA(P->kernel_type, P->dim, th), R = P->kappa * th;
        double xi = o->x[i], yi = o->y[i], zi = o->z[i];
        int ic, jc, kc;
        cell_ijk(S, xi, yi, zi, &ic, &jc, &kc);
        double txx = 0, tyy = 0, tzz = 0, txy = 0, tyz = 0, tzx = 0;
        FOR_NEIGHBOR_CELLS(S, o, ic, jc, kc, j) {
            if (o->p_type[j] <= 1000) {
                double xj = o->x[j], yj = o->y[j], zj = o->z[j];
                double td = dist3(xi, yi, zi, xj, yj, zj);
                if (td > 0 && td < R) {
                    double dw = knl_dw(P->kernel_type, tA, th, td);
                    double mtd = o->m[j] * dw, rtd = 1.0 / (o->rho[j] * td), t;
                    t = -mtd * (xi - xj) * (xi - xj); t *= rtd; txx += t;
                    t = -mtd * (yi - yj) * (xi - xj); t *= rtd; txy += t;
                    t = -mtd * (yi - yj) * (yi - yj); t *= rtd; tyy += t;
                    t = -mtd * (xi - xj) * (zi - zj); t *= rtd; tzx += t;
                    t = -mtd * (yi - yj) * (zi - zj); t *= rtd; tyz += t;
                    t = -mtd * (zi - zj) * (zi - zj); t *= rtd; tzz += t;
                }
            }
        }
        double* C = o->Cm + (size_t)i * 9;
        if (P->dim == 2) {   /* the x-z block */
            double det2 = txx * tzz - tzx * tzx;
            for (int q = 0; q < 9; q++) C[q] = 0;
            C[4] = 1;
            if (fabs(det2) > 1e-4) {
                double r = 1.0 / det2;
                C[0] = tzz * r; C[2] = -tzx * r; C[6] = -tzx * r; C[8] = txx * r;
            } else {
                C[0] = 1; C[8] = 1;
            }
            continue;
        }
        double det = txx * (tyy * tzz - tyz * tyz);
        det -= txy * (txy * tzz - tyz * tzx);
        det += tzx * (txy * tyz - tyy * tzx);
        if (fabs(det) > 1e-4) { /* Min_det, Parameters.cuh:122 */
            double r = 1.0 / det;
            C[0] = (tyy * tzz - tyz * tyz) * r;
            C[1] = (tzx * tyz - txy * tzz) * r;
            C[2] = (txy * tyz - tzx * tyy) * r;
            C[3] = (tzx * tyz - txy * tzz) * r;
            C[4] = (txx * tzz - tzx * tzx) * r;
            C[5] = (tzx * txy - txx * tyz) * r;
            C[6] = (txy * tyz - tzx * tyy) * r;
            C[7] = (tzx * txy - txx * tyz) * r;
            C[8] = (txx * tyy - txy * txy) * r;
        } else {
            C[0] = 1; C[1] = 0; C[2] = 0; C[3] = 0; C[4] = 1; C[5] = 0; C[6] = 0; C[7] = 0; C[8] = 1;
        }
    }
}

/* KERNEL_clc_prep3D_coupling_sph: functions_PREP2.cuh:3190-3364 */
static void k_coupling_prep_sph(OracleState* S) {
    OSet* o = &S->s;
    OSet* d = &S->d;
    const SphdemParams* P = &S->p;
#pragma omp parallel for schedule(dynamic, 64) num_threads(S->nthreads)
    for (int i = 0; i < o->n; i++) {
        if (o->i_type[i] > 2) continue;
        int pti = o->p_type[i];
        o->dDEMpor_prev[i] = o->dDEMpor[i];
        double xi = o->x[i], yi = o->y[i], zi = o->z[i];
        double th = 1 * o->h[i], tA = knl_tmpA(P->kernel_type, P->dim, 1.0 * th), R = P->kappa * 1.0 * th;
        int ic, jc, kc;
        cell_ijk(S, xi, yi, zi, &ic, &jc, &kc);
        double por = 0, sflt = 0, dfx = 0, dfy = 0, dfz = 0;
        FOR_NEIGHBOR_CELLS(S, o, ic, jc, kc, j) {
            double td = dist3(xi, yi, zi, o->x[j], o->y[j], o->z[j]) + 1e-20;
            if (td < R) {
                double w = knl_w(P->kernel_type, tA, 1.0 * th, td);
                int ptj = o->p_type[j];
                if (pti <= 1000 && ptj <= 1000) sflt += o->m[j] / o->rho[j] * w * (ptj == 1);
            }
        }
        FOR_NEIGHBOR_CELLS(S, d, ic, jc, kc, j) {
            double xj = d->x[j], yj = d->y[j], zj = d->z[j];
            double td = dist3(xi, yi, zi, xj, yj, zj) + 1e-20;
            if (td < R) {
                double w = knl_w(P->kernel_type, tA, 1.0 * th, td);
                double dw = knl_dw(P->kernel_type, tA, 1.0 * th, td);
                double tdwx = dw * (xi - xj) / td, tdwy = dw * (yi - yj) / td, tdwz = dw * (zi - zj) / td;
                double rj = d->rad[j];
                int ptj = d->p_type[j];
                if (pti <= 1000 && ptj > 1000 && P->dim == 2) {
                    por += w * 3.14159 * rj * rj;
                    dfx += tdwx * d->ux[j] * 3.14159 * rj * rj;
                    dfy += tdwy * d->uy[j] * 3.14159 * rj * rj;
                    dfz += tdwz * d->uz[j] * 3.14159 * rj * rj;
                } else if (pti <= 1000 && ptj > 1000) {
                    por += w * 4.18879 * rj * rj * rj;
                    dfx += tdwx * d->ux[j] * 4.18879 * rj * rj * rj;
                    dfy += tdwy * d->uy[j] * 4.18879 * rj * rj * rj;
                    dfz += tdwz * d->uz[j] * 4.18879 * rj * rj * rj;
                }
            }
        }
        if (pti <= 1000) {
            o->DEMpor[i] = 1.0 - (por / (sflt + 1e-20));
            o->dDEMpor[i] = (dfx + dfy + dfz) / (sflt + 1e-20);
        }
    }
}

/* KERNEL_clc_prep3D_coupling_dem: functions_PREP2.cuh:3367-3523 */
static void k_coupling_prep_dem(OracleState* S) {
    OSet* o = &S->s;
    OSet* d = &S->d;
    const SphdemParams* P = &S->p;
#pragma omp parallel for schedule(dynamic, 16) num_threads(S->nthreads)
    for (int i = 0; i < d->n; i++) {
        if (d->i_type[i] > 2) continue;
        int pti = d->p_type[i];
        double xi = d->x[i], yi = d->y[i], zi = d->z[i];
        double th = 1 * d->h[i], tA = knl_tmpA(P->kernel_type, P->dim, 1.0 * th), R = P->kappa * 1.0 * th;
        int ic, jc, kc;
        cell_ijk(S, xi, yi, zi, &ic, &jc, &kc);
        double por = 0, f3 = 0, f1 = 0, f1b = 0;
        FOR_NEIGHBOR_CELLS(S, o, ic, jc, kc, j) {
            double td = dist3(xi, yi, zi, o->x[j], o->y[j], o->z[j]) + 1e-20;
            if (td < R) {
                double w = knl_w(P->kernel_type, tA, 1.0 * th, td);
                int ptj = o->p_type[j];
                if (pti > 1000) {
                    if (ptj <= 1000 && ptj != 0 && ptj != 9 && ptj == 1) {
                        f1 += o->m[j] / o->rho[j] * w;
                        f1b += o->m[j] / o->rho[j] * w;
                    }
                    if (ptj <= 1000 && ptj != 0 && ptj != 9 && ptj == 3) f3 += o->m[j] / o->rho[j] * w;
                }
            }
        }
        FOR_NEIGHBOR_CELLS(S, d, ic, jc, kc, j) {
            double td = dist3(xi, yi, zi, d->x[j], d->y[j], d->z[j]) + 1e-20;
            if (td < R) {
                double w = knl_w(P->kernel_type, tA, 1.0 * th, td);
                double rj = d->rad[j];
                if (pti > 1000 && d->p_type[j] > 1000)
                    por += P->dim == 2 ? w * 3.14159 * rj * rj : w * 4.18879 * rj * rj * rj;
            }
        }
        if (pti > 1000) {
            d->flt_s[i] = f3;
            d->flt_sd[i] = f1;
            d->flt_sd_2[i] = f1b;
            d->DEMpor[i] = 1.0 - (por / (f3 + f1 + 1.0e-20));
        }
    }
}

/* KERNEL_clc_prep3D_prep_sph: functions_PREP2.cuh:1623-1679 */
static void k_prep_sph(OracleState* S) {
    OSet* o = &S->s;
    const SphdemParams* P = &S->p;
    double hd = P->h_over_dx;
    for (int i = 0; i < o->n; i++) {
        if (o->i_type[i] > 2 || o->p_type[i] > 1000) continue;
        int pt = o->p_type[i];
        double th = o->h[i], pori = o->DEMpor[i], zi = o->z[i], mref;
        double v = sph_volume(P->dim, th, hd);
        if (pt == -3) mref = P->rho_gas * v * pori;
        else if (pt == 9) mref = P->rho_liquid * v * pori;
        else if (pt == 0) mref = P->rho_gas * v * pori;
        else if (pt == 3) mref = P->rho_gas * v * pori;
        else if (pt == 1) mref = P->rho_gas * v * pori;
        else mref = P->rho_liquid * v * pori;
        if (pt == 9 && zi < 0.05) mref = P->rho_gas * v * pori;
        if (P->dim == 2) o->rho_ref[i] = mref / ((th / hd) * (th / hd));
        if (P->dim == 3) o->rho_ref[i] = mref / ((th / hd) * (th / hd) * (th / hd));
        if (P->rho_type == 1) {
            o->rho0[i] = mref / sph_volume(P->dim, th, hd);
            o->rho[i] = mref / sph_volume(P->dim, th, hd);
            o->m[i] = mref;
        }
    }
}

/* KERNEL_clc_prep3D_sph: functions_PREP2.cuh:1985-2227 (filter, strain
 * rate and SPS eddy viscosity, delta-SPH density gradient).  The surface
 * normals of its fs_solve branch are not formed: the colour function they
 * differentiate is never computed in this step, and the only reader, the
 * curvature model of the advection pass, then adds no force. */
static void k_prep3d_sph(OracleState* S) {
    OSet* o = &S->s;
    const SphdemParams* P = &S->p;
    int filt = (S->count % (P->freq_filt * P->decouple_stride)) == 0;
#pragma omp parallel for schedule(dynamic, 64) num_threads(S->nthreads)
    for (int i = 0; i < o->n; i++) {
        if (o->i_type[i] > 2 || o->p_type[i] > 1000) continue;
        double xi = o->x[i], yi = o->y[i], zi = o->z[i];
        double th = o->h[i], tA = knl_tmpA(P->kernel_type, P->dim, th), R = P->kappa * th;
        double rhoi = o->rho[i], rri = o->rho_ref[i];
        const double* Cm = o->Cm + (size_t)i * 9;
        int ic, jc, kc;
        cell_ijk(S, xi, yi, zi, &ic, &jc, &kc);
        double flt = 0, gx = 0, gy = 0, gz = 0, sr = 0;
        double uxi = o->ux[i], uyi = o->uy[i], uzi = o->uz[i];
        int turb = P->fv_solve == 1 && P->turbulence_model != 0;
        FOR_NEIGHBOR_CELLS(S, o, ic, jc, kc, j) {
            if (o->p_type[j] <= 1000) {
                double xj = o->x[j], yj = o->y[j], zj = o->z[j];
                double mj = o->m[j], rhoj = o->rho[j];
                double td = dist3(xi, yi, zi, xj, yj, zj) + 1e-20;
                if (td < R) {
                    double w = knl_w(P->kernel_type, tA, th, td);
                    double dw = knl_dw(P->kernel_type, tA, th, td);
                    double tdwx = dw * (xi - xj) / td, tdwy = dw * (yi - yj) / td, tdwz = dw * (zi - zj) / td;
                    if (filt) flt += mj / rhoj * w;
                    if (turb) {   /* strain rate, functions_PREP2.cuh:2113-2118 */
                        double ux = uxi - o->ux[j], uy = uyi - o->uy[j], uz = uzi - o->uz[j];
                        double uij2 = ux * ux + uy * uy + uz * uz;
                        double v = -0.5 * mj * (rhoi + rhoj) * uij2;
                        v /= (rhoi * rhoj * td * td);
                        sr += v * (xi - xj) * tdwx + v * (yi - yj) * tdwy + v * (zi - zj) * tdwz;
                    }
                    if (P->delSPH_solve == 2) {
                        kgc_apply(P, Cm, &tdwx, &tdwy, &tdwz);
                        double rj = o->rho_ref[j];
                        gx += -(rhoj / rj - rhoi / rri) * (mj / rhoj) * tdwx;
                        gy += -(rhoj / rj - rhoi / rri) * (mj / rhoj) * tdwy;
                        gz += -(rhoj / rj - rhoi / rri) * (mj / rhoj) * tdwz;
                    }
                }
            }
        }
        if (turb) {   /* functions_PREP2.cuh:2166-2171: Cs_SPS 0.12, L_SPS 0.01 (Parameters.cuh:102-104) */
            double tv = 0.0, tl = th * 0.01;
            sr = sr > 1e-20 ? sr : 1e-20;
            if (P->turbulence_model == 3) tv = (0.12 * tl) * (0.12 * tl) * sr;
            o->vis_t[i] = tv * rhoi;
        }
        if (filt) o->flt_s[i] = flt;
        if (P->delSPH_solve == 2) {
            o->grad_rhox[i] = gx;
            o->grad_rhoy[i] = gy;
            o->grad_rhoz[i] = gz;
        }
    }
}

/* KERNEL_advection_force3D_sph: functions_PPE2.cuh:1251-1607 (pressure-
 * gradient force density, viscous Laplacian with the eddy viscosity,
 * artificial viscosity, interface sharpness force, repulsive boundary
 * force, inter-particle surface tension, gravity, Eulerian convection,
 * conduction).  The curvature surface tension adds no force (its normals
 * are zero, see k_prep3d_sph) and the concentration rate is zero (zero
 * diffusion coefficient, functions_PROP.cuh:460-466); the Boussinesq term
 * reads an unassigned local in the reference and is rejected by the
 * engine's switch check. */
static void k_advection(OracleState* S) {
    OSet* o = &S->s;
    const SphdemParams* P = &S->p;
#pragma omp parallel for schedule(dynamic, 64) num_threads(S->nthreads)
    for (int i = 0; i < o->n; i++) {
        if (o->i_type[i] > 2) continue;
        if (P->open_boundary > 0 && o->buffer_type[i] > 0) continue;
        if (o->p_type[i] >= 1000 || o->p_type[i] <= 0) continue;
        int pti = o->p_type[i];
        double xi = o->x[i], yi = o->y[i], zi = o->z[i];
        double uxi = o->ux[i], uyi = o->uy[i], uzi = o->uz[i];
        double hi = o->h[i], tempi = o->temp[i], pi = o->pres[i], mi = o->m[i], rhoi = o->rho[i];
        double pori = o->DEMpor[i];
        double tA = knl_tmpA(P->kernel_type, P->dim, hi), R = P->kappa * hi;
        double kci = 0, cpi = 0;
        if (P->con_solve) {
            kci = prop_conductivity(P, pti);
            cpi = prop_heat_capacity(P, pti);
        }
        double visi = prop_viscosity(P) + o->vis_t[i];
        const double* Cm = o->Cm + (size_t)i * 9;
        double elix = o->elix[i], eliy = o->eliy[i], eliz = o->eliz[i];
        int ic, jc, kc;
        cell_ijk(S, xi, yi, zi, &ic, &jc, &kc);
        double tx = 0, ty = 0, tz = 0, Rc = 0, px = 0, py = 0, pz = 0;
        double ex = 0, ey = 0, ez = 0, et = 0;
        FOR_NEIGHBOR_CELLS(S, o, ic, jc, kc, j) {
            double xj = o->x[j], yj = o->y[j], zj = o->z[j];
            if (o->p_type[j] < 1000) {
                double td = dist3(xi, yi, zi, xj, yj, zj) + 1e-20;
                if (td < R) {
                    double w = knl_w(P->kernel_type, tA, hi, td);
                    double dw = knl_dw(P->kernel_type, tA, hi, td);
                    double tdwx = dw * (xi - xj) / td, tdwy = dw * (yi - yj) / td, tdwz = dw * (zi - zj) / td;
                    kgc_apply(P, Cm, &tdwx, &tdwy, &tdwz);
                    (void)w;
                    int ptj = o->p_type[j];
                    double uxj = o->ux[j], uyj = o->uy[j], uzj = o->uz[j], mj = o->m[j];
                    double tempj = o->temp[j], rhoj = o->rho[j], pj = o->pres[j], hj = o->h[j];
                    if (P->fp_solve) {
                        double Cp = -pori * (mj) * (pi + pj) / (rhoi * rhoj);
                        px += rhoi / pori * Cp * tdwx;
                        py += rhoi / pori * Cp * tdwy;
                        pz += rhoi / pori * Cp * tdwz;
                    }
                    if (P->fv_solve) {
                        double visj = prop_viscosity(P) + o->vis_t[j], Cv;
                        Cv = (xi - xj) * tdwx + (yi - yj) * tdwy + (zi - zj) * tdwz;
                        Cv *= (visi * visj) / (visi + visj);
                        Cv *= 4 * pori * (mj / (rhoi * rhoj));
                        Cv /= td;
                        Cv /= td;
                        tx += Cv * (uxi - uxj);
                        ty += Cv * (uyi - uyj);
                        tz += Cv * (uzi - uzj);
                    }
                    if (P->fva_solve) {
                        double uij_xij = (uxi - uxj) * (xi - xj) + (uyi - uyj) * (yi - yj) + (uzi - uzj) * (zi - zj);
                        if (uij_xij < 0) {
                            double h_ij = (hi + hj) * 0.5, phi, Pij;
                            phi = h_ij * uij_xij;
                            phi /= (td * td + 0.01 * h_ij * h_ij);
                            Pij = mi * phi * (-0.1 * P->soundspeed + 0.02 * phi); /* Alpha, Beta */
                            Pij /= (rhoi + rhoj);
                            Pij *= 0.5;
                            tx += -(Pij) * tdwx;
                            ty += -(Pij) * tdwy;
                            tz += -(Pij) * tdwz;
                        }
                    }
                    if (P->interface_solve) {
                        /* interface sharpness force (functions_PPE2.cuh:1450-1464): the raw
                         * kernel slope, the neighbour's pressure only across a fluid-fluid
                         * interface (BOUNDARY 0, MOVING 9) */
                        int flag = (pti != 0) && (pti != 9) && (ptj != 0) && (ptj != 9) && (pti != ptj);
                        double mri = mi / rhoi, mrj = mj / rhoj;
                        double Ci = fabs(pi) * mri * mri + fabs(pj) * mrj * mrj * (flag);
                        Ci *= (0.08 / mi) * dw / td;
                        tx += Ci * (xj - xi);
                        ty += Ci * (yj - yi);
                        tz += Ci * (zj - zi);
                    }
                    if (P->fb_solve) {
                        /* repulsive force of non-fluid neighbours on a fluid particle
                         * (functions_PPE2.cuh:1465-1472), with the kernel value */
                        if ((pti == 1) & (ptj != 1)) {
                            double fb = P->c_repulsive / (td + 1e-10) / (td + 1e-10) * w * (2 * mj / (mi + mj));
                            tx += fb * (xi - xj);
                            ty += fb * (yi - yj);
                            tz += fb * (zi - zj);
                        }
                    }
                    if (P->fs_solve && P->surf_model == 1) {
                        /* inter-particle force (functions_PPE2.cuh:1490-1542) with the
                         * cosine kernel of functions_INTERACTION.cuh:1-33 and the half-
                         * distance kernel 0; of the pair strengths of Parameters.cuh:
                         * 134-148 only s_ff1 = 1.1e-6 (fluid-fluid) is non-zero, every
                         * A is 0, and the other pairs add 0 */
                        double tR = td / hi, wipf = -(tR < 2) * 1.0 * cos(3 * 3.141592653 / 4 * tR), whalf = 0.0;
                        double Cs = 0.0;
                        if ((pti == 1) & (ptj == 1)) {
                            Cs = 1.1e-6 * (0.0 * whalf / (mi * (td + 1.0e-10)));
                            Cs -= 1.1e-6 * (wipf / (mi * (td + 1.0e-10)));
                        }
                        tx += Cs * (xi - xj);
                        ty += Cs * (yi - yj);
                        tz += Cs * (zi - zj);
                    }
                    if (elix < 1.0 || eliy < 1.0) {
                        ex += (uxi * (uxj - uxi) * tdwx + uyi * (uxj - uxi) * tdwy + uzi * (uxj - uxi) * tdwz) * mj / rhoj * (1 - elix);
                        ey += (uxi * (uyj - uyi) * tdwx + uyi * (uyj - uyi) * tdwy + uzi * (uyj - uyi) * tdwz) * mj / rhoj * (1 - eliy);
                        ez += (uxi * (uzj - uzi) * tdwx + uyi * (uzj - uzi) * tdwy + uzi * (uzj - uzi) * tdwz) * mj / rhoj * (1 - eliz);
                        if (P->con_solve)
                            et += (uxi * (tempj - tempi) * tdwx + uyi * (tempj - tempi) * tdwy + uzi * (tempj - tempi) * tdwz) * mj / rhoj * (1 - elix);
                    }
                    if (P->con_solve) {
                        double kcj = prop_conductivity(P, ptj), h;
                        h = 4.0 * pori * mj * kcj * kci * (tempi - tempj) * dw;
                        h /= (td + 1e-10) * rhoi * rhoj * (kci + kcj);
                        Rc += h;
                    }
                }
            }
        }
        if (P->fg_solve) tz += -P->g_sph;
        o->ftotalx[i] = 1 * (tx - ex);
        o->ftotaly[i] = 1 * (ty - ey);
        o->ftotalz[i] = 1 * (tz - ez);
        if (P->con_solve) o->dtemp[i] = Rc / cpi * (pti != -1) - et;
        o->pgf_x[i] = px;
        o->pgf_y[i] = py;
        o->pgf_z[i] = pz;
        o->ftotal[i] = sqrt(tx * tx + ty * ty + tz * tz);
    }
}

/* KERNEL_DEM_interaction3D_dem: functions_DEM_INTERACTION2.cuh:888-1766 */
static void k_dem_contact(OracleState* S) {
    OSet* d = &S->d;
    const SphdemParams* P = &S->p;
    const double kdt = P->dt;
#pragma omp parallel for schedule(dynamic, 16) num_threads(S->nthreads)
    for (int i = 0; i < d->n; i++) {
        if (d->i_type[i] != 1 || d->p_type[i] <= 1000) continue;
        int pti = d->p_type[i];
        double xi = d->x[i], yi = d->y[i], zi = d->z[i];
        double uxi = d->ux[i], uyi = d->uy[i], uzi = d->uz[i];
        double wxi = d->wx[i], wyi = d->wy[i], wzi = d->wz[i];
        double radi = d->rad[i], tempi = d->temp[i];
        double temp1i = d->temp1[i], temp2i = d->temp2[i], temp3i = d->temp3[i];
        double pri = P->dem_poisson, Gi = P->dem_shear_modulus, ymi = Gi * (2 * (1 + pri));
        double mi = d->m[i], rii = d->ri[i], rhoi = d->rho[i];
        double kc0 = 0, kc1 = 0, kc2 = 0, kc3 = 0, a0 = 0, a1 = 0, a2 = 0, a3 = 0, kci = 0, cpi = 0, emi = 0;
        if (P->con_solve) {
            double cp = prop_heat_capacity(P, pti);
            kc0 = prop_conductivity(P, pti); a0 = kc0 / (rhoi * cp);
            kc1 = prop_conductivity(P, pti); a1 = kc1 / (rhoi * cp);
            kc2 = prop_conductivity(P, pti); a2 = kc2 / (rhoi * cp);
            kc3 = prop_conductivity(P, pti); a3 = kc3 / (rhoi * cp);
            kci = prop_conductivity(P, pti);
            cpi = prop_heat_capacity(P, pti);
            emi = prop_emissivity(tempi, pti);
        }
        int ic, jc, kc;
        cell_ijk(S, xi, yi, zi, &ic, &jc, &kc);
        double tx = 0, ty = 0, tz = 0, tqx = 0, tqy = 0, tqz = 0;
        double dt0 = 0, dt1 = 0, dt2 = 0, dt3 = 0, dtr = 0, dtc = 0;
        const int n_dr = 3;
        double dr1 = (5.0 / 6.0) * radi / n_dr, dr2 = (1.0 / 6.0) * radi;
        double volm = (4.0 / 3.0) * 3.141592 * (radi * radi * radi - (radi - dr2) * (radi - dr2) * (radi - dr2));
        if (P->con_solve) {
            /* intra-particle 4-shell conduction (diff_conductivity_1 = 0) */
            double A = (2 * kc1 / dr1) / (2 * kc1 / dr1 + kc0 / dr2), B = 1 - A;
            double ts = A * temp1i + B * tempi;
            dt0 = 0.0 * ((tempi - ts) / (2 * dr2)) * ((tempi - ts) / (2 * dr2)) +
                  2 * (a0 / (radi)) * (tempi - ts) / (2 * dr2) + a0 * (tempi - 2 * tempi + ts) / (dr2 * dr2);
            dt1 = 0.0 * ((2 * ts - temp1i - temp2i) / (2 * dr1)) * ((2 * ts - temp1i - temp2i) / (2 * dr1)) +
                  (2 * a1 / (2.5 * dr1)) * (2 * ts - temp1i - temp2i) / (2 * dr1) +
                  a1 * (2 * ts - 3 * temp1i + temp2i) / (dr1 * dr1);
            dt2 = 0.0 * ((temp1i - temp3i) / (2 * dr1)) * ((temp1i - temp3i) / (2 * dr1)) +
                  2 * (a2 / (1.5 * dr1)) * (temp1i - temp3i) / (2 * dr1) +
                  a2 * (temp1i - 2 * temp2i + temp3i) / (dr1 * dr1);
            dt3 = 0.0 * ((temp2i - temp3i) / (2 * dr1)) * ((temp2i - temp3i) / (2 * dr1)) +
                  2 * (a3 / (0.5 * dr1)) * ((temp2i - temp3i) / (2 * dr1)) +
                  a3 * (temp2i - temp3i) / (dr1 * dr1);
        }
        const double* old_id = d->ct_idx + (size_t)i * NSLOT;
        double* new_id = d->ct_idx_new + (size_t)i * NSLOT;
        double* new_ds = d->del_s_new + (size_t)i * NSLOT * 3;
        const double* old_ds = d->del_s + (size_t)i * NSLOT * 3;
        FOR_NEIGHBOR_CELLS(S, d, ic, jc, kc, j) {
            if (d->p_type[j] > 1000) {
                double xj = d->x[j], yj = d->y[j], zj = d->z[j], radj = d->rad[j], tempj = d->temp[j];
                double radij = 1 / (1 / radi + 1 / radj);
                int demj = d->dem_idx[j], ptj = d->p_type[j];
                double td = dist3(xi, yi, zi, xj, yj, zj);
                double ovlp = radi + radj - td;
                if (td < P->dem_search_range * radi && td > 0.0) {
                    if (P->con_solve) {
                        /* radiation between spheres, :1040-1077 */
                        double sb = 5.6704e-8, emj = prop_emissivity(tempj, ptj);
                        double ai = radi / td, aj = radj / td;
                        double dc_r = 0.56 * (2 * radij) * 1.0; /* pow(1-por, -1/3) with integer -1/3 == 0 */
                        double dc_ar = 3.14159 * dc_r * dc_r;
                        double dij = aj - ai;
                        double dmax = 0.5 * (sqrt(1 + 4.0 * dc_ar / (3.14159 * td * td * (1 - dij * dij))) - dij);
                        double ci = (1 - dij * dij) / (2 * dmax) - dij;
                        double cj = (1 - dij * dij) / (2 * (dmax + dij)) + dij;
                        double si = sqrt(1 - ci * ci), sj = sqrt(1 - cj * cj);
                        double ri_cr = radi * si, rj_cr = radj * sj;
                        double td_cr = td - radi * ci - radj * cj;
                        double z_cr = 1 + (4 * rj_cr * rj_cr + td_cr * td_cr) / (ri_cr * ri_cr);
                        double F_cr = 0.5 * (z_cr - sqrt(z_cr * z_cr - 4.0 * rj_cr * rj_cr / (ri_cr * ri_cr)));
                        double F_ij = (1 + ci) * F_cr * 0.5;
                        double ar_i = 2.0 * 3.14159 * radi * radi * (1 - ci);
                        double ar_j = 2.0 * 3.14159 * radj * radj * (1 - cj);
                        double arr = ar_j / ar_i;
                        double Y = F_ij + (1 - F_ij) * (arr / (1 + arr));
                        double einv = (1 - emi) / (emi * ar_i) + (1 - emj) / (emj * ar_j) + 1 / (Y * ar_i);
                        dtr += -sb * (tempi * tempi * tempi * tempi - tempj * tempj * tempj * tempj) / (einv * (rhoi * volm) * cpi);
                    }
                    if (td < P->dem_contact_range * radi) {
                        if (td > 0 && ovlp > 0) {
                            double uxj = d->ux[j], uyj = d->uy[j], uzj = d->uz[j];
                            double wxj = d->wx[j], wyj = d->wy[j], wzj = d->wz[j];
                            double mj = d->m[j], tov = ovlp;
                            if (P->con_solve) {
                                double kcj = prop_conductivity(P, ptj), kij = 1 / (1 / kci + 1 / kcj);
                                dtc += -4.0 * kij * sqrt((2 * ovlp) * (radij - 0.5 * tov)) * (tempi - tempj) / ((rhoi * volm) * cpi);
                            }
                            double prj = P->dem_poisson, Gj = P->dem_shear_modulus, ymj = Gj * (2 * (1 + prj));
                            double dsx = 0, dsy = 0, dsz = 0;
                            int slot = -1;
                            /* history lookup in slot order (:1206-1301) */
                            for (int s = 0; s < NSLOT; s++) {
                                if (old_id[s] == (double)demj) {
                                    dsx = old_ds[s * 3 + 0]; dsy = old_ds[s * 3 + 1]; dsz = old_ds[s * 3 + 2];
                                    slot = s;
                                    break;
                                }
                            }
                            if (slot < 0) {
                                /* quirk: the free-slot test reads the start-of-step copy,
                                 * so two new partners in one step share a slot (:1326-1391) */
                                for (int s = 0; s < NSLOT; s++) {
                                    if (old_id[s] < 1) {
                                        new_id[s] = demj;
                                        slot = s;
                                        break;
                                    }
                                }
                            }
                            /* no free slot (a 17th partner): the reference then writes through an
                             * unset slot index (:1567, undefined); here the new contact acts this step
                             * and is not recorded (slot stays -1), as in the engine */
                            double nx = (xj - xi) / td, ny = (yj - yi) / td, nz = (zj - zi) / td;
                            double rcxi = (radi - 0.5 * tov) * nx, rcyi = (radi - 0.5 * tov) * ny, rczi = (radi - 0.5 * tov) * nz;
                            double rcxj = -(radj - 0.5 * tov) * nx, rcyj = -(radj - 0.5 * tov) * ny, rczj = -(radj - 0.5 * tov) * nz;
                            double urxi = wyi * rczi - wzi * rcyi, uryi = wzi * rcxi - wxi * rczi, urzi = wxi * rcyi - wyi * rcxi;
                            double urxj = wyj * rczj - wzj * rcyj, uryj = wzj * rcxj - wxj * rczj, urzj = wxj * rcyj - wyj * rcxj;
                            double urelx = (uxj + urxj) - (uxi + urxi);
                            double urely = (uyj + uryj) - (uyi + uryi);
                            double urelz = (uzj + urzj) - (uzi + urzi);
                            double unm = nx * urelx + ny * urely + nz * urelz;
                            double unx = unm * nx, uny = unm * ny, unz = unm * nz;
                            double usx = urelx - unx, usy = urely - uny, usz = urelz - unz;
                            dsx += usx * kdt;
                            dsy += usy * kdt;
                            dsz += usz * kdt;
                            double sx = usx / (sqrt(usx * usx + usy * usy + usz * usz) + 1e-20);
                            double sy = usy / (sqrt(usx * usx + usy * usy + usz * usz) + 1e-20);
                            double sz = usz / (sqrt(usx * usx + usy * usy + usz * usz) + 1e-20);
                            double ymij = 1 / (((1 - pri * pri) / ymi) + ((1 - prj * prj) / ymj));
                            double Gij = 1 / (((2 - pri) / Gi) + ((2 - prj) / Gj));
                            radij = 1 / (1 / radi + 1 / radj);
                            double mij = 1 / (1 / mi + 1 / mj);
                            double Cspr = (1.33333) * ymij * sqrt(radij) * sqrt(tov) * tov / mi;
                            double Cspr_s = 8.0 * Gij * sqrt(radij * tov) / mi;
                            double Kn = 2 * ymij * sqrt(radij * tov);
                            double Kd = sqrt(mij * Kn);
                            double Cd = sqrt(3.333333333) * P->dem_damp_coef * Kd / mi;
                            double Kds = sqrt(mij * Cspr_s * mi);
                            double Cds = sqrt(3.333333333) * P->dem_damp_coef * Kds / mi;
                            tx += Cspr * (xi - xj) / td;
                            ty += Cspr * (yi - yj) / td;
                            tz += Cspr * (zi - zj) / td;
                            tx += Cd * unx;
                            ty += Cd * uny;
                            tz += Cd * unz;
                            double fssx = Cspr_s * dsx + Cds * usx;
                            double fssy = Cspr_s * dsy + Cds * usy;
                            double fssz = Cspr_s * dsz + Cds * usz;
                            double sgx = 1.0 * (fssx >= 0) - 1.0 * (fssx < 0);
                            double sgy = 1.0 * (fssy >= 0) - 1.0 * (fssy < 0);
                            double sgz = 1.0 * (fssz >= 0) - 1.0 * (fssz < 0);
                            double mfss = sqrt(fssx * fssx + fssy * fssy + fssz * fssz);
                            double ffx = P->dem_friction_ratio * Cspr * sx;
                            double ffy = P->dem_friction_ratio * Cspr * sy;
                            double ffz = P->dem_friction_ratio * Cspr * sz;
                            double mfsf = sqrt(ffx * ffx + ffy * ffy + ffz * ffz);
                            double fsx = fssx * (mfss < mfsf) + sgx * fabs(ffx) * (mfss >= mfsf);
                            double fsy = fssy * (mfss < mfsf) + sgy * fabs(ffy) * (mfss >= mfsf);
                            double fsz = fssz * (mfss < mfsf) + sgz * fabs(ffz) * (mfss >= mfsf);
                            tx += fsx;
                            ty += fsy;
                            tz += fsz;
                            tqx += mi * (rcyi * fsz - rczi * fsy);
                            tqy += mi * (rczi * fsx - rcxi * fsz);
                            tqz += mi * (rcxi * fsy - rcyi * fsx);
                            if (slot >= 0) {
                                new_id[slot] = demj;
                                new_ds[slot * 3 + 0] = dsx;
                                new_ds[slot * 3 + 1] = dsy;
                                new_ds[slot * 3 + 2] = dsz;
                            }
                        } else {
                            /* release (:1574-1671) */
                            for (int s = 0; s < NSLOT; s++) {
                                if (old_id[s] == (double)demj) {
                                    new_ds[s * 3 + 0] = 0.0;
                                    new_ds[s * 3 + 1] = 0.0;
                                    new_ds[s * 3 + 2] = 0.0;
                                    new_id[s] = 0;
                                    break;
                                }
                            }
                        }
                    }
                }
            }
        }
        if (P->fg_solve) tz += -P->g_dem;
        if (P->con_solve) {
            dt0 = dt0 + dtr + dtc;
            d->dtemp[i] = dt0;
            d->dtemp1[i] = dt1;
            d->dtemp2[i] = dt2;
            d->dtemp3[i] = dt3;
            d->drad[i] = 0.0;
        }
        d->ftotalx[i] = tx;
        d->ftotaly[i] = ty;
        d->ftotalz[i] = tz;
        d->torqx[i] = tqx / rii;
        d->torqy[i] = tqy / rii;
        d->torqz[i] = tqz / rii;
    }
}

/* KERNEL_DEM_coupling3D_dem: functions_SPH_DEM_COUPLING2.cuh:627-1129 */
static void k_dem_coupling(OracleState* S) {
    OSet* o = &S->s;
    OSet* d = &S->d;
    const SphdemParams* P = &S->p;
#pragma omp parallel for schedule(dynamic, 16) num_threads(S->nthreads)
    for (int i = 0; i < d->n; i++) {
        if (d->i_type[i] != 1 || d->p_type[i] <= 1000) continue;
        double xi = d->x[i], yi = d->y[i], zi = d->z[i];
        double uxi = d->ux[i], uyi = d->uy[i], uzi = d->uz[i];
        double radi = d->rad[i], di = 2 * radi, voli = (4.0 / 3.0) * 3.14159 * radi * radi * radi;
        double mi = d->m[i], rhoi = d->rho[i], tempi = d->temp[i];
        double ki, ali, cpi;
        if (radi < 0.0012) { ki = prop_conductivity_1(1); ali = prop_diffusivity_1(1); }
        else { ki = prop_conductivity_1(0); ali = prop_diffusivity_1(0); }
        cpi = (ki) / (ali * rhoi);
        double fa = d->flt_s[i], ff = d->flt_sd[i];
        double ftx = d->ftotalx[i], fty = d->ftotaly[i], ftz = d->ftotalz[i];
        double hi = 1 * d->h[i], tA = knl_tmpA(P->kernel_type, P->dim, 1.0 * hi), R = P->kappa * 1.0 * hi;
        int ic, jc, kc;
        cell_ijk(S, xi, yi, zi, &ic, &jc, &kc);
        double tx = 0, ty = 0, tz = 0, ufx = 0, ufy = 0, ufz = 0, uax = 0, uay = 0, uaz = 0, por = 0;
        double ttf = 0, tta = 0;
        double vis_kif = P->nu_gas, rho_f = 0, vis_kia = P->nu_gas, rho_a = 0;
        FOR_NEIGHBOR_CELLS(S, o, ic, jc, kc, j) {
            if (o->p_type[j] <= 1000 && o->DEMpor[j] < 1.0) {
                double td = dist3(xi, yi, zi, o->x[j], o->y[j], o->z[j]);
                if (td < R) {
                    double w = knl_w(P->kernel_type, tA, 1.0 * hi, td);
                    double mj = o->m[j], porj = o->DEMpor[j], rhoj = o->rho[j], tempj = o->temp[j];
                    int ptj = o->p_type[j];
                    if (ptj == 1 && ff > 0.000001) {
                        vis_kif = P->nu_gas;
                        rho_f = P->rho_gas;
                        ufx += o->ux[j] * mj * w / rhoj;
                        ufy += o->uy[j] * mj * w / rhoj;
                        ufz += o->uz[j] * mj * w / rhoj;
                        por += porj * mj * w / rhoj;
                        ttf += tempj * mj * w / rhoj;
                    }
                    if (ptj == 3 && fa > 0.000001) {
                        vis_kia = P->nu_gas;
                        rho_a = P->rho_gas;
                        uax += o->ux[j] * mj * w / rhoj;
                        uay += o->uy[j] * mj * w / rhoj;
                        uaz += o->uz[j] * mj * w / rhoj;
                        por += porj * mj * w / rhoj;
                        tta += tempj * mj * w / rhoj;
                    }
                    if (ptj != 0 && ptj != 9 && ptj != -3 && ptj != 3) {
                        if (ff > 0.01) {
                            tx += o->pgf_x[j] * (mj / rhoj) * w * voli / (mi * ff + 1.0e-15);
                            ty += o->pgf_y[j] * (mj / rhoj) * w * voli / (mi * ff + 1.0e-15);
                            tz += o->pgf_z[j] * (mj / rhoj) * w * voli / (mi * ff + 1.0e-15);
                        }
                    }
                }
            }
        }
        double pori = por / (d->flt_sd[i] + 1.0e-15);
        double ufxf = ufx / (ff + 1.0e-15), ufyf = ufy / (ff + 1.0e-15), ufzf = ufz / (ff + 1.0e-15);
        double tf = ttf / (ff + 1.0e-15);
        double ufxa = uax / (fa + 1.0e-15), ufya = uay / (fa + 1.0e-15), ufza = uaz / (fa + 1.0e-15);
        double ta = tta / (fa + 1.0e-15);
        double ufxfa = (ufx + uax) / (ff + fa + 1.0e-15), ufyfa = (ufy + uay) / (ff + fa + 1.0e-15), ufzfa = (ufz + uaz) / (ff + fa + 1.0e-15);
        double tfa = (ttf + tta) / (ff + fa + 1.0e-15);
        double uxf = ufxf - uxi, uyf = ufyf - uyi, uzf = ufzf - uzi, tijf = tf - tempi;
        double uxa = ufxa - uxi, uya = ufya - uyi, uza = ufza - uzi, tija = ta - tempi;
        double uxfa = ufxfa - uxi, uyfa = ufyfa - uyi, uzfa = ufzfa - uzi, tijfa = tfa - tempi;
        double f_fluid = ff / (ff + fa + 1.0e-15), f_air = fa / (ff + fa + 1.0e-15);
        double mf = sqrt(uxf * uxf + uyf * uyf + uzf * uzf);
        double ma = sqrt(uxa * uxa + uya * uya + uza * uza);
        double mfa = sqrt(uxfa * uxfa + uyfa * uyfa + uzfa * uzfa);
        double dfx = 0, dfy = 0, dfz = 0, dax = 0, day = 0, daz = 0;
        double dq = 0.0; /* quirk: uninitialised in the reference when no branch runs */
        double a_ht = 6.0 / di;
        d->DEMpor[i] = pori;
        if (mf > 1.0e-8 && (ff + fa) > 0.00001 && f_fluid > 0.65) {
            double Re = di * mf * pori / (vis_kif + 1.0e-15);
            double Cdf = (0.63 + 4.8 / sqrt(Re)) * (0.63 + 4.8 / sqrt(Re));
            double bf = 3.7 - 0.65 * exp(-(1.5 - log10(Re)) * (1.5 - log10(Re)) / 2.0);
            dfx = (1.0 / 8.0) * Cdf * rho_f * 3.14159 * di * di * uxf * mf * pow(pori, 2 - bf) / mi;
            dfy = (1.0 / 8.0) * Cdf * rho_f * 3.14159 * di * di * uyf * mf * pow(pori, 2 - bf) / mi;
            dfz = (1.0 / 8.0) * Cdf * rho_f * 3.14159 * di * di * uzf * mf * pow(pori, 2 - bf) / mi;
            double Nu = 2.0 + 0.6 * pow(Re, 0.5) * 1.0; /* pow(Pr, 1/3) with 1/3 == 0 */
            double hc = Nu * 0.0518 / di;
            dq = hc * a_ht * tijf;
            d->Fdx_df[i] = dfx;
            d->Fdy_df[i] = dfy;
            d->Fdz_df[i] = dfz;
        }
        if (ma > 1.0e-8 && (ff + fa) > 0.00001 && f_air > 0.65) {
            double Re = di * pori * ma / (vis_kia + 1.0e-15);
            double Cd = (0.63 + 4.8 / sqrt(Re)) * (0.63 + 4.8 / sqrt(Re));
            double b = 2.65 * (1.0 + pori) - (5.3 - 3.5 * pori) * pori * pori * exp(-(1.5 - log10(Re)) * (1.5 - log10(Re)) / 2.0);
            dax = (1.0 / 8.0) * Cd * rho_a * 3.14159 * di * di * uxa * ma * pow(pori, -1 - b) / mi;
            day = (1.0 / 8.0) * Cd * rho_a * 3.14159 * di * di * uya * ma * pow(pori, -1 - b) / mi;
            daz = (1.0 / 8.0) * Cd * rho_a * 3.14159 * di * di * uza * ma * pow(pori, -1 - b) / mi;
            double Nu = 2.0 + 0.6 * pow(Re, 0.5) * 1.0;
            double hc = Nu * ki / di;
            dq = hc * a_ht * tija;
        }
        if ((ma > 1.0e-8 || mf > 1.0e-8) && (ff + fa) > 0.00001 && f_air <= 0.65 && f_fluid <= 0.65) {
            double rfa = P->rho_gas * f_air + P->rho_liquid * f_fluid;
            double vfa = P->mu_gas * f_air + P->mu_liquid * f_fluid;
            double vk = vfa / (rfa + 1.0e-15);
            double Re = di * pori * mfa / (vk + 1.0e-15);
            double Cd = (0.63 + 4.8 / sqrt(Re)) * (0.63 + 4.8 / sqrt(Re));
            double b = 2.65 * (1.0 + pori) - (5.3 - 3.5 * pori) * pori * pori * exp(-(1.5 - log10(Re)) * (1.5 - log10(Re)) / 2.0);
            dax = (1.0 / 8.0) * Cd * rfa * 3.14159 * di * di * uxfa * mfa * pow(pori, -1 - b) / mi;
            day = (1.0 / 8.0) * Cd * rfa * 3.14159 * di * di * uyfa * mfa * pow(pori, -1 - b) / mi;
            daz = (1.0 / 8.0) * Cd * rfa * 3.14159 * di * di * uzfa * mfa * pow(pori, -1 - b) / mi;
            double Nu = 2.0 + 0.6 * pow(Re, 0.5) * 1.0;
            double hc = Nu * ki / di;
            dq = hc * a_ht * tijfa;
        }
        d->ftotalx[i] = ftx + dfx / pori + tx;
        d->ftotaly[i] = fty + dfy / pori + ty;
        d->ftotalz[i] = ftz + dfz / pori + tz;
        if (P->con_solve == 1) {
            d->dtemp[i] = dq / (rhoi * cpi);
            d->Q_sd[i] = dq * mi / rhoi;
        }
        d->Fdx_da[i] = dax;
        d->Fdy_da[i] = day;
        d->Fdz_da[i] = daz;
        d->Fdx_b[i] = tx;
        d->Fdy_b[i] = ty;
        d->Fdz_b[i] = tz;
    }
}

/* KERNEL_SPH_coupling3D_sph: functions_SPH_DEM_COUPLING2.cuh:1815-2019 */
static void k_sph_coupling(OracleState* S) {
    OSet* o = &S->s;
    OSet* d = &S->d;
    const SphdemParams* P = &S->p;
#pragma omp parallel for schedule(dynamic, 64) num_threads(S->nthreads)
    for (int i = 0; i < o->n; i++) {
        if (o->i_type[i] != 1 || o->p_type[i] > 1000) continue;
        int pti = o->p_type[i];
        double xi = o->x[i], yi = o->y[i], zi = o->z[i];
        double rhoi = o->rho[i], tempi = o->temp[i];
        double ftx = o->ftotalx[i], fty = o->ftotaly[i], ftz = o->ftotalz[i], dti = o->dtemp[i];
        /* quirk: heat_capacity(ptypei, tempi) -- arguments swapped (:1860) */
        double cpi = (abs((int)tempi) > 1000) ? P->cp_dem : P->cp_sph;
        double hi = 1 * o->h[i], tA = knl_tmpA(P->kernel_type, P->dim, 1.0 * hi), R = P->kappa * 1.0 * hi;
        int ic, jc, kc;
        cell_ijk(S, xi, yi, zi, &ic, &jc, &kc);
        double tx = 0, ty = 0, tz = 0, tt = 0;
        FOR_NEIGHBOR_CELLS(S, d, ic, jc, kc, j) {
            if (d->p_type[j] > 1000) {
                double td = dist3(xi, yi, zi, d->x[j], d->y[j], d->z[j]);
                if (td < R) {
                    if (pti != 9 && pti != -3 && pti != 0) {
                        double w = knl_w(P->kernel_type, tA, 1.0 * hi, td);
                        if (P->dim == 2) w *= 0.75 / d->rad[j];   /* per unit depth, depth 4 r / 3 */
                        double mj = d->m[j];
                        double ffj = d->flt_sd_2[j] + d->flt_s[j];
                        if (pti == 1 || pti == 3) {
                            if (ffj > 0.0) {
                                tx += -(mj / (rhoi)) * d->Fdx_df[j] * w / (ffj + 1.0e-20);
                                ty += -(mj / (rhoi)) * d->Fdy_df[j] * w / (ffj + 1.0e-20);
                                tz += -(mj / (rhoi)) * d->Fdz_df[j] * w / (ffj + 1.0e-20);
                                tt += -d->Q_sd[j] / (rhoi * cpi) * w / (ffj + 1.0e-20);
                            }
                        }
                    }
                }
            }
        }
        o->ftotalx[i] = ftx + tx;
        o->ftotaly[i] = fty + ty;
        o->ftotalz[i] = ftz + tz;
        o->ftotal[i] = sqrt((ftx + tx) * (ftx + tx) + (fty + ty) * (fty + ty) + (ftz + tz) * (ftz + tz));
        if (P->con_solve == 1) o->dtemp[i] = dti + tt;
    }
}

/* KERNEL_clc_projection_{sph,dem}: functions_TIME_ISPH2.cuh:104-308 */
static void k_projection(OracleState* S, OSet* o, double tdt) {
    const SphdemParams* P = &S->p;
    for (int i = 0; i < o->n; i++) {
        if (o->i_type[i] > 2) continue;
        int pt = o->p_type[i], bt = o->buffer_type[i];
        if (pt == 9) {
            o->x0[i] = o->x[i]; o->y0[i] = o->y[i]; o->z0[i] = o->z[i];
            o->ux[i] = P->ball_vel; o->uy[i] = 0; o->uz[i] = 0;
            o->ux0[i] = P->ball_vel; o->uy0[i] = 0; o->uz0[i] = 0;
        } else {
            double tx0 = o->x[i], ty0 = o->y[i], tz0 = o->z[i];
            double tux0 = o->ux[i], tuy0 = o->uy[i], tuz0 = o->uz[i];
            double txp, typ, tzp, tuxp, tuyp, tuzp;
            if (pt >= 0) {
                double ax = o->ftotalx[i] * (bt == 0), ay = o->ftotaly[i] * (bt == 0), az = o->ftotalz[i] * (bt == 0);
                tuxp = tux0 + ax * (tdt);
                tuyp = tuy0 + ay * (tdt);
                tuzp = tuz0 + az * (tdt);
                txp = tx0 + tuxp * (tdt) * (pt > 0) * (o->elix[i]);
                typ = ty0 + tuyp * (tdt) * (pt > 0) * (o->eliy[i]);
                tzp = tz0 + tuzp * (tdt) * (pt > 0) * (o->eliz[i]);
            } else {
                txp = tx0; typ = ty0; tzp = tz0;
                tuxp = o->ux[i]; tuyp = o->uy[i]; tuzp = o->uz[i];
            }
            o->x_star[i] = txp; o->y_star[i] = typ; o->z_star[i] = tzp;
            o->ux[i] = tuxp; o->uy[i] = tuyp; o->uz[i] = tuzp;
            o->x0[i] = tx0; o->y0[i] = ty0; o->z0[i] = tz0;
            o->ux0[i] = tux0; o->uy0[i] = tuy0; o->uz0[i] = tuz0;
        }
        if (S->time == 0) o->rho_ref[i] = o->rho[i];
        if (P->con_solve == 1 && o->p_type[i] > 0) o->temp0[i] = o->temp[i];
    }
}

/* KERNEL_Neumann_boundary3D_sph: functions_BC.cuh:139-274 */
static void k_neumann(OracleState* S) {
    OSet* o = &S->s;
    const SphdemParams* P = &S->p;
#pragma omp parallel for schedule(dynamic, 64) num_threads(S->nthreads)
    for (int i = 0; i < o->n; i++) {
        if (o->p_type[i] > 0) continue;
        double th = o->h[i], tA = knl_tmpA(P->kernel_type, P->dim, 1.0 * th), R = P->kappa * th;
        double xi = o->x[i], yi = o->y[i], zi = o->z[i], pori = o->DEMpor[i];
        int ic, jc, kc;
        cell_ijk(S, xi, yi, zi, &ic, &jc, &kc);
        double tp = 0, flt = 0, tt = 0, tr = 0;
        FOR_NEIGHBOR_CELLS(S, o, ic, jc, kc, j) {
            double td = dist3(xi, yi, zi, o->x[j], o->y[j], o->z[j]) + 1e-20;
            if (o->p_type[j] < 1000 && td < 2.0 * R) {
                int ptj = o->p_type[j];
                if (ptj >= 1) { /* every term is multiplied by (ptype_j>=1) */
                    double w = knl_w(P->kernel_type, tA, 2.0 * th, td);
                    double mj = o->m[j], rhoj = o->rho[j];
                    tp += mj / rhoj * o->pres[j] * w * (ptj >= 1);
                    flt += mj / rhoj * w * (ptj >= 1);
                    tt += mj / rhoj * o->temp[j] * w * (ptj >= 1);
                    tr += rhoj / o->DEMpor[j] * w * mj / rhoj * (ptj >= 1);
                }
            }
        }
        if (flt < 1e-6) {
            o->rho[i] = o->rho_ref[i];
            o->pres[i] = 0.0;
        } else {
            o->pres[i] = (tp) / flt;
            o->temp[i] = tt / flt;
            o->rho[i] = pori * tr / flt;
        }
    }
}

/* ---------------------------------------------------------------------- */
/* PPE solved to a relative residual (engine extension, no reference       */
/* counterpart).  Row i of a solved particle (the rows the reference sweep */
/* updates): d_i p_i - sum_{j solved} a_ij p_j = b_i + sum_{j fixed} a_ij p_j */
/* with a_ij and b_i the terms of KERNEL_PPE3D_sph and d_i = sum_j a_ij, so */
/* one Jacobi sweep from the current pressure is the reference update.    */
/* Jacobi-preconditioned BiCGStab (KRYLOV) or CG (PCG), FP64, stopping at  */
/* ||r||/||b|| <= ppe_tol or ppe_max_iter iterations.                      */
/* ---------------------------------------------------------------------- */
static int ppe_solved_row(const SphdemParams* P, const OSet* o, int i) {
    return o->i_type[i] <= 2 && !(P->open_boundary > 0 && o->buffer_type[i] > 0) && o->p_type[i] < 1000 &&
           o->p_type[i] > 0;
}

typedef struct {
    int n;
    int* rp;        /* row pointers (solved neighbours only) */
    int* cj;
    double* av;
    double *d, *b;
} PpeSys;

static void ppe_matvec(const PpeSys* A, const int* solved, const double* x, double* y, int nthreads) {
#pragma omp parallel for schedule(static) num_threads(nthreads)
    for (int i = 0; i < A->n; i++) {
        if (!solved[i]) {
            y[i] = 0;
            continue;
        }
        double acc = 0;
        for (int k = A->rp[i]; k < A->rp[i + 1]; k++) acc += A->av[k] * x[A->cj[k]];
        y[i] = A->d[i] * x[i] - acc;
    }
}
static double ppe_dot(int n, const double* a, const double* b) {
    double s = 0;
    for (int i = 0; i < n; i++) s += a[i] * b[i];
    return s;
}
static double ppe_wdot(int n, const double* w, const double* a, const double* b) {
    double s = 0;
    for (int i = 0; i < n; i++) s += w[i] * a[i] * b[i];
    return s;
}

static void ppe_krylov(OracleState* S, double tdt) {
    OSet* o = &S->s;
    const SphdemParams* P = &S->p;
    int n = o->n;
    (void)tdt;
    int* solved = (int*)xcalloc(n, sizeof(int));
    int* cnt = (int*)xcalloc(n, sizeof(int));
    for (int i = 0; i < n; i++) solved[i] = ppe_solved_row(P, o, i);
    /* pass 1: solved-neighbour counts; pass 2: coefficients */
    PpeSys A;
    A.n = n;
    A.rp = (int*)xcalloc(n + 1, sizeof(int));
    A.d = (double*)xcalloc(n, sizeof(double));
    A.b = (double*)xcalloc(n, sizeof(double));
    for (int pass = 0; pass < 2; pass++) {
#pragma omp parallel for schedule(dynamic, 64) num_threads(S->nthreads)
        for (int i = 0; i < n; i++) {
            if (!solved[i]) continue;
            double hi = o->h[i], tA = knl_tmpA(P->kernel_type, P->dim, hi), R = P->kappa * hi;
            double xi = o->x[i], yi = o->y[i], zi = o->z[i], rhoi = o->rho[i], pori = o->DEMpor[i];
            const double* Cm = o->Cm + (size_t)i * 9;
            int ic, jc, kc;
            cell_ijk(S, xi, yi, zi, &ic, &jc, &kc);
            int c = 0, k0 = pass ? A.rp[i] : 0;
            double dsum = 0, bfix = 0;
            FOR_NEIGHBOR_CELLS(S, o, ic, jc, kc, j) {
                if (o->p_type[j] < 1000 && o->i_type[j] != 4) {
                    double xj = o->x[j], yj = o->y[j], zj = o->z[j];
                    double td = dist3(xi, yi, zi, xj, yj, zj) + 1e-20;
                    if (td < R) {
                        if (!pass) {
                            if (solved[j]) c++;
                            continue;
                        }
                        double mj = o->m[j], rhoj = o->rho[j], porj = o->DEMpor[j];
                        double dw = knl_dw(P->kernel_type, tA, hi, td);
                        double tdwx = dw * (xi - xj) / td, tdwy = dw * (yi - yj) / td, tdwz = dw * (zi - zj) / td;
                        kgc_apply(P, Cm, &tdwx, &tdwy, &tdwz);
                        double cc = -((xi - xj) * tdwx + (yi - yj) * tdwy + (zi - zj) * tdwz) / td / td;
                        double a = mj * ((pori * rhoi + porj * rhoj) / (rhoj * rhoi)) * cc;
                        dsum += a;
                        if (solved[j]) {
                            A.cj[k0 + c] = j;
                            A.av[k0 + c] = a;
                            c++;
                        } else {
                            bfix += a * o->pres[j];
                        }
                    }
                }
            }
            if (!pass) cnt[i] = c;
            else {
                A.d[i] = dsum;
                A.b[i] = o->PPE3[i] + bfix;
            }
        }
        if (!pass) {
            for (int i = 0; i < n; i++) A.rp[i + 1] = A.rp[i] + cnt[i];
            A.cj = (int*)xcalloc(A.rp[n], sizeof(int));
            A.av = (double*)xcalloc(A.rp[n], sizeof(double));
        }
    }
    double *x = (double*)xcalloc(n, sizeof(double)), *r = (double*)xcalloc(n, sizeof(double));
    double *rh = (double*)xcalloc(n, sizeof(double)), *pp = (double*)xcalloc(n, sizeof(double));
    double *v = (double*)xcalloc(n, sizeof(double)), *ss = (double*)xcalloc(n, sizeof(double));
    double *t = (double*)xcalloc(n, sizeof(double)), *y = (double*)xcalloc(n, sizeof(double));
    double *z = (double*)xcalloc(n, sizeof(double));
    for (int i = 0; i < n; i++) x[i] = solved[i] ? o->pres[i] : 0.0;
    ppe_matvec(&A, solved, x, y, S->nthreads);
    int cg = P->ppe_mode == SPHDEM_PPE_PCG;
    for (int i = 0; i < n; i++) {
        double bi = solved[i] ? A.b[i] : 0.0;
        A.b[i] = bi;
        r[i] = bi - y[i];
        if (cg) {
            z[i] = r[i] / (solved[i] ? A.d[i] : 1.0);
            pp[i] = z[i];
        } else {
            rh[i] = r[i];
        }
    }
    double bn = sqrt(ppe_dot(n, A.b, A.b));
    double res = bn > 0 ? sqrt(ppe_dot(n, r, r)) / bn : 0.0;
    int it = 0, status = 0;
    double tol = P->ppe_tol;
    if (cg) {
        /* Chronopoulos-Gear PCG (the engine's form): u = M^-1 r, w = A u;
         * p = u + beta p, s = w + beta s, x += alpha p, r -= alpha s,
         * u = M^-1 r, w = A u, gamma = r.u, delta = w.u,
         * beta' = gamma/gamma_old, alpha' = gamma/(delta - beta' gamma/alpha) */
        /* a_ij = m_j s_ij with s symmetric: CG on M A p = M b with the
         * preconditioner M D, i.e. inner products weighted by m_i */
        double* w = v;
        double* u = z;
        double* wm = t;
        for (int i = 0; i < n; i++) ss[i] = 0.0, pp[i] = 0.0, wm[i] = solved[i] ? o->m[i] : 0.0;
        ppe_matvec(&A, solved, u, w, S->nthreads);
        double gam = ppe_wdot(n, wm, r, u), del = ppe_wdot(n, wm, w, u);
        double alpha = 0, beta = 0;
        if (bn > 0 && res > tol && it < P->ppe_max_iter) {
            if (!(del != 0.0) || !isfinite(del)) status = 2;
            else alpha = gam / del;
        }
        while (status == 0 && bn > 0 && res > tol && it < P->ppe_max_iter) {
            for (int i = 0; i < n; i++) {
                pp[i] = u[i] + beta * pp[i];
                ss[i] = w[i] + beta * ss[i];
                x[i] += alpha * pp[i];
                r[i] -= alpha * ss[i];
                u[i] = r[i] / (solved[i] ? A.d[i] : 1.0);
            }
            ppe_matvec(&A, solved, u, w, S->nthreads);
            double g1 = ppe_wdot(n, wm, r, u), d1 = ppe_wdot(n, wm, w, u);
            it++;
            res = sqrt(ppe_dot(n, r, r)) / bn;
            if (!isfinite(res)) { status = 2; break; }
            if (res <= tol || it >= P->ppe_max_iter) break;
            double be = g1 / gam;
            double den = d1 - be * g1 / alpha;
            if (!(den != 0.0) || !isfinite(den)) { status = 2; break; }
            beta = be;
            alpha = g1 / den;
            gam = g1;
        }
    } else {
        double rho = 1, alpha = 1, om = 1;
        while (bn > 0 && res > tol && it < P->ppe_max_iter) {
            double rho_new = ppe_dot(n, rh, r);
            double beta = (rho_new / rho) * (alpha / om);
            for (int i = 0; i < n; i++) {
                pp[i] = r[i] + beta * (pp[i] - om * v[i]);
                y[i] = pp[i] / (solved[i] ? A.d[i] : 1.0);
            }
            ppe_matvec(&A, solved, y, v, S->nthreads);
            double rv = ppe_dot(n, rh, v);
            if (!(rv != 0.0) || !isfinite(rv)) { status = 2; break; }
            alpha = rho_new / rv;
            for (int i = 0; i < n; i++) {
                ss[i] = r[i] - alpha * v[i];
                x[i] += alpha * y[i];
                z[i] = ss[i] / (solved[i] ? A.d[i] : 1.0);
            }
            ppe_matvec(&A, solved, z, t, S->nthreads);
            double ts = ppe_dot(n, t, ss), tt = ppe_dot(n, t, t);
            om = tt > 0 ? ts / tt : 0.0;
            for (int i = 0; i < n; i++) {
                x[i] += om * z[i];
                r[i] = ss[i] - om * t[i];
            }
            rho = rho_new;
            it++;
            res = sqrt(ppe_dot(n, r, r)) / bn;
            if (!isfinite(res) || om == 0.0) { status = 2; break; }
        }
    }
    if (status == 0 && res > tol) status = 1;
    for (int i = 0; i < n; i++)
        if (solved[i]) o->pres[i] = x[i];
    S->ppe_iters = it;
    S->ppe_res = res;
    S->ppe_status = status;
    free(x); free(r); free(rh); free(pp); free(v); free(ss); free(t); free(y); free(z);
    free(A.rp); free(A.cj); free(A.av); free(A.d); free(A.b); free(solved); free(cnt);
}

/* KERNEL_PPE3D_sph + KERNEL_PPE3D_calc_sph: functions_PPE2.cuh:542-698, 868-878 */
static void k_ppe(OracleState* S, double tdt) {
    OSet* o = &S->s;
    const SphdemParams* P = &S->p;
#pragma omp parallel for schedule(dynamic, 64) num_threads(S->nthreads)
    for (int i = 0; i < o->n; i++) {
        if (o->i_type[i] > 2) continue;
        if (P->open_boundary > 0 && o->buffer_type[i] > 0) continue;
        if (o->p_type[i] >= 1000 || o->p_type[i] <= 0) continue;
        double hi = o->h[i], tA = knl_tmpA(P->kernel_type, P->dim, hi), R = P->kappa * hi;
        double xi = o->x[i], yi = o->y[i], zi = o->z[i];
        double uxi = o->ux[i], uyi = o->uy[i], uzi = o->uz[i], rhoi = o->rho[i];
        double pori = o->DEMpor[i], dp = o->dDEMpor[i], dpp = o->dDEMpor_prev[i];
        const double* Cm = o->Cm + (size_t)i * 9;
        int ic, jc, kc;
        cell_ijk(S, xi, yi, zi, &ic, &jc, &kc);
        double bx = 0, by = 0, bz = 0, A = 0, AP = 0;
        FOR_NEIGHBOR_CELLS(S, o, ic, jc, kc, j) {
            if (o->p_type[j] < 1000 && o->i_type[j] != 4) {
                double xj = o->x[j], yj = o->y[j], zj = o->z[j];
                double td = dist3(xi, yi, zi, xj, yj, zj) + 1e-20;
                if (td < R) {
                    double mj = o->m[j], rhoj = o->rho[j], porj = o->DEMpor[j], pj = o->pres[j];
                    double dw = knl_dw(P->kernel_type, tA, hi, td);
                    double tdwx = dw * (xi - xj) / td, tdwy = dw * (yi - yj) / td, tdwz = dw * (zi - zj) / td;
                    kgc_apply(P, Cm, &tdwx, &tdwy, &tdwz);
                    bx += mj / rhoj * (pori * uxi - porj * o->ux[j]) * tdwx;
                    by += mj / rhoj * (pori * uyi - porj * o->uy[j]) * tdwy;
                    bz += mj / rhoj * (pori * uzi - porj * o->uz[j]) * tdwz;
                    double c = -((xi - xj) * tdwx + (yi - yj) * tdwy + (zi - zj) * tdwz) / td / td;
                    A += 1 * mj * ((pori * rhoi + porj * rhoj) / (rhoj * rhoi)) * c;
                    AP += 1 * mj * ((pori * rhoi + porj * rhoj) / (rhoj * rhoi)) * c * pj;
                }
            }
        }
        double bi = P->rho_gas * (bx + by + bz + 2 * dp - dpp) / tdt;
        o->PPE3[i] = bi;
        o->PPE4[i] = AP;
        o->PPE1[i] = rhoi * (bx + by + bz) / tdt;
        o->PPE2[i] = A;
    }
    if (P->ppe_mode != SPHDEM_PPE_REFERENCE) {
        ppe_krylov(S, tdt);
        return;
    }
    for (int i = 0; i < o->n; i++) {
        if (o->i_type[i] > 2) continue;
        if (P->open_boundary > 0 && o->buffer_type[i] > 0) continue;
        if (o->p_type[i] >= 1000 || o->p_type[i] <= 0) continue;
        o->pres[i] = (o->PPE3[i] + o->PPE4[i]) / o->PPE2[i];
    }
}

/* KERNEL_pressureforce3D_sph: functions_PPE2.cuh:2154-2335 */
static void k_pressure_force(OracleState* S) {
    OSet* o = &S->s;
    const SphdemParams* P = &S->p;
#pragma omp parallel for schedule(dynamic, 64) num_threads(S->nthreads)
    for (int i = 0; i < o->n; i++) {
        if (o->i_type[i] > 2) continue;
        if (P->open_boundary > 0 && o->buffer_type[i] > 0) continue;
        if (o->p_type[i] >= 1000 || o->p_type[i] <= 0) continue;
        double hi = o->h[i], tA = knl_tmpA(P->kernel_type, P->dim, hi), R = P->kappa * hi;
        double xi = o->x[i], yi = o->y[i], zi = o->z[i], pi = o->pres[i], rhoi = o->rho[i];
        double pori = o->DEMpor[i];
        const double* Cm = o->Cm + (size_t)i * 9;
        int ic, jc, kc;
        cell_ijk(S, xi, yi, zi, &ic, &jc, &kc);
        double tx = 0, ty = 0, tz = 0;
        FOR_NEIGHBOR_CELLS(S, o, ic, jc, kc, j) {
            double xj = o->x[j], yj = o->y[j], zj = o->z[j];
            if (o->p_type[j] < 1000) {
                double td = dist3(xi, yi, zi, xj, yj, zj) + 1e-20;
                if (td < R) {
                    double dw = knl_dw(P->kernel_type, tA, hi, td);
                    double tdwx = dw * (xi - xj) / td, tdwy = dw * (yi - yj) / td, tdwz = dw * (zi - zj) / td;
                    kgc_apply(P, Cm, &tdwx, &tdwy, &tdwz);
                    if (P->fp_solve) {
                        double Cp = -pori * 1 * o->m[j] * (pi + o->pres[j]) / (rhoi * o->rho[j]);
                        tx += Cp * tdwx;
                        ty += Cp * tdwy;
                        tz += Cp * tdwz;
                    }
                }
            }
        }
        o->fpx[i] = tx;
        o->fpy[i] = ty;
        o->fpz[i] = tz;
    }
}

/* KERNEL_time_update_projection_{sph,dem}: functions_TIME_ISPH2.cuh:467-776 */
static void k_time_update(OracleState* S, OSet* o, double tdt) {
    const SphdemParams* P = &S->p;
    for (int i = 0; i < o->n; i++) {
        if (o->i_type[i] > 2) continue;
        int pt = o->p_type[i], bt = o->buffer_type[i];
        if (pt == 9) {
            /* quirk: MOVING particles write uninitialised xc,yc,zc in the
             * reference (:482-484); the oracle keeps the position. */
        } else {
            double tx0 = o->x[i], ty0 = o->y[i], tz0 = o->z[i];
            double tux0, tuy0, tuz0, ax, ay, az;
            if (pt > 0) {
                tux0 = o->ux[i]; tuy0 = o->uy[i]; tuz0 = o->uz[i];
                ax = o->fpx[i] * (bt == 0) + 0.0 / o->rho[i]; /* fbx = 0 */
                ay = o->fpy[i] * (bt == 0) + 0.0 / o->rho[i];
                az = o->fpz[i] * (bt == 0) + 0.0 / o->rho[i];
            } else {
                tux0 = o->ux0[i]; tuy0 = o->uy0[i]; tuz0 = o->uz0[i];
                ax = ay = az = 0.0;
            }
            double uxc = tux0 + ax * (tdt), uyc = tuy0 + ay * (tdt), uzc = tuz0 + az * (tdt);
            if ((uxc * uxc + uyc * uyc + uzc * uzc) >= P->u_limit * P->u_limit) {
                uxc = tux0; uyc = tuy0; uzc = tuz0;
            }
            double xc = tx0 + (o->ux0[i] + uxc) / 2.0 * (tdt) * (pt > 0) * (o->elix[i]);
            double yc = ty0 + (o->uy0[i] + uyc) / 2.0 * (tdt) * (pt > 0) * (o->eliy[i]);
            double zc = tz0 + (o->uz0[i] + uzc) / 2.0 * (tdt) * (pt > 0) * (o->eliz[i]);
            if (!P->xsph_solve || pt > 1000) {
                o->x[i] = xc; o->y[i] = yc; o->z[i] = zc;
            }
            o->ux[i] = uxc; o->uy[i] = uyc; o->uz[i] = uzc;
        }
        if (P->con_solve == 1 && o->p_type[i] > 0)
            o->temp[i] = o->temp0[i] + o->dtemp[i] * tdt * (o->p_type[i] != -1);
    }
}

/* KERNEL_open_boundary_extrapolation3D_1{,_calc}_sph: functions_BC.cuh:787-984, 1204-1218 */
static void k_open_boundary(OracleState* S) {
    OSet* o = &S->s;
    const SphdemParams* P = &S->p;
    int n = o->n;
    double* nv = (double*)malloc(sizeof(double) * (size_t)n * 7);
#pragma omp parallel for schedule(dynamic, 64) num_threads(S->nthreads)
    for (int i = 0; i < n; i++) {
        if (o->buffer_type[i] <= 0 || o->p_type[i] >= 1000) continue;
        double th = o->h[i], tA = knl_tmpA(P->kernel_type, P->dim, th), R = P->kappa * th;
        double pori = o->DEMpor[i], xi = o->x[i], yi = o->y[i], zi = o->z[i];
        double xg = xi, yg = yi, zg = zi;
        const double* br = bed_row(S, yi);
        const double L2 = br ? br[4] : P->obc_L2, L3 = br ? br[5] : P->obc_L3;
        const double u_in = br ? br[1] : P->inlet_uz_mirror, t_in = br ? br[2] : P->inlet_temp;
        if (o->buffer_type[i] == 1) zg = 2 * L2 - zi;
        else if (o->buffer_type[i] == 2) zg = 2 * L3 - zi;
        int ic, jc, kc;
        cell_ijk(S, xg, yg, zg, &ic, &jc, &kc);
        double trho = 0, tp = 0, tux = 0, tuy = 0, tuz = 0, tt = 0, flt = 0;
        FOR_NEIGHBOR_CELLS(S, o, ic, jc, kc, j) {
            double td = dist3(xg, yg, zg, o->x[j], o->y[j], o->z[j]) + 1e-20;
            if (o->p_type[j] < 1000 && td < R) {
                if (o->p_type[j] == 1 && o->buffer_type[j] == 0) {
                    double w = knl_w(P->kernel_type, tA, th, td);
                    double volj = o->vol[j];
                    trho += o->rho[j] / o->DEMpor[j] * w * volj * 1;
                    tp += volj * o->pres[j] * w * 1;
                    tuz += volj * o->uz[j] * w * 1;
                    tux += volj * o->ux[j] * w * 1;
                    tuy += volj * o->uy[j] * w * 1;
                    tt += volj * o->temp[j] * w * 1;
                    flt += volj * w * 1;
                }
            }
        }
        double* v = nv + (size_t)i * 7; /* pres rho m uz ux uy temp */
        if (P->open_boundary == 1) {
            if (o->buffer_type[i] == 1) {
                v[0] = tp / flt + 0 * (2 * (zi - L2)) * 0.0;
                v[1] = pori * P->rho_gas;
                v[2] = o->rho[i] * o->vol0[i];
                v[3] = u_in * 2 - tuz / flt;
                v[4] = 0 - tux / flt;
                v[5] = 0 - tuy / flt;
                v[6] = t_in;
                if (o->elix[i] < 0.9999 && o->p_type[i] > 0) v[2] = o->rho[i] * o->vol[i];
            } else {
                v[0] = 0.0;
                v[1] = pori * (trho / flt + 0 * (2 * (zi - L3)) * 0.0);
                v[2] = o->rho[i] * o->vol0[i];
                v[3] = tuz / flt + 0 * (2 * (zi - L3)) * 0.0;
                v[4] = tux / flt;
                v[5] = tuy / flt;
                v[6] = tt / flt + 0 * (2 * (zi - L3)) * 0.0;
                if (o->elix[i] < 0.9999 && o->p_type[i] > 0) v[2] = o->rho[i] * o->vol[i];
            }
        }
    }
    if (P->open_boundary == 1) {
        for (int i = 0; i < n; i++) {
            if (o->buffer_type[i] <= 0 || o->p_type[i] >= 1000) continue;
            const double* v = nv + (size_t)i * 7;
            o->pres[i] = v[0]; o->rho[i] = v[1]; o->m[i] = v[2];
            o->uz[i] = v[3]; o->ux[i] = v[4]; o->uy[i] = v[5]; o->temp[i] = v[6];
        }
    }
    free(nv);
}

/* Shared body of the three DEM wall kernels (functions_DEM_BC.cuh:491-718,
 * 1770-2027, 4485-4722): given the contact point, the unit normal and the
 * wall state, apply the rolling/sliding or impulse update. */
static void dem_wall_response(OracleState* S, OSet* d, int i, double nx, double ny, double nz) {
    const SphdemParams* P = &S->p;
    double kdt = P->dt;
    double ux = d->ux[i], uy = d->uy[i], uz = d->uz[i], wx = d->wx[i], wy = d->wy[i], wz = d->wz[i];
    double m = d->m[i], ri = d->ri[i], rad = d->rad[i];
    double ftx = d->ftotalx[i], fty = d->ftotaly[i], ftz = d->ftotalz[i];
    double tqx = d->torqx[i], tqy = d->torqy[i], tqz = d->torqz[i];
    double unm = ux * nx + uy * ny + uz * nz;
    double ucx = ux - rad * (wy * nz - wz * ny), ucy = uy - rad * (wz * nx - wx * nz), ucz = uz - rad * (wx * ny - wy * nx);
    double cwx = -rad * (wy * nz - wz * ny), cwy = -rad * (wz * nx - wx * nz), cwz = -rad * (wx * ny - wy * nx);
    double ucn = ucx * nx + ucy * ny + ucz * nz, cwn = cwx * nx + cwy * ny + cwz * nz;
    double usx = ucx - ucn * nx, usy = ucy - ucn * ny, usz = ucz - ucn * nz;
    double uwx = cwx - cwn * nx, uwy = cwy - cwn * ny, uwz = cwz - cwn * nz;
    if (fabs(usx) < 1e-10) usx = 0.0;
    if (fabs(usy) < 1e-10) usy = 0.0;
    if (fabs(usz) < 1e-10) usz = 0.0;
    if (fabs(uwx) < 1e-10) uwx = 0.0;
    if (fabs(uwy) < 1e-10) uwy = 0.0;
    if (fabs(uwz) < 1e-10) uwz = 0.0;
    double usm = sqrt(usx * usx + usy * usy + usz * usz), uwm = sqrt(uwx * uwx + uwy * uwy + uwz * uwz);
    double sx = usx / (usm + 1e-20), sy = usy / (usm + 1e-20), sz = usz / (usm + 1e-20);
    double swx = uwx / (uwm + 1e-20), swy = uwy / (uwm + 1e-20), swz = uwz / (uwm + 1e-20);
    if (fabs(unm) < (50 * kdt)) {
        double fn = ftx * nx + fty * ny + ftz * nz;
        double ffx = P->wall_mu_s * m * fn * sx, ffy = P->wall_mu_s * m * fn * sy, ffz = P->wall_mu_s * m * fn * sz;
        double frx = P->wall_mu_rs * m * fn * swx, fry = P->wall_mu_rs * m * fn * swy, frz = P->wall_mu_rs * m * fn * swz;
        if (fn > 0.0) { ffx = ffy = ffz = frx = fry = frz = 0.0; }
        ftx += (ffx) / m;
        fty += (ffy) / m;
        ftz += (ffz) / m;
        tqx += -(rad / ri) * (ny * (ffz + frz) - nz * (ffy + fry));
        tqy += -(rad / ri) * (nz * (ffx + frx) - nx * (ffz + frz));
        tqz += -(rad / ri) * (nx * (ffy + fry) - ny * (ffx + frx));
        d->ftotalx[i] = ftx; d->ftotaly[i] = fty; d->ftotalz[i] = ftz;
        d->torqx[i] = tqx; d->torqy[i] = tqy; d->torqz[i] = tqz;
        double uxc = ux + ((ffx) / m) * kdt, uyc = uy + ((ffy) / m) * kdt, uzc = uz + ((ffz) / m) * kdt;
        double ucn2 = uxc * nx + uyc * ny + uzc * nz;
        d->ux[i] = uxc - ucn2 * nx;
        d->uy[i] = uyc - ucn2 * ny;
        d->uz[i] = uzc - ucn2 * nz;
        d->wx[i] = wx - (rad / ri) * (ny * (ffz + frz) - nz * (ffy + fry)) * kdt;
        d->wy[i] = wy - (rad / ri) * (nz * (ffx + frx) - nx * (ffz + frz)) * kdt;
        d->wz[i] = wz - (rad / ri) * (nx * (ffy + fry) - ny * (ffx + frx)) * kdt;
    } else {
        double Jnx = -m * (1 + P->wall_rest_n) * ucn * nx, Jny = -m * (1 + P->wall_rest_n) * ucn * ny,
               Jnz = -m * (1 + P->wall_rest_n) * ucn * nz;
        double Jsx = -1 / ((1 / m) + (rad * rad / ri)) * (1 + P->wall_rest_s) * usm * sx;
        double Jsy = -1 / ((1 / m) + (rad * rad / ri)) * (1 + P->wall_rest_s) * usm * sy;
        double Jsz = -1 / ((1 / m) + (rad * rad / ri)) * (1 + P->wall_rest_s) * usm * sz;
        double Jx = Jnx + Jsx, Jy = Jny + Jsy, Jz = Jnz + Jsz;
        d->ux[i] = ux + (1 / m) * Jx;
        d->uy[i] = uy + (1 / m) * Jy;
        d->uz[i] = uz + (1 / m) * Jz;
        d->wx[i] = wx - (rad / ri) * (ny * Jz - nz * Jy);
        d->wy[i] = wy - (rad / ri) * (nz * Jx - nx * Jz);
        d->wz[i] = wz - (rad / ri) * (nx * Jy - ny * Jx);
    }
}

static void k_dem_walls(OracleState* S) {
    OSet* d = &S->d;
    const SphdemParams* P = &S->p;
    for (int i = 0; i < d->n; i++) {
        if (d->i_type[i] != 1 || d->p_type[i] <= 1000) continue;
        /* KERNEL_treat_DEM_cylinder_z_dem, functions_DEM_BC.cuh:491-718 */
        if (P->dem_wall_mask & 1) {
            double xc = P->cyl_cx, yc = P->cyl_cy, R = P->cyl_r;
            double x = d->x[i], y = d->y[i], z = d->z[i], rad = d->rad[i];
            double F = (x - xc) * (x - xc) + (y - yc) * (y - yc) - (R - rad) * (R - rad);
            if (F > 0) {
                double cpx = xc + (R - rad) * (x - xc) / sqrt((x - xc) * (x - xc) + (y - yc) * (y - yc));
                double cpy = yc + (R - rad) * (y - yc) / sqrt((x - xc) * (x - xc) + (y - yc) * (y - yc));
                double cpz = z;
                d->x[i] = cpx; d->y[i] = cpy; d->z[i] = cpz;
                double nx = -(cpx - xc) / (R - rad), ny = -(cpy - yc) / (R - rad), nz = 0.0;
                double nm = sqrt(nx * nx + ny * ny + nz * nz);
                if (!(nm < 0.5)) dem_wall_response(S, d, i, nx, ny, nz);
            }
        }
        /* KERNEL_treat_DEM_box_z_dem, functions_DEM_BC.cuh:1770-2027 */
        if (P->dem_wall_mask & 2) {
            double xc = P->box_c[0], yc = P->box_c[1], zc = P->box_c[2];
            double Lx = P->box_L[0], Ly = P->box_L[1], Lz = P->box_L[2];
            double x = d->x[i], y = d->y[i], z = d->z[i], rad = d->rad[i];
            double F = fmax(fmax((fabs(x - xc) - (0.5 * Lx - rad)), (fabs(y - yc) - (0.5 * Ly - rad))),
                            (fabs(z - zc) - (0.5 * Lz - rad)));
            if (F > 0) {
                double cpx = xc + fmin((0.5 * Lx - rad), fmax(-(0.5 * Lx - rad), x - xc));
                double cpy = yc + fmin((0.5 * Ly - rad), fmax(-(0.5 * Ly - rad), y - yc));
                double cpz = zc + fmin((0.5 * Lz - rad), fmax(-(0.5 * Lz - rad), z - zc));
                d->x[i] = cpx; d->y[i] = cpy; d->z[i] = cpz;
                double sgx = (cpx - x) / (fabs(cpx - x) + 1e-20);
                double sgy = (cpy - y) / (fabs(cpy - y) + 1e-20);
                double sgz = (cpz - z) / (fabs(cpz - z) + 1e-20);
                if (fabs(cpy - y) < 1e-12) sgy = 0.0;
                if (fabs(cpy - x) < 1e-12) sgx = 0.0; /* quirk: cpy-x typo (:1846) */
                if (fabs(cpz - z) < 1e-12) sgz = 0.0;
                double nn = sqrt(sgx * sgx + sgy * sgy + sgz * sgz) + 1e-20;
                double nx = sgx / nn, ny = sgy / nn, nz = sgz / nn;
                double nm = sqrt(nx * nx + ny * ny + nz * nz);
                if (!(nm < 0.5)) dem_wall_response(S, d, i, nx, ny, nz);
            }
        }
        /* KERNEL_treat_DEM_truncated_cone_z_dem, functions_DEM_BC.cuh:4485-4722 */
        if (P->dem_wall_mask & 4) {
            double xc = P->cone_c[0], yc = P->cone_c[1];
            double r1 = P->cone_r1, r2 = P->cone_r2, hc = P->cone_h;
            double x = d->x[i], y = d->y[i], z = d->z[i], rad = d->rad[i];
            if (!(z <= -hc + rad)) {
                double st = hc / sqrt((r1 - r2) * (r1 - r2) + hc * hc);
                double ct = fabs((r1 - r2)) / sqrt((r1 - r2) * (r1 - r2) + hc * hc);
                double tt = st / ct;
                double rr = r2 + (hc + z) / tt - rad / st;
                double F = (x - xc) * (x - xc) + (y - yc) * (y - yc) - rr * rr;
                if (F > 0) {
                    double cpx = x, cpy = y;
                    double cpz = tt * (sqrt((x - xc) * (x - xc) + (y - yc) * (y - yc)) + rad / st - r2) - hc;
                    d->x[i] = cpx; d->y[i] = cpy; d->z[i] = cpz;
                    double rxy = sqrt((x - xc) * (x - xc) + (y - yc) * (y - yc));
                    double nx = -st * (cpx - xc) / rxy, ny = -st * (cpy - yc) / rxy, nz = ct * 1;
                    dem_wall_response(S, d, i, nx, ny, nz);
                }
            }
        }
    }
}

/* KERNEL_xsph3D_sph + KERNEL_xsph3D_calc_sph: functions_TIME.cuh:1735-1997 */
static void k_xsph(OracleState* S) {
    OSet* o = &S->s;
    const SphdemParams* P = &S->p;
#pragma omp parallel for schedule(dynamic, 64) num_threads(S->nthreads)
    for (int i = 0; i < o->n; i++) {
        if (o->i_type[i] != 1 || o->p_type[i] > 1000) continue;
        int pt = o->p_type[i];
        if (pt == 0 || pt == 9) continue;
        double th = o->h[i], tA = knl_tmpA(P->kernel_type, P->dim, th), R = P->kappa * th;
        double xi = o->x[i], yi = o->y[i], zi = o->z[i], ti = o->temp[i];
        double uxi = o->ux[i], uyi = o->uy[i], uzi = o->uz[i];
        int ic, jc, kc;
        cell_ijk(S, xi, yi, zi, &ic, &jc, &kc);
        double tx = 0, ty = 0, tz = 0, tt = 0, flt = 0;
        FOR_NEIGHBOR_CELLS(S, o, ic, jc, kc, j) {
            int ptj = o->p_type[j];
            if (ptj == 1 || ptj == 3) {
                double td = dist3(xi, yi, zi, o->x[j], o->y[j], o->z[j]);
                if (td < R) {
                    double w = knl_w(P->kernel_type, tA, th, td);
                    double mj = o->m[j], rhoj = o->rho[j];
                    tx += P->c_xsph * mj / rhoj * (-uxi + o->ux[j]) * w;
                    ty += P->c_xsph * mj / rhoj * (-uyi + o->uy[j]) * w;
                    tz += P->c_xsph * mj / rhoj * (-uzi + o->uz[j]) * w;
                    tt += 0.01 * P->c_xsph * mj / rhoj * (o->temp[j] - ti) * w;
                    flt += mj / rhoj * w;
                }
            }
        }
        o->XSPH_ux[i] = (uxi + tx / flt) * (pt > 0);
        o->XSPH_uy[i] = (uyi + ty / flt) * (pt > 0);
        o->XSPH_uz[i] = (uzi + tz / flt) * (pt > 0);
        o->XSPH_temp[i] = (ti + tt / flt) * (pt > 0);
    }
    for (int i = 0; i < o->n; i++) {
        if (o->i_type[i] != 1 || o->p_type[i] > 1000) continue;
        if (o->p_type[i] == 0 || o->p_type[i] == 9) continue;
        o->ux[i] = o->XSPH_ux[i];
        o->uy[i] = o->XSPH_uy[i];
        o->uz[i] = o->XSPH_uz[i];
        o->temp[i] = o->XSPH_temp[i];
    }
}

/* ---------------------------------------------------------------------- */
/* one step: SOPHIA_single_ISPH (ISPH_Calc_seperate.cuh:13-503)            */
/* ---------------------------------------------------------------------- */
/* ---------------------------------------------------------------------- */
/* 2-D WCSPH step (solver_type WCSPH, dim 2): SOPHIA_single               */
/* (WCSPH_Calc.cuh:15-340) in its Lagrangian variant -- ALE flags 1, NNPS  */
/* every step, KERNEL_interaction2D launched -- which the stock driver     */
/* does not run (set_alpha makes SPH Eulerian, NNPS only at count 0,       */
/* interaction2D commented out at WCSPH_Calc.cuh:187).  Viscosity is the   */
/* one constant of viscosity() without property tables (mu_gas), DEM      */
/* porosity is 1.  The 2-D loops are the 27-cell loop on a one-layer grid. */
/* ---------------------------------------------------------------------- */
/* KERNEL_clc_predictor: functions_TIME.cuh:77-228 */
static void w_predictor(OracleState* S) {
    OSet* o = &S->s;
    const SphdemParams* P = &S->p;
    double tdt = P->dt;
    for (int i = 0; i < o->n; i++) {
        if (o->i_type[i] == 3) continue;
        int pt = o->p_type[i], bt = o->buffer_type[i];
        double tx0 = o->x[i], ty0 = o->y[i], tux0 = o->ux[i], tuy0 = o->uy[i];
        if (pt >= 0) {
            o->x[i] = tx0 + tux0 * (tdt * 0.5) * (pt > 0) * 1.0;
            o->y[i] = ty0 + tuy0 * (tdt * 0.5) * (pt > 0) * 1.0;
            o->ux[i] = tux0 + o->ftotalx[i] * (bt == 0) * (tdt * 0.5);
            o->uy[i] = tuy0 + o->ftotaly[i] * (bt == 0) * (tdt * 0.5);
        }
        o->x0[i] = tx0;
        o->y0[i] = ty0;
        o->ux0[i] = tux0;
        o->uy0[i] = tuy0;
        double trho = o->rho[i];
        o->rho0[i] = trho;
        if (P->rho_type == 1 && pt > 0) o->rho[i] = trho + o->drho[i] * (tdt * 0.5);
    }
}

static inline void w_kgc_apply(const SphdemParams* P, const double* Cm, double* dx, double* dy) {
    if (P->kgc_solve != 1) return;
    double a = *dx, b = *dy;
    *dx = Cm[0] * a + Cm[1] * b;
    *dy = Cm[3] * a + Cm[4] * b;
}

/* KERNEL_clc_correction_KGC_2D: functions_PREP2.cuh:73-160 (Cm rows 0,1) */
static void w_kgc2d(OracleState* S) {
    OSet* o = &S->s;
    const SphdemParams* P = &S->p;
#pragma omp parallel for schedule(dynamic, 64) num_threads(S->nthreads)
    for (int i = 0; i < o->n; i++) {
        if (o->i_type[i] > 2 || o->p_type[i] > 1000) continue;
        double h = o->h[i], tA = knl_tmpA(P->kernel_type, 2, h), R = P->kappa * h;
        double xi = o->x[i], yi = o->y[i], zi = o->z[i];
        int ic, jc, kc;
        cell_ijk(S, xi, yi, zi, &ic, &jc, &kc);
        double txx = 0, txy = 0, tyy = 0;
        FOR_NEIGHBOR_CELLS(S, o, ic, jc, kc, j) {
            if (o->p_type[j] > 1000) continue;
            double xj = o->x[j], yj = o->y[j];
            double td = dist3(xi, yi, zi, xj, yj, o->z[j]);
            if (td > 0 && td < R) {
                double dw = knl_dw(P->kernel_type, tA, h, td);
                double mtd = o->m[j] * dw, rtd = 1.0 / (o->rho[j] * td), t;
                t = -mtd * (xi - xj) * (xi - xj); t *= rtd; txx += t;
                t = -mtd * (yi - yj) * (xi - xj); t *= rtd; txy += t;
                t = -mtd * (yi - yj) * (yi - yj); t *= rtd; tyy += t;
            }
        }
        double* Cm = o->Cm + (size_t)i * 9;
        double det = txx * tyy - txy * txy;
        if (fabs(det) > 1e-4) {
            double r = 1.0 / det;
            Cm[0] = tyy * r; Cm[1] = -txy * r; Cm[3] = -txy * r; Cm[4] = txx * r;
        } else {
            Cm[0] = 1; Cm[1] = 0; Cm[3] = 0; Cm[4] = 1;
        }
    }
}

/* KERNEL_clc_prep2D: functions_PREP2.cuh:1247-1420 (no SPS, no surface tension) */
static void w_prep2d(OracleState* S) {
    OSet* o = &S->s;
    const SphdemParams* P = &S->p;
    int filt = (S->count % P->freq_filt) == 0, anto = P->delSPH_solve == 2;
#pragma omp parallel for schedule(dynamic, 64) num_threads(S->nthreads)
    for (int i = 0; i < o->n; i++) {
        if (o->i_type[i] > 2 || o->p_type[i] > 1000) continue;
        double h = o->h[i], tA = knl_tmpA(P->kernel_type, 2, h), R = P->kappa * h;
        double xi = o->x[i], yi = o->y[i], zi = o->z[i], rhoi = o->rho[i], mi = o->m[i];
        int ic, jc, kc;
        cell_ijk(S, xi, yi, zi, &ic, &jc, &kc);
        double flt = 0, gx = 0, gy = 0;
        FOR_NEIGHBOR_CELLS(S, o, ic, jc, kc, j) {
            if (o->p_type[j] > 1000) continue;
            double xj = o->x[j], yj = o->y[j];
            double td = dist3(xi, yi, zi, xj, yj, o->z[j]) + 1e-20;
            if (td < R) {
                double w = knl_w(P->kernel_type, tA, h, td), dw = knl_dw(P->kernel_type, tA, h, td);
                double tx = dw * (xi - xj) / td, ty = dw * (yi - yj) / td;
                double mj = o->m[j], rhoj = o->rho[j];
                if (filt) flt += mj / rhoj * w;
                if (anto) {
                    w_kgc_apply(P, o->Cm + (size_t)i * 9, &tx, &ty);
                    gx += -(rhoj - rhoi) * (mj / rhoj) * tx;
                    gy += -(rhoj - rhoi) * (mj / rhoj) * ty;
                }
            }
        }
        o->rho_ref[i] = mi / ((h / 1.600) * (h / 1.600));
        if (filt) o->flt_s[i] = flt;
        if (anto) {
            o->grad_rhox[i] = gx;
            o->grad_rhoy[i] = gy;
        }
    }
}

/* KERNEL_clc_continuity_norm2D: functions_MASS.cuh:670-769 */
static void w_continuity2d(OracleState* S) {
    OSet* o = &S->s;
    const SphdemParams* P = &S->p;
    int anto = P->delSPH_solve == 2;
#pragma omp parallel for schedule(dynamic, 64) num_threads(S->nthreads)
    for (int i = 0; i < o->n; i++) {
        if (o->i_type[i] > 2 || o->p_type[i] > 1000) continue;
        int pti = o->p_type[i];
        double h = o->h[i], tA = knl_tmpA(P->kernel_type, 2, h), R = P->kappa * h;
        double xi = o->x[i], yi = o->y[i], zi = o->z[i];
        double uxi = o->ux[i] * (pti > 0), uyi = o->uy[i] * (pti > 0), rhoi = o->rho[i];
        double gxi = o->grad_rhox[i], gyi = o->grad_rhoy[i];
        int ic, jc, kc;
        cell_ijk(S, xi, yi, zi, &ic, &jc, &kc);
        double tx = 0, ty = 0, tr = 0;
        FOR_NEIGHBOR_CELLS(S, o, ic, jc, kc, j) {
            if (o->p_type[j] > 1000) continue;
            double xj = o->x[j], yj = o->y[j];
            double td = dist3(xi, yi, zi, xj, yj, o->z[j]) + 1e-20;
            if (td < R) {
                int ptj = o->p_type[j];
                double dw = knl_dw(P->kernel_type, tA, h, td);
                double mj = o->m[j], rhoj = o->rho[j];
                double uxj = o->ux[j] * (ptj > 0), uyj = o->uy[j] * (ptj > 0);
                double gx = dw * (xi - xj) / td, gy = dw * (yi - yj) / td;
                if (P->kgc_solve > 0) w_kgc_apply(P, o->Cm + (size_t)i * 9, &gx, &gy);
                double tm = mj * (rhoi / rhoj);
                tx += (uxi - uxj) * tm * gx;
                ty += (uyi - uyj) * tm * gy;
                if (P->delSPH_solve > 0) {
                    double phi = (gxi + o->grad_rhox[j]) * (xj - xi);
                    phi += (gyi + o->grad_rhoy[j]) * (yj - yi);
                    phi = (-0.5 * phi) * anto + (rhoj - rhoi);
                    double t = -2 * (P->delta_sph * 1.0) * h * P->soundspeed * (mj / rhoj);
                    t *= phi * dw / td;
                    tr += t;
                }
            }
        }
        o->drho[i] = (tx + ty) * (rhoi / o->rho_ref[i]) + tr * (P->delSPH_solve > 0);
    }
}

/* KERNEL_EOS: functions_PROP.cuh:7-28 */
static void w_eos(OracleState* S) {
    OSet* o = &S->s;
    const SphdemParams* P = &S->p;
    double tB = P->soundspeed * P->soundspeed * (1.186) / P->gamma;
    for (int i = 0; i < o->n; i++) {
        if (o->i_type[i] > 2 || o->p_type[i] > 1000 || o->buffer_type[i] != 0) continue;
        double tP = pow(o->rho[i] / o->rho_ref[i], P->gamma);
        o->pres[i] = tB * (tP - 1.0);
    }
}

/* KERNEL_interaction2D: functions_INTERACTION.cuh:64-410 (i_type 1) */
static void w_interaction2d(OracleState* S) {
    OSet* o = &S->s;
    const SphdemParams* P = &S->p;
#pragma omp parallel for schedule(dynamic, 64) num_threads(S->nthreads)
    for (int i = 0; i < o->n; i++) {
        if (o->i_type[i] != 1 || o->p_type[i] > 1000) continue;
        double h = o->h[i], tA = knl_tmpA(P->kernel_type, 2, h), R = P->kappa * h;
        double xi = o->x[i], yi = o->y[i], zi = o->z[i];
        double uxi = o->ux[i], uyi = o->uy[i], pi = o->pres[i], mi = o->m[i], rhoi = o->rho[i];
        double pori = 1.0, vis = P->mu_gas;
        int ic, jc, kc;
        cell_ijk(S, xi, yi, zi, &ic, &jc, &kc);
        double tx = 0, ty = 0, pgx = 0, pgy = 0;
        FOR_NEIGHBOR_CELLS(S, o, ic, jc, kc, j) {
            if (o->p_type[j] > 1000) continue;
            double xj = o->x[j], yj = o->y[j];
            double td = dist3(xi, yi, zi, xj, yj, o->z[j]) + 1e-20;
            if (td < R) {
                double dw = knl_dw(P->kernel_type, tA, h, td);
                double gx = dw * (xi - xj) / td, gy = dw * (yi - yj) / td;
                if (P->kgc_solve > 0) w_kgc_apply(P, o->Cm + (size_t)i * 9, &gx, &gy);
                double uxj = o->ux[j], uyj = o->uy[j], mj = o->m[j], rhoj = o->rho[j], pj = o->pres[j];
                double hj = o->h[j], porj = 1.0;
                if (P->fp_solve) {
                    double Cp = -mj * (pi + pj) / (pori * rhoi * porj * rhoj);
                    double px = Cp * gx, py = Cp * gy;
                    tx += px;
                    ty += py;
                    pgx += rhoi * pori * px;
                    pgy += rhoi * pori * py;
                }
                if (P->fv_solve) {
                    double Cv = (xi - xj) * gx + (yi - yj) * gy;
                    Cv *= 4 * (mj / (rhoi * rhoj));
                    Cv *= (vis * vis) / (vis + vis);
                    Cv /= td;
                    Cv /= td;
                    tx += Cv * (uxi - uxj);
                    ty += Cv * (uyi - uyj);
                }
                if (P->fva_solve) {
                    double uij = (uxi - uxj) * (xi - xj) + (uyi - uyj) * (yi - yj);
                    if (uij < 0) {
                        double hij = (h + hj) * 0.5;
                        double phi = hij * uij;
                        phi /= (td * td + 0.01 * hij * hij);
                        double Pij = mi * phi * (-P->art_visc_alpha * P->soundspeed + P->art_visc_beta * phi);
                        Pij /= (rhoi + rhoj);
                        Pij *= 0.5;
                        tx += -Pij * gx;
                        ty += -Pij * gy;
                    }
                }
            }
        }
        if (P->fg_solve) ty += -P->g_sph;
        o->ftotalx[i] = tx;
        o->ftotaly[i] = ty;
        o->ftotal[i] = sqrt(tx * tx + ty * ty);
        o->pgf_x[i] = pgx;
        o->pgf_y[i] = pgy;
    }
}

/* KERNEL_time_update_single (functions_TIME.cuh:676-880) and KERNEL_xsph2D
 * (functions_TIME.cuh:1520-1605): the corrector writes TP1 (new velocity,
 * density; positions when XSPH is off), XSPH reads the corrected velocity
 * and the predicted positions and density. */
static void w_correct_xsph(OracleState* S) {
    OSet* o = &S->s;
    const SphdemParams* P = &S->p;
    int n = o->n;
    double tdt = P->dt;
    if (n <= 0) return;
    double* xn = (double*)malloc(sizeof(double) * (size_t)(n ? n : 1));
    double* yn = (double*)malloc(sizeof(double) * (size_t)(n ? n : 1));
    double* rn = (double*)malloc(sizeof(double) * (size_t)(n ? n : 1));
    double* un = (double*)malloc(sizeof(double) * (size_t)(n ? n : 1));
    double* vn = (double*)malloc(sizeof(double) * (size_t)(n ? n : 1));
    for (int i = 0; i < n; i++) {
        xn[i] = o->x[i];
        yn[i] = o->y[i];
        rn[i] = o->rho[i];
        un[i] = o->ux[i];
        vn[i] = o->uy[i];
        if (o->i_type[i] == 3) continue;
        int pt = o->p_type[i], bt = o->buffer_type[i];
        double tux0 = o->ux0[i], tuy0 = o->uy0[i], ax = 0, ay = 0;
        if (pt > 0) {
            ax = o->ftotalx[i] * (bt == 0);
            ay = o->ftotaly[i] * (bt == 0);
        }
        double uxc = tux0 + ax * tdt, uyc = tuy0 + ay * tdt;
        if ((uxc * uxc + uyc * uyc) >= P->u_limit * P->u_limit) {
            uxc = tux0;
            uyc = tuy0;
        }
        if (!P->xsph_solve) {
            xn[i] = o->x0[i] + uxc * tdt * (pt > 0) * 1.0;
            yn[i] = o->y0[i] + uyc * tdt * (pt > 0) * 1.0;
        }
        un[i] = uxc;
        vn[i] = uyc;
        if (P->rho_type == 1 && pt > 0) rn[i] = o->rho0[i] + o->drho[i] * tdt;
    }
    if (P->xsph_solve) {
#pragma omp parallel for schedule(dynamic, 64) num_threads(S->nthreads)
        for (int i = 0; i < n; i++) {
            if (o->i_type[i] != 1 || o->p_type[i] > 1000) continue;
            int pt = o->p_type[i];
            double h = o->h[i], tA = knl_tmpA(P->kernel_type, 2, h), R = P->kappa * h;
            double xi = o->x[i], yi = o->y[i], zi = o->z[i], uxi = un[i], uyi = vn[i], flt = o->flt_s[i];
            int ic, jc, kc;
            cell_ijk(S, xi, yi, zi, &ic, &jc, &kc);
            double tx = 0, ty = 0;
            FOR_NEIGHBOR_CELLS(S, o, ic, jc, kc, j) {
                if (o->p_type[j] > 1000) continue;
                double xj = o->x[j], yj = o->y[j];
                double td = dist3(xi, yi, zi, xj, yj, o->z[j]);
                if (td < R) {
                    double w = knl_w(P->kernel_type, tA, h, td);
                    double mj = o->m[j], rhoj = o->rho[j];
                    tx += P->c_xsph * mj / rhoj * (-uxi + un[j]) * w / flt;
                    ty += P->c_xsph * mj / rhoj * (-uyi + vn[j]) * w / flt;
                }
            }
            xn[i] = o->x0[i] + (uxi + tx) * tdt * (pt > 0);
            yn[i] = o->y0[i] + (uyi + ty) * tdt * (pt > 0);
        }
    }
    memcpy(o->x, xn, sizeof(double) * (size_t)n);
    memcpy(o->y, yn, sizeof(double) * (size_t)n);
    memcpy(o->rho, rn, sizeof(double) * (size_t)n);
    memcpy(o->ux, un, sizeof(double) * (size_t)n);
    memcpy(o->uy, vn, sizeof(double) * (size_t)n);
    free(xn); free(yn); free(rn); free(un); free(vn);
}

static void oracle_wcsph2d_step(OracleState* S) {
    w_predictor(S);
    nnps(S, &S->s);   /* every step; P3 (forces, drho) zeroed after the predictor */
    build_sph_list(S);
    if (S->p.kgc_solve == 1 || S->p.delSPH_solve == 2) w_kgc2d(S);
    w_prep2d(S);
    w_continuity2d(S);
    w_eos(S);
    w_interaction2d(S);
    w_correct_xsph(S);
}

static void oracle_one_step(OracleState* S) {
    const SphdemParams* P = &S->p;
    int sph_turn = (S->count % P->decouple_stride) == 0;
    double sdt = P->decouple_stride * P->dt;
    if (sph_turn) k_set_alpha(&S->s);
    k_set_alpha(&S->d);
    if (sph_turn) nnps(S, &S->s);
    nnps(S, &S->d);
    if (sph_turn) build_sph_list(S);
    if (sph_turn) k_mass_init(S);   /* dim 3 in the reference; the 2-D model runs it too */
    if (sph_turn && P->kgc_solve > 0) k_kgc(S);
    if (sph_turn) k_coupling_prep_sph(S);
    k_coupling_prep_dem(S);
    if (sph_turn) k_prep_sph(S);
    if (sph_turn) k_prep3d_sph(S);
    if (sph_turn) k_advection(S);
    k_dem_contact(S);
    k_dem_coupling(S);
    if (sph_turn) k_sph_coupling(S);
    if (P->time_type == 1) {
        if (sph_turn) k_projection(S, &S->s, sdt);
        k_projection(S, &S->d, P->dt);
    }
    if (S->count == 0 && sph_turn) k_neumann(S);
    if (sph_turn) k_ppe(S, sdt);
    if (sph_turn) k_neumann(S);
    if (sph_turn) k_pressure_force(S);
    /* the DEM history written by the contact kernel becomes the state */
    {
        OSet* d = &S->d;
        double* t = d->ct_idx; d->ct_idx = d->ct_idx_new; d->ct_idx_new = t;
        t = d->del_s; d->del_s = d->del_s_new; d->del_s_new = t;
    }
    if (sph_turn) k_time_update(S, &S->s, sdt);
    k_time_update(S, &S->d, P->dt);
    if (P->open_boundary > 0 && sph_turn) k_open_boundary(S);
    k_dem_walls(S);
    if (P->xsph_solve && sph_turn) k_xsph(S);
}

/* ---------------------------------------------------------------------- */
/* API                                                                     */
/* ---------------------------------------------------------------------- */
OracleState* oracle_create(const SphdemParams* p, int n_sph, int n_dem) {
    OracleState* S = (OracleState*)calloc(1, sizeof(OracleState));
    if (!S) return NULL;
    S->p = *p;
    S->nthreads = 1;
    if (oset_alloc(&S->s, n_sph) || oset_alloc(&S->d, n_dem)) {
        oracle_destroy(S);
        return NULL;
    }
    S->time = p->time;
    S->count = (int)floor(p->time / p->dt + 0.5); /* ISPH_Calc_seperate.cuh:522 */
    return S;
}

void oracle_destroy(OracleState* s) {
    if (!s) return;
    oset_free(&s->s);
    oset_free(&s->d);
    free(s->nb_cnt);
    free(s->nb_list);
    free(s->beds);
    free(s);
}

static double* dfield(OSet* o, int f) {
    switch (f) {
    case SPHDEM_F_X: return o->x; case SPHDEM_F_Y: return o->y; case SPHDEM_F_Z: return o->z;
    case SPHDEM_F_UX: return o->ux; case SPHDEM_F_UY: return o->uy; case SPHDEM_F_UZ: return o->uz;
    case SPHDEM_F_WX: return o->wx; case SPHDEM_F_WY: return o->wy; case SPHDEM_F_WZ: return o->wz;
    case SPHDEM_F_M: return o->m; case SPHDEM_F_RHO: return o->rho; case SPHDEM_F_PRES: return o->pres;
    case SPHDEM_F_TEMP: return o->temp; case SPHDEM_F_H: return o->h; case SPHDEM_F_RAD: return o->rad;
    case SPHDEM_F_RI: return o->ri; case SPHDEM_F_DEMPOR: return o->DEMpor; case SPHDEM_F_DDEMPOR: return o->dDEMpor;
    case SPHDEM_F_FLT_S: return o->flt_s; case SPHDEM_F_FLT_SD: return o->flt_sd; case SPHDEM_F_FLT_SD2: return o->flt_sd_2;
    case SPHDEM_F_FTOTALX: return o->ftotalx; case SPHDEM_F_FTOTALY: return o->ftotaly; case SPHDEM_F_FTOTALZ: return o->ftotalz;
    case SPHDEM_F_FPX: return o->fpx; case SPHDEM_F_FPY: return o->fpy; case SPHDEM_F_FPZ: return o->fpz;
    case SPHDEM_F_PGFX: return o->pgf_x; case SPHDEM_F_PGFY: return o->pgf_y; case SPHDEM_F_PGFZ: return o->pgf_z;
    case SPHDEM_F_FDX_DF: return o->Fdx_df; case SPHDEM_F_FDY_DF: return o->Fdy_df; case SPHDEM_F_FDZ_DF: return o->Fdz_df;
    case SPHDEM_F_TORQX: return o->torqx; case SPHDEM_F_TORQY: return o->torqy; case SPHDEM_F_TORQZ: return o->torqz;
    case SPHDEM_F_RHO_REF: return o->rho_ref; case SPHDEM_F_TEMP1: return o->temp1; case SPHDEM_F_TEMP2: return o->temp2;
    case SPHDEM_F_TEMP3: return o->temp3; case SPHDEM_F_DTEMP: return o->dtemp; case SPHDEM_F_Q_SD: return o->Q_sd;
    case SPHDEM_F_FTOTAL: return o->ftotal; case SPHDEM_F_DRHO: return o->drho;
    case SPHDEM_F_GRAD_RHOX: return o->grad_rhox; case SPHDEM_F_GRAD_RHOY: return o->grad_rhoy;
    case SPHDEM_F_VIS_T: return o->vis_t;
    default: return NULL;
    }
}
static int* ifield(OSet* o, int f) {
    switch (f) {
    case SPHDEM_F_PTYPE: return o->p_type; case SPHDEM_F_ITYPE: return o->i_type;
    case SPHDEM_F_BUFFER_TYPE: return o->buffer_type; case SPHDEM_F_DEM_IDX: return o->dem_idx;
    case SPHDEM_F_PID: return o->pid; case SPHDEM_F_CELL: return o->g_idx;
    default: return NULL;
    }
}

int oracle_set_field(OracleState* s, int which, int field, const void* src, int n) {
    if (!s || !src) return SPHDEM_E_ARG;
    OSet* o = which ? &s->d : &s->s;
    if (n != o->n) return SPHDEM_E_ARG;
    double* d = dfield(o, field);
    if (d) { memcpy(d, src, sizeof(double) * (size_t)n); return 0; }
    int* ip = ifield(o, field);
    if (ip) { memcpy(ip, src, sizeof(int) * (size_t)n); return 0; }
    return SPHDEM_E_ARG;
}

int oracle_get_field(OracleState* s, int which, int field, void* dst, int n) {
    if (!s || !dst) return SPHDEM_E_ARG;
    OSet* o = which ? &s->d : &s->s;
    if (n != o->n) return SPHDEM_E_ARG;
    double* d = dfield(o, field);
    if (d) { memcpy(dst, d, sizeof(double) * (size_t)n); return 0; }
    int* ip = ifield(o, field);
    if (ip) { memcpy(dst, ip, sizeof(int) * (size_t)n); return 0; }
    return SPHDEM_E_ARG;
}

int oracle_set_beds(OracleState* s, int nbeds, const double* rows7) {
    if (!s || nbeds < 1 || !rows7) return SPHDEM_E_ARG;
    free(s->beds);
    s->beds = (double*)malloc(sizeof(double) * 7 * (size_t)nbeds);
    if (!s->beds) return SPHDEM_E_NOMEM;
    memcpy(s->beds, rows7, sizeof(double) * 7 * (size_t)nbeds);
    s->nbeds = nbeds;
    return 0;
}

int oracle_set_domain(OracleState* s, const double* mins, const double* maxs, double h0) {
    s->xmin = mins[0]; s->ymin = mins[1]; s->zmin = mins[2];
    s->xmax = maxs[0]; s->ymax = maxs[1]; s->zmax = maxs[2];
    s->h0 = h0;
    s->domain_fixed = 1;
    return 0;
}

/* find_minmax (function_init.cuh:913-950, quirk: the loop stops one row
 * short of num_part) on the input rows in file order: SPH rows then DEM
 * rows is the caller's convention for synthetic beds. */
int oracle_commit(OracleState* S) {
    const SphdemParams* P = &S->p;
    int ns = S->s.n, nd = S->d.n, n = ns + nd;
    if (n == 0) return SPHDEM_E_ARG;
    if (!S->domain_fixed) {
#define GETX(k, F) ((k) < ns ? S->s.F[(k)] : S->d.F[(k)-ns])
        double mnx = GETX(0, x), mxx = mnx, mny = GETX(0, y), mxy = mny, mnz = GETX(0, z), mxz = mnz;
        for (int k = 0; k < n - 1; k++) {
            double tx = GETX(k, x), ty = GETX(k, y), tz = GETX(k, z);
            if (tx < mnx) mnx = tx; if (tx > mxx) mxx = tx;
            if (ty < mny) mny = ty; if (ty > mxy) mxy = ty;
            if (tz < mnz) mnz = tz; if (tz > mxz) mxz = tz;
        }
        mnx -= (mxx - mnx) * P->margin[0]; mxx += (mxx - mnx) * P->margin[1];
        mny -= (mxy - mny) * P->margin[2]; mxy += (mxy - mny) * P->margin[3];
        mnz -= (mxz - mnz) * P->margin[4]; mxz += (mxz - mnz) * P->margin[5];
        S->xmin = mnx; S->xmax = mxx; S->ymin = mny; S->ymax = mxy; S->zmin = mnz; S->zmax = mxz;
        S->h0 = GETX(0, h);
#undef GETX
    }
    /* ISPH.cuh:104-113 */
    S->dcell = 1.1 * P->kappa * S->h0;
    S->NI = (int)((S->xmax - S->xmin) / S->dcell) + 1;
    S->NJ = (int)((S->ymax - S->ymin) / S->dcell) + 1;
    S->NK = (int)((S->zmax - S->zmin) / S->dcell) + 1;
    S->num_cells = S->NI * S->NJ * S->NK + 1;
    S->s.g_str = (int*)calloc((size_t)S->num_cells + 1, sizeof(int));
    S->s.g_end = (int*)calloc((size_t)S->num_cells + 1, sizeof(int));
    S->d.g_str = (int*)calloc((size_t)S->num_cells + 1, sizeof(int));
    S->d.g_end = (int*)calloc((size_t)S->num_cells + 1, sizeof(int));
    /* c_initial_inner_outer_particle_single_{sph,dem}: functions_NNPS.cuh:60-200 */
    OSet* sets[2] = {&S->s, &S->d};
    for (int q = 0; q < 2; q++) {
        OSet* o = sets[q];
        for (int i = 0; i < o->n; i++) {
            o->i_type[i] = 1;
            o->buffer_type[i] = 0;
            if (P->open_boundary > 0 && o->p_type[i] < 1000 && o->p_type[i] >= 1) {
                const double* br = bed_row(S, o->y[i]);
                double L1 = br ? br[3] : P->obc_L1, L2 = br ? br[4] : P->obc_L2;
                double L3 = br ? br[5] : P->obc_L3, L4 = br ? br[6] : P->obc_L4;
                if (o->z[i] >= (L1 - 1e-6) && (o->z[i] < L2 - 1e-6)) { o->buffer_type[i] = 1; o->i_type[i] = 2; }
                if (o->z[i] >= (L3 - 1e-6) && (o->z[i] < L4 - 1e-6)) { o->buffer_type[i] = 2; o->i_type[i] = 2; }
            }
        }
    }
    S->nb_cap = 512;
    S->nb_cnt = (int*)calloc((size_t)(ns ? ns : 1), sizeof(int));
    S->nb_list = (int*)calloc((size_t)(ns ? ns : 1) * S->nb_cap, sizeof(int));
    S->committed = 1;
    return 0;
}

int oracle_step(OracleState* s, int nsteps) {
    if (!s || !s->committed) return SPHDEM_E_ARG;
    for (int k = 0; k < nsteps; k++) {
        if (s->p.solver_type == SPHDEM_WCSPH) oracle_wcsph2d_step(s);
        else oracle_one_step(s);
        s->time += s->p.dt; /* ISPH_Calc_seperate.cuh:924-925 */
        s->count++;
    }
    return 0;
}

int oracle_get_neighbors(OracleState* s, int* counts, int* dst, int cap) {
    int n = s->s.n;
    for (int i = 0; i < n; i++) {
        counts[i] = s->nb_cnt[i];
        int c = s->nb_cnt[i] < cap ? s->nb_cnt[i] : cap;
        c = c < s->nb_cap ? c : s->nb_cap;
        for (int k = 0; k < c; k++) dst[(size_t)i * cap + k] = s->nb_list[(size_t)i * s->nb_cap + k];
    }
    return 0;
}

int oracle_get_grid(OracleState* s, int* nijk, double* bbox6, double* dcell) {
    nijk[0] = s->NI; nijk[1] = s->NJ; nijk[2] = s->NK;
    bbox6[0] = s->xmin; bbox6[1] = s->xmax; bbox6[2] = s->ymin;
    bbox6[3] = s->ymax; bbox6[4] = s->zmin; bbox6[5] = s->zmax;
    *dcell = s->dcell;
    return 0;
}

int oracle_get_time(OracleState* s, double* time, int* count) {
    *time = s->time;
    *count = s->count;
    return 0;
}

int oracle_get_history(OracleState* s, double* ct, double* ds, int n) {
    if (n != s->d.n) return SPHDEM_E_ARG;
    memcpy(ct, s->d.ct_idx, sizeof(double) * (size_t)n * NSLOT);
    memcpy(ds, s->d.del_s, sizeof(double) * (size_t)n * NSLOT * 3);
    return 0;
}

int oracle_set_history(OracleState* s, const double* ct, const double* ds, int n) {
    if (n != s->d.n) return SPHDEM_E_ARG;
    memcpy(s->d.ct_idx, ct, sizeof(double) * (size_t)n * NSLOT);
    memcpy(s->d.del_s, ds, sizeof(double) * (size_t)n * NSLOT * 3);
    return 0;
}

int oracle_get_ppe(OracleState* s, int* iters, double* rel_res, int* status) {
    if (!s) return -1;
    if (iters) *iters = s->ppe_iters;
    if (rel_res) *rel_res = s->ppe_res;
    if (status) *status = s->ppe_status;
    return 0;
}

int oracle_set_threads(OracleState* s, int nthreads) {
    s->nthreads = nthreads > 0 ? nthreads : 1;
    return 0;
}

double oracle_kernel(int kt, int dim, double h, double r, int deriv) {
    double tA = knl_tmpA(kt, dim, h);
    return deriv ? knl_dw(kt, tA, h, r) : knl_w(kt, tA, h, r);
}
