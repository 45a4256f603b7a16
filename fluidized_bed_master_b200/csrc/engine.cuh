// engine.cuh -- device state of one SPH-DEM engine handle.
//
// Layout in HBM (structure of arrays, one array per field, cell-sorted):
//   positions, smoothing length and DEM radius: double
//   the DEM set (state and work arrays): double in both builds -- it is
//     small (spheres are ~6 % of the particles), and its stiff contacts
//     amplify rounding in the tangential and angular terms
//   every other field: R (float in the FP32 build, double in the FP64 one);
//     the SPH temperature is stored as T - DevParams::t_ref
//   DEM contact history: SPHDEM_NSLOT slot-major planes, partner id int32
//     and tangential spring double[3]  (slot s of particle i at s*n+i)
//   packed records of what the neighbour passes read of a neighbour
//     (records.cuh): position + tag, {m,rho}, {m',rho',T,eps}, {u,p}, {u,T}
// Persistent fields live in two copies (A/B) that the per-step reorder
// gathers between; work arrays are single copies overwritten each step.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>
#include "cell_sort.cuh"
#include "device_common.cuh"
#include "records.cuh"

namespace sphdem {

template <typename R>
struct SphState {
    double *x, *y, *z, *h;
    R *ux, *uy, *uz, *m, *rho, *pres, *temp, *dDEMpor, *flt_s;
    R* dpres;    // pressure change of the last PPE solve (learned warm start feature)
    int *ptype, *btype, *itype, *pid;
};

template <typename R>
struct DemState {
    double *x, *y, *z, *h, *rad;
    R *ux, *uy, *uz, *wx, *wy, *wz, *m, *rho, *ri, *temp, *temp1, *temp2, *temp3;
    R *Fdx_df, *Fdy_df, *Fdz_df, *Q_sd;
    int *ptype, *btype, *itype, *pid, *dem_idx;
    int* hid;      // NSLOT*n
    double* hds;   // NSLOT*3*n
};

// packed neighbour records (records.cuh), indexed by the current slot
template <typename R>
struct SphRec {
    PosRec<R>* pos;
    V2<R>* mr0;
    V4<R>* f1;
    V4<R>* up;
    V4<R>* ut;
};

template <typename R>
struct SphWork {
    R *m_new, *rho_new, *rho_ref, *DEMpor, *dDEMpor_prev;
    R* Cm;                       // 9*n, row-major per particle plane: Cm[k*n+i]
    R *ftx, *fty, *ftz, *ftot;
    R *fpx, *fpy, *fpz;
    R *pgfx, *pgfy, *pgfz;
    R *dtemp, *temp0;
    R* vist;                     // SPS eddy viscosity (k_sps), read by pass B
    R *ux0, *uy0, *uz0;
    R *p_new;
    R *u_tmpx, *u_tmpy, *u_tmpz, *temp_tmp;
    int *key_in, *key_out, *val_in, *val_out;
    int *g_str, *g_end;
    int4* rows;                  // per-cell stencil rows (for_rows)
    int *nbr, *ncnt;
    int *nbrd, *ncntd;           // SPH -> DEM list (k_build_dlist): nbrd[k*n+i], exact count
    int *wall_idx, *buf_idx, *counters;   // per-step compacted wall / buffer slots
    SphRec<R> rec;
};

template <typename R>
struct DemWork {
    R *flt_s, *flt_sd, *flt_sd2, *DEMpor;
    R *ftx, *fty, *ftz, *tqx, *tqy, *tqz;
    R *dtemp, *dtemp1, *dtemp2, *dtemp3;
    R *Fdx_b, *Fdy_b, *Fdz_b, *Fdx_da, *Fdy_da, *Fdz_da;
    R *ux0, *uy0, *uz0, *temp0;
    R *magf;                     // |u_f - u_a| of the drag closure (VTK mag_uijf)
    int *key_in, *key_out, *val_in, *val_out;
    int *g_str, *g_end;
    int4* rows;
    int *nbs, *ncs;              // SPH neighbours of each sphere (k_dem_prep): nbs[i*DEM_SPH_CAP+k], exact count
    R* dcs;                      // 14*n pair sums of k_dem_coupling for k_dem_finish (DcSums, plane-major)
    int* dcf;                    // n: bit0 coupled, bit1 fluid seen, bit2 air seen; -1 not reached
};
constexpr int DEM_SPH_CAP = 256;

// device-side status words (checked by the host at sync points)
struct DevFlags {
    int overflow;   // bit0 SPH neighbour list, bit1 DEM contact history
    int nan;
    int max_ncnt;
    int step_count; // the reference's count (vii[43]), advanced by k_tick at the end of a step
    int max_ncntd;  // largest SPH -> DEM list count seen
};

template <typename R>
struct Engine {
    DevParams P;
    SphState<R> S[2];    // ping-pong; cur = S[cur_s]
    DemState<double> D[2];   // the DEM set is FP64 in both builds (see DevParams)
    int cur_s, cur_d;
    SphWork<R> sw;
    DemWork<double> dw;
    DevFlags* flags;
    CellSort cs_s, cs_d; // NNPS sort by cell of the SPH and DEM sets
    double* red_buf;     // reductions for stats
};

}  // namespace sphdem
