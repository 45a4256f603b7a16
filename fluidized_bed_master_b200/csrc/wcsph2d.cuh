// wcsph2d.cuh -- the 2-D weakly compressible SPH step (solver_type WCSPH,
// dim 2): the reference's SOPHIA_single (WCSPH_Calc.cuh:15-340) for a
// Lagrangian fluid, in its kernel order:
//
//   k_w_predictor   KERNEL_clc_predictor (functions_TIME.cuh:77-228), with
//                   the NNPS cell key of the predicted position
//   NNPS            stable sort / gather every step
//   k_w_list        neighbour list (kappa h_i, 9-cell stencil)
//   k_w_kgc         KERNEL_clc_correction_KGC_2D (functions_PREP2.cuh:73-160)
//   k_w_prep        KERNEL_clc_prep2D (functions_PREP2.cuh:1247-1420):
//                   reference density, Shepard filter, density gradient
//   k_w_continuity  KERNEL_clc_continuity_norm2D (functions_MASS.cuh:670-769)
//                   and KERNEL_EOS (functions_PROP.cuh:7-28) in its epilogue
//   k_w_interaction KERNEL_interaction2D (functions_INTERACTION.cuh:64-410)
//   k_w_corrector   KERNEL_time_update_single (functions_TIME.cuh:676-880)
//   k_w_xsph        KERNEL_xsph2D (functions_TIME.cuh:1520-1605)
//   k_w_finish      (XSPH on) corrected positions and density become the state
//
// The reference's stock 2-D driver cannot run a moving fluid: it sets the
// ALE flags to Eulerian (KERNEL_set_alpha, functions_ALE.cuh:2-20), runs
// NNPS only at count 0 (WCSPH_Calc.cuh:34) and has KERNEL_interaction2D
// commented out (WCSPH_Calc.cuh:187).  This step is the Lagrangian variant
// of that driver (ALE flags 1, NNPS every step, interaction2D launched),
// which is also what the oracle and the reference harness run.
//
// Precision: the FP32 build keeps positions, density, its predictor start
// value, mass and reference density in FP64 and evaluates the EOS in FP64.
// The Tait pressure is B ((rho/rho_ref)^gamma - 1) with rho/rho_ref - 1 of
// order 1e-3, so one FP32 rounding of rho, m or rho_ref (6e-8) alone would
// move p by 1e-4 of itself; the neighbour sums (forces, drho, filters)
// stay FP32.  Density differences are taken in FP64 before the cast.
//
// Properties as in the reference without property tables: viscosity() is
// one constant for every p_type (VISCOSITY_AIR, functions_PROP.cuh:228-245;
// here mu_gas); DEM porosity is 1 (no DEM particles in this mode);
// artificial viscosity alpha/beta and the delta-SPH coefficient are
// parameters whose reference-compat values are the hard-wired 0.1, 0.02,
// 0.1 (Parameters.cuh:83-96).  z is 0 for every particle, so the 3-D grid
// has one z-layer and its 9-cell stencil is the reference's 2-D loop
// (y outer, x inner).
#pragma once
#include "engine.cuh"

namespace sphdem {

template <typename R>
struct WState {      // persistent, ping-pong, permuted by the cell gather
    double *x, *y, *z, *h, *m, *rho;
    R *ux, *uy, *pres, *temp, *flt_s;
    double *x0, *y0, *rho0;      // predictor start positions and density (part2::x0, y0, rho0)
    R *ux0, *uy0;                // predictor start velocity
    int *ptype, *btype, *itype, *pid;
    // batch of beds (sphdem_create_batch): the bed of each particle and the
    // placement shift of every bed.  Cells are computed at x + shift, so the
    // beds lie in separate cells of one grid; positions and every pair
    // distance stay in the bed's own coordinates.  nullptr: one bed, no shift.
    int* bed;
    const double2* boff;
};

// shift of the cell computation of particle i (zero outside a batch)
template <typename R>
__device__ __forceinline__ double2 w_cell_off(const WState<R>& S, int i) {
    return S.boff ? S.boff[S.bed[i]] : make_double2(0.0, 0.0);
}

template <typename R>
struct WWork {
    R *ftx, *fty, *ftot, *drho;  // last step's values (read by the predictor in the old order)
    double* rho_ref;
    R *grx, *gry, *pgfx, *pgfy;
    R* Cm;                       // 4*n, Cm[q*n+i] = (00, 01, 10, 11)
    double *xn, *yn;             // corrected positions
    double* rhon;                // corrected density
    int *key_in, *key_out, *val_in, *val_out, *g_str, *g_end, *nbr, *ncnt;
    int4* rows;
};

struct WParams {
    double alpha, beta, delta;   // artificial viscosity, delta-SPH
    int freq_filt, delsph, rho_cont;
    double gamma, eos_B;         // Tait: p = B ((rho/rho_ref)^gamma - 1), B = c0^2 1.186/gamma
};

__device__ __forceinline__ double w_dist(double xi, double yi, double xj, double yj) {
    double dx = __dsub_rn(xi, xj), dy = __dsub_rn(yi, yj);
    return __dsqrt_rn(__dadd_rn(__dmul_rn(dx, dx), __dmul_rn(dy, dy)));
}

// KERNEL_clc_predictor, Lagrangian (ALE flags 1), no MOVING particles,
// fused with the NNPS cell key of the predicted position
// (KERNEL_index_particle_to_cell, functions_NNPS.cuh:732-760): key[i],
// i_type 3 -> num_cells; the cell-sort count (cell_count) is fused in
template <typename R>
__device__ __forceinline__ int w_predict(const DevParams& P, const WParams& Q, WState<R>& S, WWork<R>& W, int i);

template <typename R>
__global__ void k_w_predictor(DevParams P, WParams Q, WState<R> S, WWork<R> W, int* key, int* cnt) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    int k = -1;
    if (i < P.ns) {
        k = (S.itype[i] == 3) ? P.num_cells : w_predict<R>(P, Q, S, W, i);
        key[i] = k;
    }
    cell_count(cnt, k);
}

// predictor of slot i (i_type != 3); returns the cell key of the predicted position
template <typename R>
__device__ __forceinline__ int w_predict(const DevParams& P, const WParams& Q, WState<R>& S, WWork<R>& W, int i) {
    int pt = S.ptype[i], bt = S.btype[i];
    double x0 = S.x[i], y0 = S.y[i];
    R ux0 = S.ux[i], uy0 = S.uy[i];
    double hdt = P.dt * 0.5;
    double xp = x0, yp = y0;
    if (pt >= 0) {
        xp = x0 + (double)ux0 * hdt * (double)(pt > 0);
        yp = y0 + (double)uy0 * hdt * (double)(pt > 0);
        S.x[i] = xp;
        S.y[i] = yp;
        R b = (R)(bt == 0);
        S.ux[i] = ux0 + W.ftx[i] * b * (R)hdt;
        S.uy[i] = uy0 + W.fty[i] * b * (R)hdt;
    }
    S.x0[i] = x0;
    S.y0[i] = y0;
    S.ux0[i] = ux0;
    S.uy0[i] = uy0;
    double rho = S.rho[i];
    S.rho0[i] = rho;
    if (Q.rho_cont && pt > 0) S.rho[i] = rho + (double)W.drho[i] * hdt;
    int ic, jc, kc;
    const double2 o = w_cell_off(S, i);
    cell_ijk(P, xp + o.x, yp + o.y, S.z[i], ic, jc, kc);
    return ic + P.NI * jc + P.NI * P.NJ * kc;
}

// ---- lanes per particle ------------------------------------------------
// The gathers run L lanes per particle (L = 1, 2, 4, 8, 16; a group of L
// consecutive threads of one warp).  Lane l takes list entries l, l+L, ...
// and the group adds its partial sums with a fixed xor tree, so a given L
// gives bit-identical results run to run.  The list build visits candidate
// slots in ascending order L at a time and compacts the hits with a ballot
// in that order, so the list is the same for every L.
template <int L>
struct Grp {
    int i, lane;
    unsigned mask;   // the group's lanes in the warp
    int base;        // the group's first lane in the warp
    __device__ __forceinline__ Grp() {
        int t = blockIdx.x * blockDim.x + threadIdx.x;
        i = t / L;
        lane = threadIdx.x % L;
        base = (threadIdx.x & 31) & ~(L - 1);
        mask = (L == 32 ? 0xffffffffu : ((1u << L) - 1u)) << base;
    }
    template <typename T>
    __device__ __forceinline__ T sum(T v) const {
#pragma unroll
        for (int o = L / 2; o > 0; o >>= 1) v += __shfl_xor_sync(mask, v, o);
        return v;
    }
};

// neighbour list: sqrt(dx^2+dy^2) + 1e-20 < kappa h_i, FP64, exact
template <typename R, int L>
__global__ void __launch_bounds__(128) k_w_list(DevParams P, WState<R> S, const int4* __restrict__ rows, int* nbr,
                                                int* ncnt, DevFlags* F) {
    const Grp<L> g;
    const int i = g.i;
    if (i >= P.ns) return;   // the whole group
    double xi = S.x[i], yi = S.y[i];
    double Rr = __dmul_rn(P.kappa, S.h[i]);
    int ic, jc, kc;
    const double2 o = w_cell_off(S, i);
    cell_ijk(P, xi + o.x, yi + o.y, 0.0, ic, jc, kc);
    int c = 0, cap = P.nb_cap, n = P.ns;
    const Cull cu = make_cull(xi + o.x, yi + o.y, 0.0, Rr);
    const unsigned low = (1u << g.lane) - 1u;
    for_rows(P, ic, jc, kc, rows, cu, [&](int a, int b) {
        for (int j0 = a; j0 < b; j0 += L) {
            const int j = j0 + g.lane;
            bool hit = false;
            if (j < b && S.ptype[j] <= 1000) hit = __dadd_rn(w_dist(xi, yi, S.x[j], S.y[j]), 1e-20) < Rr;
            unsigned grp = (__ballot_sync(g.mask, hit) & g.mask) >> g.base;
            if (hit) {
                int pos = c + __popc(grp & low);
                if (nbr && pos < cap) nbr[(size_t)pos * n + i] = j;
            }
            c += __popc(grp);
        }
    });
    if (g.lane == 0) {
        ncnt[i] = c;
        if (c > cap) atomicOr(&F->overflow, 1);
        atomicMax(&F->max_ncnt, c);
    }
}

template <typename R>
__device__ __forceinline__ void w_pair(double xi, double yi, double xj, double yj, R& dx, R& dy, R& r) {
    double d = w_dist(xi, yi, xj, yj);
    dx = (R)(xi - xj);
    dy = (R)(yi - yj);
    r = (R)d;
}

// gradient correction (KGC) of a kernel gradient
template <typename R>
__device__ __forceinline__ void w_kgc(const R* __restrict__ Cm, int n, int i, R& gx, R& gy) {
    R a = gx, b = gy;
    gx = Cm[0 * n + i] * a + Cm[1 * n + i] * b;
    gy = Cm[2 * n + i] * a + Cm[3 * n + i] * b;
}

// KERNEL_clc_correction_KGC_2D
template <typename R, int L>
__global__ void __launch_bounds__(128) k_w_kgc(DevParams P, WState<R> S, WWork<R> W) {
    const Grp<L> g;
    const int i = g.i, n = P.ns;
    if (i >= n || S.itype[i] > 2 || S.ptype[i] > 1000) return;
    double xi = S.x[i], yi = S.y[i];
    R th = (R)S.h[i], tA = knl_tmpA<R>(P.kernel_type, 2, th);
    int cnt = min(W.ncnt[i], P.nb_cap);
    R txx = 0, txy = 0, tyy = 0;
    for (int k = g.lane; k < cnt; k += L) {
        int j = W.nbr[(size_t)k * n + i];
        R dx, dy, r;
        w_pair<R>(xi, yi, S.x[j], S.y[j], dx, dy, r);
        if (!(r > (R)0)) continue;
        R dw = knl_dw<R>(P.kernel_type, tA, th, r);
        R mtd = (R)S.m[j] * dw, rtd = (R)1 / ((R)S.rho[j] * r), t;
        t = -mtd * dx * dx; t *= rtd; txx += t;
        t = -mtd * dy * dx; t *= rtd; txy += t;
        t = -mtd * dy * dy; t *= rtd; tyy += t;
    }
    txx = g.sum(txx);
    txy = g.sum(txy);
    tyy = g.sum(tyy);
    if (g.lane) return;
    R det = txx * tyy - txy * txy;
    R c00 = 1, c01 = 0, c10 = 0, c11 = 1;
    if (fabs(det) > (R)1e-4) {
        R rr = (R)1 / det;
        c00 = tyy * rr;
        c01 = -txy * rr;
        c10 = -txy * rr;
        c11 = txx * rr;
    }
    W.Cm[0 * n + i] = c00;
    W.Cm[1 * n + i] = c01;
    W.Cm[2 * n + i] = c10;
    W.Cm[3 * n + i] = c11;
}

// KERNEL_clc_prep2D: reference density, Shepard filter (every freq_filt
// steps), density gradient for Antuono's delta-SPH (corrected when KGC)
template <typename R, int L>
__global__ void __launch_bounds__(128) k_w_prep(DevParams P, WParams Q, WState<R> S, WWork<R> W,
                                                const DevFlags* F) {
    const Grp<L> g;
    const int i = g.i, n = P.ns;
    if (i >= n || S.itype[i] > 2 || S.ptype[i] > 1000) return;
    const int count = F->step_count;   // the host loop's count (vii[43])
    double xi = S.x[i], yi = S.y[i];
    R th = (R)S.h[i], tA = knl_tmpA<R>(P.kernel_type, 2, th);
    const double rhoi = S.rho[i];
    const bool filt = (count % Q.freq_filt) == 0, anto = Q.delsph == 2, kgc = P.kgc == 1;
    int cnt = min(W.ncnt[i], P.nb_cap);
    R flt = 0, gx = 0, gy = 0;
    for (int k = g.lane; k < cnt; k += L) {
        int j = W.nbr[(size_t)k * n + i];
        R dx, dy, r;
        w_pair<R>(xi, yi, S.x[j], S.y[j], dx, dy, r);
        r += (R)1e-20;
        R w = knl_w<R>(P.kernel_type, tA, th, r), dw = knl_dw<R>(P.kernel_type, tA, th, r);
        R mj = (R)S.m[j], rhoj = (R)S.rho[j];
        if (filt) flt += mj / rhoj * w;
        if (anto) {
            R tx = dw * dx / r, ty = dw * dy / r;
            if (kgc) w_kgc<R>(W.Cm, n, i, tx, ty);
            R dr = (R)(S.rho[j] - rhoi);
            gx += -dr * (mj / rhoj) * tx;
            gy += -dr * (mj / rhoj) * ty;
        }
    }
    flt = g.sum(flt);
    gx = g.sum(gx);
    gy = g.sum(gy);
    if (g.lane) return;
    double v = S.h[i] / 1.6;
    W.rho_ref[i] = S.m[i] / (v * v);
    if (filt) S.flt_s[i] = flt;
    if (anto) {
        W.grx[i] = gx;
        W.gry[i] = gy;
    }
}

// KERNEL_clc_continuity_norm2D
template <typename R, int L>
__global__ void __launch_bounds__(128) k_w_continuity(DevParams P, WParams Q, WState<R> S, WWork<R> W) {
    const Grp<L> g;
    const int i = g.i, n = P.ns;
    if (i >= n || S.itype[i] > 2 || S.ptype[i] > 1000) return;
    int pti = S.ptype[i];
    double xi = S.x[i], yi = S.y[i];
    R th = (R)S.h[i], tA = knl_tmpA<R>(P.kernel_type, 2, th);
    R uxi = S.ux[i] * (R)(pti > 0), uyi = S.uy[i] * (R)(pti > 0);
    const double rhoi_d = S.rho[i];
    R rhoi = (R)rhoi_d;
    R gxi = W.grx[i], gyi = W.gry[i];
    const bool kgc = P.kgc == 1, anto = Q.delsph == 2;
    int cnt = min(W.ncnt[i], P.nb_cap);
    R tx = 0, ty = 0, tr = 0;
    for (int k = g.lane; k < cnt; k += L) {
        int j = W.nbr[(size_t)k * n + i];
        R dx, dy, r;
        w_pair<R>(xi, yi, S.x[j], S.y[j], dx, dy, r);
        r += (R)1e-20;
        int ptj = S.ptype[j];
        R dw = knl_dw<R>(P.kernel_type, tA, th, r);
        R mj = (R)S.m[j], rhoj = (R)S.rho[j];
        R uxj = S.ux[j] * (R)(ptj > 0), uyj = S.uy[j] * (R)(ptj > 0);
        R gx = dw * dx / r, gy = dw * dy / r;
        if (kgc) w_kgc<R>(W.Cm, n, i, gx, gy);
        R tm = mj * (rhoi / rhoj);
        tx += (uxi - uxj) * tm * gx;
        ty += (uyi - uyj) * tm * gy;
        if (Q.delsph > 0) {
            R phi = (gxi + W.grx[j]) * (-dx) + (gyi + W.gry[j]) * (-dy);
            phi = ((R)-0.5 * phi) * (R)anto + (R)(S.rho[j] - rhoi_d);
            R t = (R)-2 * ((R)Q.delta * (R)1.0) * th * (R)P.soundspeed * (mj / rhoj);
            t *= phi * dw / r;
            tr += t;
        }
    }
    tx = g.sum(tx);
    ty = g.sum(ty);
    tr = g.sum(tr);
    if (g.lane) return;
    W.drho[i] = (tx + ty) * (R)(rhoi_d / W.rho_ref[i]) + tr * (R)(Q.delsph > 0);
    // KERNEL_EOS (functions_PROP.cuh:7-28), Tait, for the same rows with
    // buffer_type 0: it reads only row i's density and reference density,
    // and nothing in this pass reads a pressure
    if (S.btype[i] == 0) {
        double tP = pow(rhoi_d / W.rho_ref[i], Q.gamma);
        S.pres[i] = (R)(Q.eos_B * (tP - 1.0));
    }
}

// KERNEL_interaction2D (i_type 1): pressure, viscous and artificial-viscosity
// forces and gravity along -y
template <typename R, int L>
__global__ void __launch_bounds__(128) k_w_interaction(DevParams P, WParams Q, WState<R> S, WWork<R> W) {
    const Grp<L> g;
    const int i = g.i, n = P.ns;
    if (i >= n || S.itype[i] != 1 || S.ptype[i] > 1000) return;
    double xi = S.x[i], yi = S.y[i];
    R th = (R)S.h[i], tA = knl_tmpA<R>(P.kernel_type, 2, th);
    R uxi = S.ux[i], uyi = S.uy[i], pi = S.pres[i], mi = (R)S.m[i], rhoi = (R)S.rho[i];
    const R pori = 1, porj = 1;
    const R vis = (R)P.mu_gas;
    const bool kgc = P.kgc == 1;
    int cnt = min(W.ncnt[i], P.nb_cap);
    R tx = 0, ty = 0, pgx = 0, pgy = 0;
    for (int k = g.lane; k < cnt; k += L) {
        int j = W.nbr[(size_t)k * n + i];
        R dx, dy, r;
        w_pair<R>(xi, yi, S.x[j], S.y[j], dx, dy, r);
        r += (R)1e-20;
        R dw = knl_dw<R>(P.kernel_type, tA, th, r);
        R gx = dw * dx / r, gy = dw * dy / r;
        if (kgc) w_kgc<R>(W.Cm, n, i, gx, gy);
        R uxj = S.ux[j], uyj = S.uy[j], mj = (R)S.m[j], rhoj = (R)S.rho[j], pj = S.pres[j];
        if (P.fp) {
            R Cp = -mj * (pi + pj) / (pori * rhoi * porj * rhoj);
            R px = Cp * gx, py = Cp * gy;
            tx += px;
            ty += py;
            pgx += rhoi * pori * px;
            pgy += rhoi * pori * py;
        }
        if (P.fv) {
            R Cv = dx * gx + dy * gy;
            Cv *= (R)4 * (mj / (rhoi * rhoj));
            Cv *= (vis * vis) / (vis + vis);
            Cv /= r;
            Cv /= r;
            tx += Cv * (uxi - uxj);
            ty += Cv * (uyi - uyj);
        }
        if (P.fva) {
            R uij = (uxi - uxj) * dx + (uyi - uyj) * dy;
            if (uij < (R)0) {
                R hij = (th + (R)S.h[j]) * (R)0.5;
                R phi = hij * uij;
                phi /= (r * r + (R)0.01 * hij * hij);
                R Pij = mi * phi * (-(R)Q.alpha * (R)P.soundspeed + (R)Q.beta * phi);
                Pij /= (rhoi + rhoj);
                Pij *= (R)0.5;
                tx += -Pij * gx;
                ty += -Pij * gy;
            }
        }
    }
    tx = g.sum(tx);
    ty = g.sum(ty);
    pgx = g.sum(pgx);
    pgy = g.sum(pgy);
    if (g.lane) return;
    if (P.fg) ty += -(R)P.g_sph;
    W.ftx[i] = tx;
    W.fty[i] = ty;
    W.ftot[i] = sqrt(tx * tx + ty * ty);
    W.pgfx[i] = pgx;
    W.pgfy[i] = pgy;
}

// KERNEL_time_update_single (velocity, density; positions when XSPH is off).
// Without XSPH no later pass reads the predicted positions and density, so
// the corrected ones go straight into the state; with XSPH they wait in
// xn, yn, rhon for k_w_finish.  Thread 0 also advances the device step
// counter (read by the next step's prep).
template <typename R>
__global__ void k_w_corrector(DevParams P, WParams Q, WState<R> S, WWork<R> W, DevFlags* F) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i == 0) F->step_count += 1;
    if (i >= P.ns) return;
    const bool direct = !P.xsph;
    if (!direct) {
        W.xn[i] = S.x[i];
        W.yn[i] = S.y[i];
        W.rhon[i] = S.rho[i];
    }
    if (S.itype[i] == 3) return;
    int pt = S.ptype[i], bt = S.btype[i];
    R ux0 = S.ux0[i], uy0 = S.uy0[i], ax = 0, ay = 0;
    if (pt > 0) {
        R b = (R)(bt == 0);
        ax = W.ftx[i] * b;
        ay = W.fty[i] * b;
    }
    R dt = (R)P.dt;
    R uxc = ux0 + ax * dt, uyc = uy0 + ay * dt;
    R lim = (R)P.u_limit;
    if ((uxc * uxc + uyc * uyc) >= lim * lim) {
        uxc = ux0;
        uyc = uy0;
    }
    if (direct) {
        S.x[i] = S.x0[i] + (double)uxc * P.dt * (double)(pt > 0);
        S.y[i] = S.y0[i] + (double)uyc * P.dt * (double)(pt > 0);
    }
    S.ux[i] = uxc;
    S.uy[i] = uyc;
    if (Q.rho_cont && pt > 0) {
        double rn = S.rho0[i] + (double)W.drho[i] * P.dt;
        if (direct) S.rho[i] = rn;
        else W.rhon[i] = rn;
    }
}

// KERNEL_xsph2D: positions from the corrected velocity plus the XSPH term
// (neighbours' corrected velocity, predicted positions and density)
template <typename R, int L>
__global__ void __launch_bounds__(128) k_w_xsph(DevParams P, WState<R> S, WWork<R> W) {
    const Grp<L> g;
    const int i = g.i, n = P.ns;
    if (i >= n || S.itype[i] != 1 || S.ptype[i] > 1000) return;
    int pt = S.ptype[i];
    double xi = S.x[i], yi = S.y[i];
    R th = (R)S.h[i], tA = knl_tmpA<R>(P.kernel_type, 2, th);
    R uxi = S.ux[i], uyi = S.uy[i], flt = S.flt_s[i];
    R c = (R)P.c_xsph;
    int cnt = min(W.ncnt[i], P.nb_cap);
    R tx = 0, ty = 0;
    for (int k = g.lane; k < cnt; k += L) {
        int j = W.nbr[(size_t)k * n + i];
        R dx, dy, r;
        w_pair<R>(xi, yi, S.x[j], S.y[j], dx, dy, r);
        R w = knl_w<R>(P.kernel_type, tA, th, r);
        R mj = (R)S.m[j], rhoj = (R)S.rho[j];
        tx += c * mj / rhoj * (-uxi + S.ux[j]) * w / flt;
        ty += c * mj / rhoj * (-uyi + S.uy[j]) * w / flt;
    }
    tx = g.sum(tx);
    ty = g.sum(ty);
    if (g.lane) return;
    W.xn[i] = S.x0[i] + ((double)uxi + (double)tx) * P.dt * (double)(pt > 0);
    W.yn[i] = S.y0[i] + ((double)uyi + (double)ty) * P.dt * (double)(pt > 0);
}

template <typename R>
__global__ void k_w_finish(DevParams P, WState<R> S, WWork<R> W) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= P.ns) return;
    S.x[i] = W.xn[i];
    S.y[i] = W.yn[i];
    S.rho[i] = W.rhon[i];
}

// cell gather of the WCSPH state
template <typename R>
__global__ void k_w_gather(DevParams P, WState<R> src, WState<R> dst, const int* __restrict__ perm) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    int n = P.ns;
    if (i >= n) return;
    int p = perm[i];
    dst.x[i] = src.x[p]; dst.y[i] = src.y[p]; dst.z[i] = src.z[p]; dst.h[i] = src.h[p];
    dst.ux[i] = src.ux[p]; dst.uy[i] = src.uy[p]; dst.m[i] = src.m[p]; dst.rho[i] = src.rho[p];
    dst.pres[i] = src.pres[p]; dst.temp[i] = src.temp[p]; dst.flt_s[i] = src.flt_s[p];
    dst.x0[i] = src.x0[p]; dst.y0[i] = src.y0[p];
    dst.ux0[i] = src.ux0[p]; dst.uy0[i] = src.uy0[p]; dst.rho0[i] = src.rho0[p];
    dst.ptype[i] = src.ptype[p]; dst.btype[i] = src.btype[p]; dst.itype[i] = src.itype[p]; dst.pid[i] = src.pid[p];
    if (src.bed) dst.bed[i] = src.bed[p];
}

// cell key of the state as it stands (the first NNPS at commit; in a step
// the predictor writes the keys): KERNEL_index_particle_to_cell
template <typename R>
__global__ void k_w_hash(DevParams P, WState<R> S, int* key, int* cnt) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    int k = -1;
    if (i < P.ns) {
        if (S.itype[i] == 3) {
            k = P.num_cells;
        } else {
            int ic, jc, kc;
            const double2 o = w_cell_off(S, i);
            cell_ijk(P, S.x[i] + o.x, S.y[i] + o.y, S.z[i], ic, jc, kc);
            k = ic + P.NI * jc + P.NI * P.NJ * kc;
        }
        key[i] = k;
    }
    cell_count(cnt, k);
}

}  // namespace sphdem
