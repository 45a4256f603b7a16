// device_common.cuh -- device-side helpers shared by the step kernels.
//
// Smoothing kernels, cell hashing and the FP64 pair-distance test.  The
// distance and cell arithmetic are written with explicit round-to-nearest
// intrinsics so that no FMA contraction happens: neighbour sets and cell
// indices then agree bit for bit with a plain IEEE evaluation of
//   sqrt((xi-xj)*(xi-xj)+(yi-yj)*(yi-yj)+(zi-zj)*(zi-zj))
//   min(floor((x-xmin)/(xmax-xmin)*NI), NI-1), clamped at 0
// (functions_NNPS.cuh:774-784, e.g. functions_PPE2.cuh:629).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#define SPHDEM_NSLOT 16

namespace sphdem {

// Constants that travel with every launch.  Copied from SphdemParams plus
// the grid computed at commit time.
struct DevParams {
    int kernel_type, dim, kgc, delsph, fp, fv, fva, fg, con, xsph, open_bc, rho_type;
    int iface, fb;            // interface sharpness force, repulsive boundary force (pass B)
    int sps;                  // fv_solve with the SPS turbulence model: eddy viscosity (k_sps)
    int ipf;                  // surface tension, inter-particle force model (fs_solve, surf_model 1)
    double c_repulsive;       // vif[14], strength of the repulsive boundary force
    int NI, NJ, NK, num_cells;
    int ns, nd, nb_cap;
    int nbd_cap;              // SPH -> DEM list entries per particle
    int nwall, nbuf;
    int filt_period;          // freq_filt * decouple_stride
    int wall_mask;
    int sph_lagrangian;
    double kappa, dt, sdt, soundspeed, u_limit, c_xsph;
    double xmin, xmax, ymin, ymax, zmin, zmax;
    double rho_gas, rho_liquid, mu_gas, mu_liquid, nu_gas, g_sph, g_dem, h_over_dx;
    double k_sph, cp_sph, k_dem, cp_dem;
    double G, nu_p, damp, fric, r_contact, r_search;
    double inlet_uz, inlet_temp, L2, L3, ball_vel;
    // 2-D beds in planes y = const (sphdem_set_beds): nbeds rows of
    // {y, inlet_uz, inlet_temp, L2, L3}, sorted by y; 0 = the values above
    int nbeds;
    const double* beds;
    // The SPH temperature is stored as T - t_ref (t_ref: the mean initial SPH
    // temperature, an FP32 value): in the FP32 build a temperature near
    // 300 K keeps increments of 1e-4 K per step only as an offset, and the
    // pair sums read differences of neighbours' temperatures.  Kernels that
    // need the absolute temperature add t_ref; the C ABI converts.
    double t_ref;
    double cyl_cx, cyl_cy, cyl_r;
    double box_c[3], box_L[3];
    double cone_c[3], cone_r1, cone_r2, cone_h;
    double rest_n, rest_s, mu_s, mu_rs;
    // fixed-point positions of the FP32 build (records.cuh): origin, 1/step
    // and step per axis; q_abs = 8 x the largest step, which sets the width
    // of the band a prefilter leaves to the exact FP64 test.
    double q_org[3], q_inv[3], q_abs;
    float q_step[3];
};

// The open-boundary parameters of the bed whose plane is nearest y.
constexpr int BED_COLS = 5;
struct BedObc {
    double inlet_uz, inlet_temp, L2, L3;
};
__device__ __forceinline__ BedObc bed_obc(const DevParams& P, double y) {
    if (P.nbeds <= 0) return BedObc{P.inlet_uz, P.inlet_temp, P.L2, P.L3};
    int lo = 0, hi = P.nbeds - 1;   // the last row with plane <= y, or row 0
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (P.beds[mid * BED_COLS] <= y) lo = mid;
        else hi = mid - 1;
    }
    if (lo + 1 < P.nbeds && fabs(P.beds[(lo + 1) * BED_COLS] - y) < fabs(P.beds[lo * BED_COLS] - y)) lo++;
    const double* r = P.beds + lo * BED_COLS;
    return BedObc{r[1], r[2], r[3], r[4]};
}

// ---- cell index ---------------------------------------------------------
__device__ __forceinline__ int cell_coord(double v, double vmin, double vmax, int N) {
    if (vmax == vmin) return 0;
    double f = floor(__dmul_rn(__ddiv_rn(__dsub_rn(v, vmin), __dsub_rn(vmax, vmin)), (double)N));
    double r = (f < (double)(N - 1)) ? f : (double)(N - 1);
    int c = (int)r;
    return c < 0 ? 0 : c;
}

__device__ __forceinline__ void cell_ijk(const DevParams& P, double x, double y, double z, int& ic, int& jc, int& kc) {
    ic = cell_coord(x, P.xmin, P.xmax, P.NI);
    jc = cell_coord(y, P.ymin, P.ymax, P.NJ);
    kc = cell_coord(z, P.zmin, P.zmax, P.NK);
}

// reference predicate distance, no contraction
__device__ __forceinline__ double pair_dist(double xi, double yi, double zi, double xj, double yj, double zj) {
    double dx = __dsub_rn(xi, xj), dy = __dsub_rn(yi, yj), dz = __dsub_rn(zi, zj);
    double d2 = __dadd_rn(__dadd_rn(__dmul_rn(dx, dx), __dmul_rn(dy, dy)), __dmul_rn(dz, dz));
    return __dsqrt_rn(d2);
}

// ---- smoothing kernels (functions_KNL.cuh:2-144) -----------------------
// Wendland normalisations use the literal constants of the reference.
template <typename R>
__device__ __forceinline__ R knl_tmpA(int kt, int dim, R tH) {
    const R PI_REF = (R)3.141592653;
    if (dim == 3) {
        switch (kt) {
        case 0: return (R)1.0 / (pow(PI_REF, (R)1.5) * tH * tH * tH);
        case 1: return (R)3.0 / ((R)359.0 * PI_REF * tH * tH * tH);
        case 2: return (R)315.0 / ((R)208.0 * PI_REF * tH * tH * tH);
        case 3: return (R)3.342253804929802 / ((R)8 * tH * tH * tH);
        case 4: return (R)4.923856051905513 / ((R)8 * tH * tH * tH);
        case 5: return (R)6.788953041263660 / ((R)8 * tH * tH * tH);
        }
    } else {
        switch (kt) {
        case 0: return (R)1.0 / (PI_REF * tH * tH);
        case 1: return (R)7.0 / ((R)478.0 * PI_REF * tH * tH);
        case 2: return (R)15.0 / ((R)7.0 * PI_REF * tH * tH);
        case 3: return (R)2.228169203286535 / ((R)4 * tH * tH);
        case 4: return (R)2.864788975654116 / ((R)4 * tH * tH);
        case 5: return (R)3.546881588905096 / ((R)4 * tH * tH);
        }
    }
    return (R)0;
}

template <typename R>
__device__ __forceinline__ R ipow(R b, int e) {
    R r = (R)1;
    for (int k = 0; k < e; k++) r *= b;
    return r;
}

template <typename R>
__device__ __forceinline__ R knl_w(int kt, R tA, R tH, R rr) {
    R tR;
    switch (kt) {
    case 5: {
        tR = rr / tH * (R)0.5;
        if (!(tR < (R)1)) return (R)0;
        R a = (R)1 - tR, a2 = a * a, a4 = a2 * a2;
        return tA * a4 * a4 * ((R)1 + (R)8 * tR + (R)25 * tR * tR + (R)32 * tR * tR * tR);
    }
    case 3: {
        tR = rr / tH * (R)0.5;
        if (!(tR < (R)1)) return (R)0;
        R a = (R)1 - tR, a2 = a * a;
        return tA * a2 * a2 * ((R)1 + (R)4 * tR);
    }
    case 4: {
        tR = rr / tH * (R)0.5;
        if (!(tR < (R)1)) return (R)0;
        R a = (R)1 - tR, a3 = a * a * a;
        return tA * a3 * a3 * ((R)1 + (R)6 * tR + (R)11.666666666666666 * tR * tR);
    }
    case 0:
        tR = rr / tH;
        return tA * exp(-tR * tR);
    case 1:
        tR = rr / tH;
        if (tR < (R)1) return tA * (ipow((R)3 - tR, 5) - (R)6 * ipow((R)2 - tR, 5) + (R)15 * ipow((R)1 - tR, 5));
        if (tR < (R)2) return tA * (ipow((R)3 - tR, 5) - (R)6 * ipow((R)2 - tR, 5));
        if (tR < (R)3) return tA * ipow((R)3 - tR, 5);
        return (R)0;
    case 2:
        tR = rr / tH;
        if (!(tR < (R)2)) return (R)0;
        return tA * ((R)2 / (R)3 - (R)9 / (R)8 * tR * tR + (R)19 / (R)24 * tR * tR * tR - (R)5 / (R)32 * tR * tR * tR * tR);
    }
    return (R)0;
}

// dW/dr
template <typename R>
__device__ __forceinline__ R knl_dw(int kt, R tA, R tH, R rr) {
    R tR;
    switch (kt) {
    case 5: {
        tR = rr / tH * (R)0.5;
        if (!(tR < (R)1)) return (R)0;
        R a = (R)1 - tR, a2 = a * a, a4 = a2 * a2;
        return ((R)1 / ((R)2 * tH)) * tA * ((R)-22 * tR * a4 * a2 * a * ((R)16 * tR * tR + (R)7 * tR + (R)1));
    }
    case 3: {
        tR = rr / tH * (R)0.5;
        if (!(tR < (R)1)) return (R)0;
        R a = (R)1 - tR;
        return ((R)1 / ((R)2 * tH)) * tA * ((R)-20 * tR * a * a * a);
    }
    case 4: {
        tR = rr / tH * (R)0.5;
        if (!(tR < (R)1)) return (R)0;
        R a = (R)1 - tR, a2 = a * a;
        return ((R)1 / ((R)2 * tH)) * tA * ((R)-18.666666666666668 * tR * a2 * a2 * a * ((R)5 * tR + (R)1));
    }
    case 0:
        tR = rr / tH;
        return ((R)1 / tH) * tA * (R)-2 * tR * exp(-tR * tR);
    case 1:
        tR = rr / tH;
        if (tR < (R)1) return ((R)1 / tH) * tA * (ipow((R)3 - tR, 5) + (R)30 * ipow((R)2 - tR, 4) - (R)75 * ipow((R)1 - tR, 4));
        if (tR < (R)2) return ((R)1 / tH) * tA * ((R)-5 * ipow((R)3 - tR, 4) + (R)30 * ipow((R)2 - tR, 4));
        if (tR < (R)3) return ((R)1 / tH) * tA * ((R)-5 * ipow((R)3 - tR, 4));
        return (R)0;
    case 2:
        tR = rr / tH;
        if (!(tR < (R)2)) return (R)0;
        return ((R)1 / tH) * tA * ((R)-9 / (R)8 * (R)2 * tR + (R)19 / (R)24 * (R)3 * tR * tR - (R)5 / (R)32 * (R)4 * tR * tR * tR);
    }
    return (R)0;
}

// ---- pair test with FP32 prefilter -------------------------------------
// inside == (sqrt(dx^2+dy^2+dz^2) + add < Rr) evaluated exactly in FP64.
// The FP32 build first compares the squared distance formed from the
// float-rounded differences against Rr^2 (1 -/+ 1e-6); the relative error
// of that square is below 3e-7, so only pairs inside that band need the
// exact FP64 evaluation.  r is the pair distance in field precision.
template <typename R>
struct PairT {
    R dx, dy, dz, r;
    bool in;
};

template <typename R>
__device__ __forceinline__ PairT<R> pair_test(double xi, double yi, double zi, double xj, double yj, double zj,
                                              double Rr, double add, float r2lo, float r2hi);

template <>
__device__ __forceinline__ PairT<float> pair_test<float>(double xi, double yi, double zi, double xj, double yj,
                                                         double zj, double Rr, double add, float r2lo, float r2hi) {
    PairT<float> g;
    g.dx = (float)(xi - xj);
    g.dy = (float)(yi - yj);
    g.dz = (float)(zi - zj);
    float d2 = g.dx * g.dx + g.dy * g.dy + g.dz * g.dz;
    if (d2 < r2lo) g.in = true;
    else if (d2 > r2hi) g.in = false;
    else g.in = __dadd_rn(pair_dist(xi, yi, zi, xj, yj, zj), add) < Rr;
    g.r = sqrtf(d2);
    return g;
}

template <>
__device__ __forceinline__ PairT<double> pair_test<double>(double xi, double yi, double zi, double xj, double yj,
                                                           double zj, double Rr, double add, float, float) {
    PairT<double> g;
    g.dx = xi - xj;
    g.dy = yi - yj;
    g.dz = zi - zj;
    g.r = pair_dist(xi, yi, zi, xj, yj, zj);
    g.in = __dadd_rn(g.r, add) < Rr;
    return g;
}

__device__ __forceinline__ float r2_lo(double Rr) { return (float)(Rr * Rr * (1.0 - 1e-6)); }
__device__ __forceinline__ float r2_hi(double Rr) { return (float)(Rr * Rr * (1.0 + 1e-6)); }

// ---- stencil rows from a per-cell row table ------------------------------
// The three cells (ix-1..ix+1, jy, kz) have consecutive keys, so their
// particles are one contiguous slot range of the cell-sorted arrays, and
// visiting the 9 (z,y) rows in order with ascending slots inside each row
// is the reference's 27-cell (z,y,x) visit order.  rows[c] holds the cell
// boundaries of the row around cell c (clamped to the grid):
//   [x: first slot of cell ix-1, y: first of ix, z: first of ix+1, w: end),
// built once per step after the cell sort (empty cells have zero width).
//
// Scans skip cells whose box lies farther than the search radius from the
// particle (rows whose y-z distance already exceeds it, and the end cells
// of a row whose x distance does).  Cell boxes follow the hash
// (vmin + c (vmax - vmin)/N); the edge cells of an axis hold every clamped
// particle, so they extend to infinity.  The skip threshold is the radius
// squared times (1 + 1e-8), far above the rounding of the box bounds, so a
// skipped cell cannot hold a particle inside the radius: neighbour sets
// are unchanged, only candidates that fail the test are not visited.
__device__ __forceinline__ int4 row_bounds(const int* __restrict__ gs, const int* __restrict__ ge, int NI, int base,
                                           int ic) {
    int x0 = ic > 0 ? ic - 1 : 0, x1 = ic < NI - 1 ? ic + 1 : NI - 1;
    int lo = -1, hi = 0;
    for (int ix = x0; ix <= x1; ix++) {
        int s = gs[base + ix];
        if (s == -1) continue;
        if (lo < 0) lo = s;
        hi = ge[base + ix];
    }
    if (lo < 0) return make_int4(0, 0, 0, 0);
    int b1 = lo, b2 = hi;
    if (ic > 0 && gs[base + ic - 1] != -1) b1 = ge[base + ic - 1];
    if (ic < NI - 1 && gs[base + ic + 1] != -1) b2 = gs[base + ic + 1];
    return make_int4(lo, b1, b2, hi);
}

// distance from v to the slab of cell c on an axis of N cells
__device__ __forceinline__ double axis_gap(double v, int c, int N, double vmin, double w) {
    double lo = vmin + c * w, hi = vmin + (c + 1) * w;
    double g = 0.0;
    if (c > 0 && v < lo) g = lo - v;
    if (c < N - 1 && v > hi) g = v - hi;
    return g;
}

struct Cull {
    double x, y, z, thr2;   // particle (or point) and (radius)^2 (1 + 1e-8)
};
__device__ __forceinline__ Cull make_cull(double x, double y, double z, double radius) {
    return Cull{x, y, z, radius * radius * (1.0 + 1e-8)};
}

// trimmed slot range of row (jy, kz) around cell ic; false if the row is skipped
__device__ __forceinline__ bool row_range_cull(const DevParams& P, const int4* __restrict__ rows, int ic, int jy,
                                               int kz, const Cull& C, double gxm2, double gxp2, int& a, int& b) {
    double wy = (P.ymax - P.ymin) / P.NJ, wz = (P.zmax - P.zmin) / P.NK;
    double gy = axis_gap(C.y, jy, P.NJ, P.ymin, wy), gz = axis_gap(C.z, kz, P.NK, P.zmin, wz);
    double dyz = gy * gy + gz * gz;
    if (dyz > C.thr2) return false;
    int4 r = __ldg(rows + ic + P.NI * jy + P.NI * P.NJ * kz);
    a = (gxm2 + dyz > C.thr2) ? r.y : r.x;
    b = (gxp2 + dyz > C.thr2) ? r.z : r.w;
    return a < b;
}

__device__ __forceinline__ void x_gaps(const DevParams& P, int ic, const Cull& C, double& gxm2, double& gxp2) {
    double wx = (P.xmax - P.xmin) / P.NI;
    double gm = ic > 0 ? axis_gap(C.x, ic - 1, P.NI, P.xmin, wx) : 0.0;
    double gp = ic < P.NI - 1 ? axis_gap(C.x, ic + 1, P.NI, P.xmin, wx) : 0.0;
    gxm2 = gm * gm;
    gxp2 = gp * gp;
}

template <typename F>
__device__ __forceinline__ void for_rows(const DevParams& P, int ic, int jc, int kc, const int4* __restrict__ rows,
                                         const Cull& C, F f) {
    double gxm2, gxp2;
    x_gaps(P, ic, C, gxm2, gxp2);
    for (int z = -1; z <= 1; z++) {
        int kz = kc + z;
        if (kz < 0 || kz > P.NK - 1) continue;
        for (int y = -1; y <= 1; y++) {
            int jy = jc + y;
            if (jy < 0 || jy > P.NJ - 1) continue;
            int a, b;
            if (row_range_cull(P, rows, ic, jy, kz, C, gxm2, gxp2, a, b)) f(a, b);
        }
    }
}

// One warp scanning the 27-cell stencil of one particle: the 9 (trimmed)
// row ranges are concatenated and lane l takes candidates l, l+32, ... of
// the concatenation, so no lane idles at the end of each row.  sm is 20
// ints of shared memory owned by the warp (row offsets and starts).  Each
// lane visits its candidates in ascending slot order.
template <typename F>
__device__ __forceinline__ void for_rows_warp(const DevParams& P, int ic, int jc, int kc, const int4* __restrict__ rows,
                                              const Cull& C, int* sm, int lane, F f) {
    int len = 0, lo = 0;
    if (lane < 9) {
        int kz = kc + lane / 3 - 1, jy = jc + lane % 3 - 1;
        if (kz >= 0 && kz <= P.NK - 1 && jy >= 0 && jy <= P.NJ - 1) {
            double gxm2, gxp2;
            x_gaps(P, ic, C, gxm2, gxp2);
            int a, b;
            if (row_range_cull(P, rows, ic, jy, kz, C, gxm2, gxp2, a, b)) {
                lo = a;
                len = b - a;
            }
        }
    }
    // inclusive prefix over lanes 0..8
    int inc = len;
#pragma unroll
    for (int o = 1; o < 16; o <<= 1) {
        int v = __shfl_up_sync(0xffffffffu, inc, o);
        if (lane >= o) inc += v;
    }
    if (lane < 9) {
        sm[lane + 1] = inc;
        sm[10 + lane] = lo;
    }
    if (lane == 0) sm[0] = 0;
    int tot = __shfl_sync(0xffffffffu, inc, 8);
    __syncwarp();
    int r = 0, nxt = sm[1], base = sm[10];
    for (int t = lane; t < tot; t += 32) {
        while (t >= nxt) {
            r++;
            nxt = sm[r + 1];
            base = sm[10 + r] - sm[r];
        }
        f(base + t);
    }
    __syncwarp();
}

// for_rows_warp for a body that needs the whole warp every round (a
// ballot): every lane calls f(j) once per round of 32 candidates, j = -1
// where the lane has no candidate.  Lane l still visits candidates l,
// l+32, ... in order.
template <typename F>
__device__ __forceinline__ void for_rows_warp_all(const DevParams& P, int ic, int jc, int kc,
                                                  const int4* __restrict__ rows, const Cull& C, int* sm, int lane,
                                                  F f) {
    int len = 0, lo = 0;
    if (lane < 9) {
        int kz = kc + lane / 3 - 1, jy = jc + lane % 3 - 1;
        if (kz >= 0 && kz <= P.NK - 1 && jy >= 0 && jy <= P.NJ - 1) {
            double gxm2, gxp2;
            x_gaps(P, ic, C, gxm2, gxp2);
            int a, b;
            if (row_range_cull(P, rows, ic, jy, kz, C, gxm2, gxp2, a, b)) {
                lo = a;
                len = b - a;
            }
        }
    }
    int inc = len;
#pragma unroll
    for (int o = 1; o < 16; o <<= 1) {
        int v = __shfl_up_sync(0xffffffffu, inc, o);
        if (lane >= o) inc += v;
    }
    if (lane < 9) {
        sm[lane + 1] = inc;
        sm[10 + lane] = lo;
    }
    if (lane == 0) sm[0] = 0;
    int tot = __shfl_sync(0xffffffffu, inc, 8);
    __syncwarp();
    int r = 0, nxt = sm[1], base = sm[10];
    for (int t0 = 0; t0 < tot; t0 += 32) {
        const int t = t0 + lane;
        int j = -1;
        if (t < tot) {
            while (t >= nxt) {
                r++;
                nxt = sm[r + 1];
                base = sm[10 + r] - sm[r];
            }
            j = base + t;
        }
        f(j);
    }
    __syncwarp();
}

__device__ __forceinline__ float warp_sum(float v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}
__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// one grid-stride-free 1-D launch helper
__host__ __device__ inline int nblocks(int n, int t) { return n <= 0 ? 1 : (n + t - 1) / t; }

}  // namespace sphdem
