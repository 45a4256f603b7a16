// step_kernels.cuh -- the kernels of one ISPH-DEM step.
//
// One kernel per fused pass, launched in the order of SOPHIA_single_ISPH
// (ISPH_Calc_seperate.cuh:13-503):
//
//   k_hash_* / sort / k_cells_gather_*   NNPS: cell key, stable sort by cell,
//                                        cell start/end + SoA permutation
//   k_build_list                         SPH neighbour list (kappa*h_i)
//   k_passA          mass_init + KGC + SPH porosity + prep_sph
//   k_dem_prep       DEM filters and porosity
//   k_passB          prep3D filter + advection forces
//   k_dem_contact    Hertz-Mindlin contact with tangential history
//   k_dem_coupling   Di Felice drag + pressure-gradient force + DEM predictor
//   k_sph_coupling   reaction force + SPH predictor
//   k_neumann        wall pressure/density/temperature extrapolation
//   k_ppe            one Jacobi sweep of the pressure Poisson equation
//   k_passC          pressure force + SPH corrector
//   k_dem_update     DEM corrector + cylinder/box/cone walls
//   k_open_bc        inlet/outlet ghost extrapolation
//   k_xsph           XSPH velocity/temperature smoothing
//
// Each kernel cites the reference kernels it replaces.  R is the field
// precision (float or double); positions, h and radii are always double.
#pragma once
#include "engine.cuh"

namespace sphdem {

// pair geometry in field precision from double positions
template <typename R>
struct Pair {
    R dx, dy, dz, r2, r;
};

template <typename R>
__device__ __forceinline__ Pair<R> make_pair(double xi, double yi, double zi, double xj, double yj, double zj) {
    Pair<R> g;
    g.dx = (R)(xi - xj);
    g.dy = (R)(yi - yj);
    g.dz = (R)(zi - zj);
    g.r2 = g.dx * g.dx + g.dy * g.dy + g.dz * g.dz;
    g.r = sqrt(g.r2);
    return g;
}

template <typename R>
__device__ __forceinline__ void kgc3(const R* __restrict__ Cm, int n, int i, int on, R& ax, R& ay, R& az) {
    if (!on) return;
    R a = ax, b = ay, c = az;
    ax = Cm[0 * n + i] * a + Cm[1 * n + i] * b + Cm[2 * n + i] * c;
    ay = Cm[3 * n + i] * a + Cm[4 * n + i] * b + Cm[5 * n + i] * c;
    az = Cm[6 * n + i] * a + Cm[7 * n + i] * b + Cm[8 * n + i] * c;
}

// Two-dimensional beds (dim 2) lie in a plane y = const and run this step
// with: the 2-D kernel normalisation; SPH particle volume (h / h_over_dx)^2;
// the gradient correction on the x-z block; a DEM sphere (centre in the
// plane; contact, drag and heat as for a sphere) in the porosity with its
// equatorial disc 3.14159 r^2, as the reference's 2-D coupling prep
// (KERNEL_clc_prep2D_coupling, functions_PREP2.cuh:2944-3033) -- the
// sphere's volume over a depth 4 r / 3 -- and its drag and heat acting on
// the fluid per unit depth (divided by that depth).
template <typename R>
__device__ __forceinline__ R dem_measure(const DevParams& P, R r) {
    return P.dim == 2 ? (R)3.14159 * r * r : (R)4.18879 * r * r * r;
}
template <typename R>
__device__ __forceinline__ R sph_volume(const DevParams& P, R th, R hd) {
    return P.dim == 2 ? (th / hd) * (th / hd) : (th / hd) * (th / hd) * (th / hd);
}

// The solver switches the neighbour loops test per pair (gradient
// correction, pressure, viscous and artificial-viscosity forces, heat,
// Lagrangian SPH), fixed at compile time for the common set (SW_COMMON:
// KGC, pressure and viscous forces and heat on, Eulerian) so those loops
// carry no switch tests; SW = -1 reads them from DevParams.
constexpr int SW_KGC = 1, SW_FP = 2, SW_FV = 4, SW_FVA = 8, SW_CON = 16, SW_LAGR = 32;
constexpr int SW_COMMON = SW_KGC | SW_FP | SW_FV | SW_CON;
template <int SW>
__device__ __forceinline__ bool sw_on(int bit, bool runtime) {
    if constexpr (SW < 0) return runtime;
    else return (SW & bit) != 0;
}
inline int switch_set(const DevParams& P) {
    return (P.kgc == 1 ? SW_KGC : 0) | (P.fp ? SW_FP : 0) | (P.fv ? SW_FV : 0) | (P.fva ? SW_FVA : 0) |
           (P.con ? SW_CON : 0) | (P.sph_lagrangian ? SW_LAGR : 0);
}

// 27-cell stencil in the reference order (z,y,x), calling f(j) for every
// slot j of every non-empty cell: the 9 rows in order, ascending slots
// inside a row.
template <typename F>
__device__ __forceinline__ void for_stencil_j(const DevParams& P, int ic, int jc, int kc,
                                              const int4* __restrict__ rows, const Cull& C, F f) {
    for_rows(P, ic, jc, kc, rows, C, [&](int a, int b) {
        for (int j = a; j < b; j++) f(j);
    });
}

// ---------------------------------------------------------------------------
// NNPS
// ---------------------------------------------------------------------------
// KERNEL_index_particle_to_cell_{sph,dem}: functions_NNPS.cuh:762-821
// The cell-sort count (cell_count, cell_sort.cuh) is fused in.
__global__ void k_hash(DevParams P, int n, const double* __restrict__ x, const double* __restrict__ y,
                       const double* __restrict__ z, const int* __restrict__ itype, int* key, int* cnt) {
    grid_dep_wait();
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    int k = -1;
    if (i < n) {
        if (itype[i] == 3) k = P.num_cells;
        else {
            int ic, jc, kc;
            cell_ijk(P, x[i], y[i], z[i], ic, jc, kc);
            k = ic + P.NI * jc + P.NI * P.NJ * kc;
        }
        key[i] = k;
    }
    cell_count(cnt, k);
}

// per-cell stencil row table (for_rows), one thread per cell
__global__ void k_rows(DevParams P, const int* __restrict__ gs, const int* __restrict__ ge, int4* rows) {
    grid_dep_wait();
    int c = blockIdx.x * blockDim.x + threadIdx.x;
    int nc = P.NI * P.NJ * P.NK;
    if (c >= nc) return;
    int ic = c % P.NI, base = c - ic;
    rows[c] = row_bounds(gs, ge, P.NI, base, ic);
}

// reorder of every persistent SPH field, source of m/rho/pres/u/temp is
// the array that held the end-of-step value
template <typename R>
struct SphGatherSrc {
    const R *ux, *uy, *uz, *m, *rho, *pres, *temp;
};

template <typename R>
__global__ void k_cells_gather_sph(DevParams P, SphState<R> src, SphGatherSrc<R> gsrc, SphState<R> dst,
                                   SphRec<R> rec, const int* __restrict__ perm, int* wall_idx, int* buf_idx,
                                   int* counters, DevFlags* F) {
    grid_dep_wait();
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    int n = P.ns;
    if (i >= n) return;
    int p = perm[i];
    double x = src.x[p], y = src.y[p], z = src.z[p];
    dst.x[i] = x;
    dst.y[i] = y;
    dst.z[i] = z;
    dst.h[i] = src.h[p];
    R ux = gsrc.ux[p], uy = gsrc.uy[p], uz = gsrc.uz[p], m = gsrc.m[p], rho = gsrc.rho[p], pr = gsrc.pres[p];
    dst.ux[i] = ux;
    dst.uy[i] = uy;
    dst.uz[i] = uz;
    dst.m[i] = m;
    dst.rho[i] = rho;
    dst.pres[i] = pr;
    dst.temp[i] = gsrc.temp[p];
    dst.dDEMpor[i] = src.dDEMpor[p];
    dst.flt_s[i] = src.flt_s[p];
    dst.dpres[i] = src.dpres[p];
    int pt = src.ptype[p], bt = src.btype[p], it = src.itype[p];
    dst.ptype[i] = pt;
    dst.btype[i] = bt;
    dst.itype[i] = it;
    dst.pid[i] = src.pid[p];
    store_pos(rec.pos, i, make_pos<R>(P, x, y, z, pt, bt, it));
    rec.mr0[i] = mk2<R>(m, rho);
    rec.up[i] = mk4<R>(ux, uy, uz, pr);
    // walls and buffer particles of the step (parked slots excluded), up to
    // the launch bounds of their passes
    if (it != 3 && pt <= 0) {
        int k = atomicAdd(&counters[0], 1);
        if (k < P.nwall) wall_idx[k] = i;
        else atomicOr(&F->overflow, 4);
    }
    if (it != 3 && bt > 0 && pt < 1000) {
        int k = atomicAdd(&counters[1], 1);
        if (k < P.nbuf) buf_idx[k] = i;
        else atomicOr(&F->overflow, 4);
    }
}

template <typename R>
__global__ void k_cells_gather_dem(DevParams P, DemState<R> src, DemState<R> dst, const int* __restrict__ perm) {
    grid_dep_wait();
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    int n = P.nd;
    if (i >= n) return;
    int p = perm[i];
    dst.x[i] = src.x[p]; dst.y[i] = src.y[p]; dst.z[i] = src.z[p];
    dst.h[i] = src.h[p]; dst.rad[i] = src.rad[p];
    dst.ux[i] = src.ux[p]; dst.uy[i] = src.uy[p]; dst.uz[i] = src.uz[p];
    dst.wx[i] = src.wx[p]; dst.wy[i] = src.wy[p]; dst.wz[i] = src.wz[p];
    dst.m[i] = src.m[p]; dst.rho[i] = src.rho[p]; dst.ri[i] = src.ri[p];
    dst.temp[i] = src.temp[p]; dst.temp1[i] = src.temp1[p]; dst.temp2[i] = src.temp2[p]; dst.temp3[i] = src.temp3[p];
    dst.Fdx_df[i] = src.Fdx_df[p]; dst.Fdy_df[i] = src.Fdy_df[p]; dst.Fdz_df[i] = src.Fdz_df[p];
    dst.Q_sd[i] = src.Q_sd[p];
    dst.ptype[i] = src.ptype[p]; dst.btype[i] = src.btype[p]; dst.itype[i] = src.itype[p];
    dst.pid[i] = src.pid[p]; dst.dem_idx[i] = src.dem_idx[p];
}

// SPH neighbour list: the candidate set and predicate of every SPH gather
// kernel (e.g. functions_PPE2.cuh:609-638): 27-cell stencil and
// sqrt(dx^2+dy^2+dz^2) + 1e-20 < kappa*h_i, decided exactly in FP64 (see
// test_pair).  Rows come out in ascending slot order, which is the
// reference's z,y,x cell visit order.  Column-major rows.  Threads of a
// warp are consecutive slots, mostly of one cell, so they walk the same
// candidate rows and their position-record loads coalesce.
template <typename R>
__global__ void __launch_bounds__(128) k_build_list(DevParams P, SphState<R> S, SphRec<R> rec,
                                                    const int4* __restrict__ rows,
                                                    int* __restrict__ nbr, int* __restrict__ ncnt, DevFlags* F) {
    grid_dep_wait();
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= P.ns) return;
    double xi = S.x[i], yi = S.y[i], zi = S.z[i];
    double Rr = __dmul_rn(P.kappa, S.h[i]);
    Band bd = make_band(P, Rr);
    PosRec<R> qi = ldr(rec.pos + i);
    int ic, jc, kc;
    cell_ijk(P, xi, yi, zi, ic, jc, kc);
    int c = 0, cap = P.nb_cap, n = P.ns;
    const Cull cu = make_cull(xi, yi, zi, Rr);
    for_rows(P, ic, jc, kc, rows, cu, [&](int a, int b) {
        for (int j = a; j < b; j++) {
            PosRec<R> qj = ldr(rec.pos + j);
            Disp<R> d;
            R r2;
            if (test_pair(P, qi, qj, xi, yi, zi, S.x, S.y, S.z, j, Rr, 1e-20, bd, d, r2)) {
                if (nbr && c < cap) nbr[nb_at(c, n, i)] = j;
                c++;
            }
        }
    });
    ncnt[i] = c;
    if (c > cap) atomicOr(&F->overflow, 1);
    // one atomic per converged group of threads for the largest count
    const unsigned am = __activemask();
    const int wmax = __reduce_max_sync(am, c);
    if ((threadIdx.x & 31) == __ffs(am) - 1) atomicMax(&F->max_ncnt, wmax);
}

// The 9 full stencil rows (z, y order) of cell (ic, jc, kc) for a whole
// warp: s[0..9] the prefix of the row lengths, s[10..18] the first slot of
// each row.  Returns the number of candidates; row_slot maps candidate t
// (0 <= t < that number) to its slot, in the reference's visit order.
__device__ __forceinline__ int stage_rows(const DevParams& P, int ic, int jc, int kc, const int4* __restrict__ rows,
                                          int* s, int lane) {
    int len = 0, lo = 0;
    if (lane < 9) {
        int kz = kc + lane / 3 - 1, jy = jc + lane % 3 - 1;
        if (kz >= 0 && kz <= P.NK - 1 && jy >= 0 && jy <= P.NJ - 1) {
            int4 r = __ldg(rows + ic + P.NI * jy + P.NI * P.NJ * kz);
            lo = r.x;
            len = max(r.w - r.x, 0);
        }
    }
    int inc = len;
#pragma unroll
    for (int o = 1; o < 16; o <<= 1) {
        int v = __shfl_up_sync(0xffffffffu, inc, o);
        if (lane >= o) inc += v;
    }
    if (lane < 9) {
        s[lane + 1] = inc;
        s[10 + lane] = lo;
    }
    if (lane == 0) s[0] = 0;
    __syncwarp();
    return __shfl_sync(0xffffffffu, inc, 8);
}
__device__ __forceinline__ int row_slot(const int* s, int t) {
    int r = 0;
    while (t >= s[r + 1]) r++;
    return s[10 + r] + (t - s[r]);
}

// Relative FP32 coordinates of the cell-tiled passes.  A fixed-point
// position q is staged as (q - q0) x step, q0 a particle of the cell.  A
// position within Lk = 2 cell widths of q0 on every axis (all of a cell's
// stencil, unless a particle outside the box was clamped into a boundary
// cell) is 'near'; each staged coordinate then carries at most 2 x 2^-24 Lk
// of rounding (int -> float and x step), a difference at most 6 x 2^-24 Lk,
// and r^2 near Rr^2 moves by at most 2 sqrt(3) Rr (6 x 2^-24 L) + 3 FP32
// roundings, L = max Lk.  rel_band returns b with |r^2 error| < b Rr^2:
// 1.3e-6 L/Rr covers the rounding, q_abs/Rr the fixed-point quantisation
// of both positions, 1e-6 the rest.  A pair with a position outside the
// fixed-point range or not near takes the FP64 predicate.
struct RelFrame {
    int4 q0;
    int lx, ly, lz;         // 2 cell widths in steps per axis
    double L;               // max 2 cell widths (length)
    float sx, sy, sz;
    bool o_oor;             // q0 outside the fixed-point range: every pair exact
};
__device__ __forceinline__ RelFrame rel_frame(const DevParams& P, const int4& q0) {
    RelFrame F;
    F.q0 = q0;
    const double wx = (P.xmax - P.xmin) / P.NI, wy = (P.ymax - P.ymin) / P.NJ, wz = (P.zmax - P.zmin) / P.NK;
    F.lx = (int)fmin(2.0 * wx * P.q_inv[0] + 2.0, 2147483647.0);
    F.ly = (int)fmin(2.0 * wy * P.q_inv[1] + 2.0, 2147483647.0);
    F.lz = (int)fmin(2.0 * wz * P.q_inv[2] + 2.0, 2147483647.0);
    F.L = 2.0 * fmax(fmax(wx, wy), wz);
    F.sx = P.q_step[0];
    F.sy = P.q_step[1];
    F.sz = P.q_step[2];
    F.o_oor = (q0.w & TAG_OOR) != 0;
    return F;
}
// q outside the fixed-point range or not near q0.  In-range coordinates
// are below 2^30 in magnitude (quantize), so the int differences are exact.
__device__ __forceinline__ bool rel_slow(const RelFrame& F, const int4& q) {
    return (q.w & TAG_OOR) || abs(q.x - F.q0.x) > F.lx || abs(q.y - F.q0.y) > F.ly || abs(q.z - F.q0.z) > F.lz;
}
__device__ __forceinline__ float4 rel_coord(const RelFrame& F, const int4& q, int tagw) {
    return make_float4((float)(q.x - F.q0.x) * F.sx, (float)(q.y - F.q0.y) * F.sy, (float)(q.z - F.q0.z) * F.sz,
                       __int_as_float(tagw));
}
__device__ __forceinline__ double rel_band(const DevParams& P, const RelFrame& F, double Rr) {
    return 1e-6 + 1.3e-6 * F.L / Rr + P.q_abs / Rr;
}

// Cell-tiled list build (FP32 build).  One warp per cell: the particles of
// a cell share one stencil, so the warp stages the candidates of the 9 rows
// once, as FP32 coordinates relative to a particle of the cell, into shared
// memory (chunks of 128), and every lane -- one particle of the cell --
// tests them in the same order against its own radius.  All lanes read the
// same staged candidate (a broadcast) and run in lockstep; a pair costs a
// few FP32 operations instead of a global load and the fixed-point
// conversion.  Each lane appends its hits in staged order, which is the
// reference's z, y, x cell order with ascending slots, so the list equals
// the one-particle-per-thread build.  Prefilter: r^2 against Rr^2 (1 -/+ b)
// with b from rel_band.  Pairs in the band, or with a position outside the
// fixed-point range or not near the origin, take the reference predicate in
// FP64.
//
// The fast path forms r^2 as |c|^2 - 2 p.c + |p|^2: a candidate is staged
// with |c|^2, a lane holds -2p and compares |c|^2 - 2 p.c (three FMAs)
// against its threshold minus |p|^2.  Against the difference form this adds
// rounding of the magnitudes: |c|^2 (3 roundings), the three FMAs and |p|^2
// (3 more) and the threshold's subtraction, in all at most
// 6u (|c| + |p|)^2 + u hi^2 with u = 2^-24; both positions are near the
// origin (|c|, |p| <= sqrt(3) L), so dot_band widens the band by
// 80u (L / Rr)^2 + 2u of Rr^2.  Within the wider band the FP64 predicate
// decides, so the lists are unchanged.
// LW cells (warps) per block: 2, 4 or 8, picked per handle at commit with
// the one-thread-per-particle build (k_build_list) as the fourth candidate
// (list_build_mode, engine.cu); all four write the same lists.
constexpr int LT_CH = 128;
__device__ __forceinline__ double dot_band(const RelFrame& F, double Rr) {
    const double u = 5.9604644775390625e-08, q = F.L / Rr;
    return 80.0 * u * q * q + 2.0 * u;
}
template <int LW>
__global__ void __launch_bounds__(LW * 32) k_build_list_tiled(DevParams P, SphState<float> S,
                                                                      SphRec<float> rec,
                                                                      const int* __restrict__ gs,
                                                                      const int* __restrict__ ge,
                                                                      const int4* __restrict__ rows,
                                                                      int* __restrict__ nbr,
                                                                      int* __restrict__ ncnt, DevFlags* F) {
    grid_dep_wait();
    __shared__ float4 sc[LW][LT_CH + 4];   // relative x, y, z and |c|^2
    __shared__ int sj[LW][LT_CH + 4];      // slot, bit 31: not near the origin
    __shared__ int srow[LW][20];   // prefix[10] | start[9]
    const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int c = blockIdx.x * LW + w;
    const int ncell = P.NI * P.NJ * P.NK;
    if (c >= ncell) return;
    const int a0 = __ldg(gs + c);
    if (a0 < 0) return;
    const int e0 = __ldg(ge + c);
    const int ic = c % P.NI, jc = (c / P.NI) % P.NJ, kc = c / (P.NI * P.NJ);
    const int tot = stage_rows(P, ic, jc, kc, rows, srow[w], lane);
    const RelFrame Fr = rel_frame(P, ldr(rec.pos + a0));   // origin of the relative coordinates
    const int n = P.ns, cap = P.nb_cap;
    for (int p0 = a0; p0 < e0; p0 += 32) {
        const int i = p0 + lane;
        const bool act = i < e0;
        double xi = 0, yi = 0, zi = 0, Rr = 0;
        float lo2 = 0, hi2 = 0, fx = 0, fy = 0, fz = 0;
        float ax = 0, ay = 0, az = 0, tlo = 0, thi = 0;   // -2p and the thresholds of the fast path
        bool slow = true;
        if (act) {
            xi = S.x[i];
            yi = S.y[i];
            zi = S.z[i];
            Rr = __dmul_rn(P.kappa, S.h[i]);
            const double b = rel_band(P, Fr, Rr), r2 = Rr * Rr, bd = b + dot_band(Fr, Rr);
            lo2 = (float)(r2 * (1.0 - b));
            hi2 = (float)(r2 * (1.0 + b));
            const int4 qi = ldr(rec.pos + i);
            slow = Fr.o_oor || rel_slow(Fr, qi);
            const float4 f = rel_coord(Fr, qi, 0);
            fx = f.x;
            fy = f.y;
            fz = f.z;
            ax = -2.f * fx;
            ay = -2.f * fy;
            az = -2.f * fz;
            const float pp = fmaf(fz, fz, fmaf(fy, fy, fx * fx));
            tlo = (float)(r2 * (1.0 - bd)) - pp;
            thi = (float)(r2 * (1.0 + bd)) - pp;
        }
        int cnt = 0;
        // entry cnt of particle i at pw: +1 inside a block of 8 entries, to
        // the particle's next block (8n further) after the eighth
        int* pw = nbr ? nbr + nb_at(0, n, i) : nullptr;
        const ptrdiff_t next_block = 8 * (ptrdiff_t)n - 7;
        auto push = [&](int j) {
            if (pw && cnt < cap) *pw = j;
            pw += ((cnt & 7) == 7) ? next_block : 1;
            cnt++;
        };
        const bool lanes_slow = __any_sync(0xffffffffu, act && slow);
        // Candidates that no lane of this group can reach are not staged: the
        // lanes' box [bl, bh] and their largest prefilter radius hb.  The box
        // distance is formed like a lane's r^2 from differences that are no
        // larger, and FP32 rounding is monotone, so a candidate with box
        // distance^2 > hb (1 + 2^-20) has r^2 > hi2 for every lane.  Off while
        // a lane takes the FP64 path; a candidate outside the fixed-point
        // range is always staged.
        float blx = act ? fx : 3e38f, bly = act ? fy : 3e38f, blz = act ? fz : 3e38f;
        float bhx = act ? fx : -3e38f, bhy = act ? fy : -3e38f, bhz = act ? fz : -3e38f;
        float hb = act ? hi2 : 0.f;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            blx = fminf(blx, __shfl_xor_sync(0xffffffffu, blx, o));
            bly = fminf(bly, __shfl_xor_sync(0xffffffffu, bly, o));
            blz = fminf(blz, __shfl_xor_sync(0xffffffffu, blz, o));
            bhx = fmaxf(bhx, __shfl_xor_sync(0xffffffffu, bhx, o));
            bhy = fmaxf(bhy, __shfl_xor_sync(0xffffffffu, bhy, o));
            bhz = fmaxf(bhz, __shfl_xor_sync(0xffffffffu, bhz, o));
            hb = fmaxf(hb, __shfl_xor_sync(0xffffffffu, hb, o));
        }
        hb *= 1.f + 9.5367431640625e-07f;
        const unsigned lt = (1u << lane) - 1u;
        int t = 0;
        while (t < tot) {
            // stage the next candidates that pass the box test, in order
            int tn = 0;
            bool any_oor = false;
            while (t < tot && tn <= LT_CH - 32) {
                const int tl = t + lane;
                bool keep = false;
                float4 v;
                int jt = 0;
                if (tl < tot) {
                    const int j = row_slot(srow[w], tl);
                    const int4 qj = ldr(rec.pos + j);
                    const bool oor = rel_slow(Fr, qj);
                    v = rel_coord(Fr, qj, 0);
                    v.w = fmaf(v.z, v.z, fmaf(v.y, v.y, v.x * v.x));
                    jt = j | (oor ? (int)0x80000000 : 0);
                    const float dx = fmaxf(fmaxf(blx - v.x, v.x - bhx), 0.f);
                    const float dy = fmaxf(fmaxf(bly - v.y, v.y - bhy), 0.f);
                    const float dz = fmaxf(fmaxf(blz - v.z, v.z - bhz), 0.f);
                    keep = oor || lanes_slow || dx * dx + dy * dy + dz * dz <= hb;
                    any_oor |= keep && oor;
                }
                const unsigned m = __ballot_sync(0xffffffffu, keep);
                if (keep) {
                    const int pos = tn + __popc(m & lt);
                    sc[w][pos] = v;
                    sj[w][pos] = jt;
                }
                tn += __popc(m);
                t += 32;
            }
            // padded to whole groups of four; the padding (|c|^2 = inf) fails every test
            const int tp = (tn + 3) & ~3;
            if (lane < tp - tn) {
                sc[w][tn + lane] = make_float4(0.f, 0.f, 0.f, __int_as_float(0x7f800000));
                sj[w][tn + lane] = 0;
            }
            const bool slow_chunk = lanes_slow || __any_sync(0xffffffffu, any_oor);
            __syncwarp();
            if (act && !slow_chunk) {
                // fast path: FP32 prefilter, FP64 only inside the band
                for (int u = 0; u < tp; u += 4) {
                    float tv[4];
#pragma unroll
                    for (int k = 0; k < 4; k++) {
                        const float4 cv = sc[w][u + k];
                        tv[k] = fmaf(az, cv.z, fmaf(ay, cv.y, fmaf(ax, cv.x, cv.w)));
                    }
#pragma unroll
                    for (int k = 0; k < 4; k++) {
                        if (tv[k] <= thi) {
                            const int j = sj[w][u + k];
                            bool hit = tv[k] < tlo;
                            if (!hit) hit = __dadd_rn(pair_dist(xi, yi, zi, S.x[j], S.y[j], S.z[j]), 1e-20) < Rr;
                            if (hit) push(j);
                        }
                    }
                }
            } else if (act) {
                // a particle or candidate outside the fixed-point range: FP64 where needed
                for (int u = 0; u < tn; u++) {
                    const float4 cj = sc[w][u];
                    const float dx = fx - cj.x, dy = fy - cj.y, dz = fz - cj.z;
                    const float r2 = dx * dx + dy * dy + dz * dz;
                    const int jb = sj[w][u];
                    const int j = jb & 0x7fffffff;
                    bool hit;
                    if (!slow && jb >= 0) {
                        if (r2 < lo2) hit = true;
                        else if (r2 > hi2) hit = false;
                        else hit = __dadd_rn(pair_dist(xi, yi, zi, S.x[j], S.y[j], S.z[j]), 1e-20) < Rr;
                    } else {
                        hit = __dadd_rn(pair_dist(xi, yi, zi, S.x[j], S.y[j], S.z[j]), 1e-20) < Rr;
                    }
                    if (hit) push(j);
                }
            }
            __syncwarp();
        }
        if (act) {
            ncnt[i] = cnt;
            if (cnt > cap) atomicOr(&F->overflow, 1);
        }
        // one atomic per warp for the largest count
        const int wmax = __reduce_max_sync(0xffffffffu, act ? cnt : 0);
        if (lane == 0 && wmax > 0) atomicMax(&F->max_ncnt, wmax);
    }
}

// SPH -> DEM candidate list.  The SPH kernels that sum over DEM spheres
// (pass A's porosity, the reaction force of k_sph_coupling) visit the DEM
// slots of the 27-cell stencil in the reference's order and keep those
// with |x_i - x_j| < kappa h_i.  About one stencil candidate in ten is
// inside, so this pass finds them once per step and the two kernels walk
// the short list (same slots, same order) and repeat their own test on it.
// The list holds every j with pair_dist < kappa h_i, the add = 0 form of
// the predicate; the 1e-20 form of pass A keeps a subset of it.
//
// One warp per cell, as k_build_list_tiled: the cell's DEM candidates
// (p_type > 1000) are staged compacted in shared memory as FP32 coordinates
// relative to the cell's first SPH particle, and each lane -- one SPH
// particle of the cell -- tests them in order.  A coordinate within
// Lb = 4 cells of the origin is rounded by at most e = 2^-24 Lb, a
// difference by 4 e, so r^2 moves by at most 2 sqrt(3) Rr (4 e) + 3 (4 e)^2
// near the radius, plus a few FP32 roundings; the band below is wider and
// pairs inside it take the FP64 predicate.  A particle or sphere farther
// than Lb from the origin (one clamped into a boundary cell) always takes
// the FP64 predicate.  ncntd holds the exact count; a particle with more
// than cap hits keeps only its count, and the consumers walk its stencil
// instead.
constexpr int DL_WARPS = 4, DL_CH = 128;
// one cell of k_build_dlist (scw, srw: the warp's shared staging)
__device__ __forceinline__ void dlist_cell(int c, DevParams P, const double* __restrict__ sx,
                                                                 const double* __restrict__ sy,
                                                                 const double* __restrict__ sz,
                                                                 const double* __restrict__ sh,
                                                                 const int* __restrict__ gs, const int* __restrict__ ge,
                                                                 const int4* __restrict__ drows,
                                                                 const double* __restrict__ dx,
                                                                 const double* __restrict__ dy,
                                                                 const double* __restrict__ dz,
                                                                 const int* __restrict__ dptype, int* __restrict__ nbrd,
                                                                 int* __restrict__ ncntd, int cap, DevFlags* F, float4* scw, int* srw, int lane) {    const int a0 = __ldg(gs + c);
    if (a0 < 0) return;
    const int e0 = __ldg(ge + c);
    const int ic = c % P.NI, jc = (c / P.NI) % P.NJ, kc = c / (P.NI * P.NJ);
    const int tot = stage_rows(P, ic, jc, kc, drows, srw, lane);
    const int n = P.ns;
    const double x0 = sx[a0], y0 = sy[a0], z0 = sz[a0];
    const double Lb = 4.0 * fmax(fmax((P.xmax - P.xmin) / P.NI, (P.ymax - P.ymin) / P.NJ), (P.zmax - P.zmin) / P.NK);
    const double e4 = 4.0 * 5.9604644775390625e-08 * Lb;   // 4 x 2^-24 x Lb
    const unsigned lt = (1u << lane) - 1u;
    for (int p0 = a0; p0 < e0; p0 += 32) {
        const int i = p0 + lane;
        const bool act = i < e0;
        double xi = 0, yi = 0, zi = 0, Rr = 0;
        float lo2 = 0, hi2 = 0, fx = 0, fy = 0, fz = 0;
        bool slow = false;
        if (act) {
            xi = sx[i];
            yi = sy[i];
            zi = sz[i];
            Rr = P.kappa * sh[i];
            const double r2 = Rr * Rr, d = 3.5 * Rr * e4 + 3.0 * e4 * e4 + 2e-6 * r2;
            lo2 = (float)(r2 - d);
            hi2 = (float)(r2 + d);
            const double ux = xi - x0, uy = yi - y0, uz = zi - z0;
            slow = !(fabs(ux) <= Lb && fabs(uy) <= Lb && fabs(uz) <= Lb);
            fx = (float)ux;
            fy = (float)uy;
            fz = (float)uz;
        }
        const bool lanes_slow = __any_sync(0xffffffffu, act && slow);
        int cnt = 0;
        int* pw = nbrd ? nbrd + i : nullptr;   // entry cnt of row i at pw (pw += n per hit)
        int t = 0;
        while (t < tot) {
            int ns = 0;
            bool any_far = false;
            while (t < tot && ns <= DL_CH - 32) {
                const int tl = t + lane;
                int j = 0;
                bool keep = false;
                if (tl < tot) {
                    j = row_slot(srw, tl);
                    keep = __ldg(dptype + j) > 1000;
                }
                const unsigned m = __ballot_sync(0xffffffffu, keep);
                if (keep) {
                    const double ux = dx[j] - x0, uy = dy[j] - y0, uz = dz[j] - z0;
                    const bool far = !(fabs(ux) <= Lb && fabs(uy) <= Lb && fabs(uz) <= Lb);
                    any_far |= far;
                    scw[ns + __popc(m & lt)] =
                        make_float4((float)ux, (float)uy, (float)uz, __int_as_float(j | (far ? (int)0x80000000 : 0)));
                }
                ns += __popc(m);
                t += 32;
            }
            const bool slow_chunk = lanes_slow || __any_sync(0xffffffffu, any_far);
            __syncwarp();
            if (act) {
                for (int u = 0; u < ns; u++) {
                    const float4 cj = scw[u];
                    const int jb = __float_as_int(cj.w), j = jb & 0x7fffffff;
                    bool hit;
                    if (!slow_chunk || (!slow && jb >= 0)) {
                        const float ex = fx - cj.x, ey = fy - cj.y, ez = fz - cj.z;
                        const float r2 = ex * ex + ey * ey + ez * ez;
                        if (r2 > hi2) continue;
                        hit = r2 < lo2 || pair_dist(xi, yi, zi, dx[j], dy[j], dz[j]) < Rr;
                    } else {
                        hit = pair_dist(xi, yi, zi, dx[j], dy[j], dz[j]) < Rr;
                    }
                    if (hit) {
                        if (pw && cnt < cap) *pw = j;
                        pw += n;
                        cnt++;
                    }
                }
            }
            __syncwarp();
        }
        if (act) ncntd[i] = cnt;
        const int wmax = __reduce_max_sync(0xffffffffu, act ? cnt : 0);
        if (lane == 0 && wmax > 0) atomicMax(&F->max_ncntd, wmax);
    }
}

// The same list with one thread per SPH particle over the DEM slots of its
// stencil rows (the exact predicate for every candidate): the same entries
// in the same order.  Picked per handle at commit where it is faster (2-D
// beds, whose cells hold a few particles each); parked slots (i_type 3) keep
// their count, as the warp-per-cell build leaves them.
__global__ void __launch_bounds__(128) k_build_dlist_pp(DevParams P, const double* __restrict__ sx,
                                                        const double* __restrict__ sy,
                                                        const double* __restrict__ sz,
                                                        const double* __restrict__ sh,
                                                        const int* __restrict__ itype,
                                                        const int4* __restrict__ drows,
                                                        const double* __restrict__ dx,
                                                        const double* __restrict__ dy,
                                                        const double* __restrict__ dz,
                                                        const int* __restrict__ dptype, int* __restrict__ nbrd,
                                                        int* __restrict__ ncntd, int cap, DevFlags* F) {
    grid_dep_wait();
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int n = P.ns;
    const bool act = i < n && itype[i] != 3;
    int cnt = 0;
    if (act) {
        const double xi = sx[i], yi = sy[i], zi = sz[i], Rr = P.kappa * sh[i];
        int ic, jc, kc;
        cell_ijk(P, xi, yi, zi, ic, jc, kc);
        int* pw = nbrd ? nbrd + i : nullptr;   // entry cnt of row i at pw (pw += n per hit)
        for_stencil_j(P, ic, jc, kc, drows, make_cull(xi, yi, zi, Rr), [&](int j) {
            if (__ldg(dptype + j) <= 1000) return;
            if (pair_dist(xi, yi, zi, dx[j], dy[j], dz[j]) < Rr) {
                if (pw && cnt < cap) *pw = j;
                pw += n;
                cnt++;
            }
        });
        ncntd[i] = cnt;
    }
    const int wmax = __reduce_max_sync(0xffffffffu, act ? cnt : 0);
    if ((threadIdx.x & 31) == 0 && wmax > 0) atomicMax(&F->max_ncntd, wmax);
}

template <bool OCC>
__global__ void __launch_bounds__(DL_WARPS * 32) k_build_dlist(DevParams P, const double* __restrict__ sx,
                                                                 const double* __restrict__ sy,
                                                                 const double* __restrict__ sz,
                                                                 const double* __restrict__ sh,
                                                                 const int* __restrict__ gs, const int* __restrict__ ge,
                                                                 const int4* __restrict__ drows,
                                                                 const double* __restrict__ dx,
                                                                 const double* __restrict__ dy,
                                                                 const double* __restrict__ dz,
                                                                 const int* __restrict__ dptype, int* __restrict__ nbrd,
                                                                 int* __restrict__ ncntd, int cap, DevFlags* F,
                                                                 const int* __restrict__ occ, const int* __restrict__ occ_n) {
    grid_dep_wait();
    __shared__ float4 sc[DL_WARPS][DL_CH + 32];
    __shared__ int srow[DL_WARPS][20];
    const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
    if constexpr (OCC) {   // a sparse grid: the occupied cells, grid-stride
        const int no = *occ_n;
        for (int q = blockIdx.x * DL_WARPS + w; q < no; q += gridDim.x * DL_WARPS) {
            dlist_cell(occ[q], P, sx, sy, sz, sh, gs, ge, drows, dx, dy, dz, dptype, nbrd, ncntd, cap, F, sc[w], srow[w], lane);
            __syncwarp();
        }
    } else {
        const int c = blockIdx.x * DL_WARPS + w;
        if (c < P.NI * P.NJ * P.NK)
            dlist_cell(c, P, sx, sy, sz, sh, gs, ge, drows, dx, dy, dz, dptype, nbrd, ncntd, cap, F, sc[w], srow[w], lane);
    }
}

// ---------------------------------------------------------------------------
// pass A: KERNEL_clc_mass_init_sph (functions_MASS.cuh:24-43),
// KERNEL_clc_correction_KGC_3D_sph (functions_PREP2.cuh:452-568),
// KERNEL_clc_prep3D_coupling_sph (functions_PREP2.cuh:3190-3364),
// KERNEL_clc_prep3D_prep_sph (functions_PREP2.cuh:1623-1679).
// Neighbours read the start-of-step m, rho; the new m, rho go to m_new,
// rho_new so that no thread sees a half-updated neighbour.
// ---------------------------------------------------------------------------
template <typename R, int KT, int SW>
__global__ void __launch_bounds__(128, sizeof(R) == 4 ? 8 : 1) k_passA(DevParams P, SphState<R> S, SphWork<R> W, DemState<double> D,
                                               const int4* __restrict__ drows) {
    grid_dep_wait();
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    int n = P.ns;
    if (i >= n) return;
    const SphRec<R> rec = W.rec;
    int it = S.itype[i], pt = S.ptype[i];
    R mo = S.m[i], ro = S.rho[i];
    if (it > 2) {
        W.m_new[i] = mo;
        W.rho_new[i] = ro;
        rec.f1[i] = mk4<R>(mo, ro, S.temp[i], W.DEMpor[i]);
        return;
    }
    R dprev = S.dDEMpor[i];
    W.dDEMpor_prev[i] = dprev;
    double xi = S.x[i], yi = S.y[i], zi = S.z[i], hi = S.h[i];
    R th = (R)hi;
    Knl<R, KT> K = knl_make<R, KT>(P, th);
    PosRec<R> qi = ldr(rec.pos + i);
    int cnt = min(W.ncnt[i], P.nb_cap);
    R txx = 0, tyy = 0, tzz = 0, txy = 0, tyz = 0, tzx = 0, sflt = 0;
    const int* __restrict__ nb = W.nbr;
    const bool kgc = sw_on<SW>(SW_KGC, P.kgc == 1);
    nb_walk<4, NbQ2<R>>(
        cnt, nb, n, i,
        [&](int j) {
            NbQ2<R> t;
            t.q = ldr(rec.pos + j);
            t.a = ldr(rec.mr0 + j);
            return t;
        },
        [&](int j, const NbQ2<R>& t) {
            int ptj = tag_ptype(t.q.w);
            if (ptj > 1000) return;
            Disp<R> g = disp(P, qi, t.q, S.x, S.y, S.z, i, j);
            R r2 = g.dx * g.dx + g.dy * g.dy + g.dz * g.dz, r, rinv;
            rdist(r2, r, rinv);
            R irj = rcp(t.a.y);
            if (ptj == 1) sflt += t.a.x * irj * kw(K, r);
            if (kgc && r2 > (R)0) {
                R dw = kdw(K, r);
                R c = -t.a.x * dw * irj * rinv;
                txx += c * g.dx * g.dx;
                txy += c * g.dy * g.dx;
                tyy += c * g.dy * g.dy;
                tzx += c * g.dx * g.dz;
                tyz += c * g.dy * g.dz;
                tzz += c * g.dz * g.dz;
            }
        });
    if (kgc && P.dim == 2) {
        // a bed in a plane y = const: the x-z block of the moment matrix
        const R det = txx * tzz - tzx * tzx;
        R C[9] = {1, 0, 0, 0, 1, 0, 0, 0, 1};
        if (fabs(det) > (R)1e-4) {
            const R rr = (R)1 / det;
            C[0] = tzz * rr;
            C[2] = -tzx * rr;
            C[6] = -tzx * rr;
            C[8] = txx * rr;
        }
#pragma unroll
        for (int q = 0; q < 9; q++) W.Cm[(size_t)q * n + i] = C[q];
    } else if (kgc) {
        R det = txx * (tyy * tzz - tyz * tyz);
        det -= txy * (txy * tzz - tyz * tzx);
        det += tzx * (txy * tyz - tyy * tzx);
        R C[9];
        if (fabs(det) > (R)1e-4) {
            R rr = (R)1 / det;
            C[0] = (tyy * tzz - tyz * tyz) * rr;
            C[1] = (tzx * tyz - txy * tzz) * rr;
            C[2] = (txy * tyz - tzx * tyy) * rr;
            C[3] = (tzx * tyz - txy * tzz) * rr;
            C[4] = (txx * tzz - tzx * tzx) * rr;
            C[5] = (tzx * txy - txx * tyz) * rr;
            C[6] = (txy * tyz - tzx * tyy) * rr;
            C[7] = (tzx * txy - txx * tyz) * rr;
            C[8] = (txx * tyy - txy * txy) * rr;
        } else {
            C[0] = 1; C[1] = 0; C[2] = 0; C[3] = 0; C[4] = 1; C[5] = 0; C[6] = 0; C[7] = 0; C[8] = 1;
        }
#pragma unroll
        for (int q = 0; q < 9; q++) W.Cm[(size_t)q * n + i] = C[q];
    }
    // SPH-DEM porosity over the SPH -> DEM list (DEM arrays are small and
    // L2-resident: plain loads)
    double Rr = P.kappa * hi;
    R por = 0, dfx = 0, dfy = 0, dfz = 0;
    if (P.nd > 0) {
        float r2l = r2_lo(Rr), r2h = r2_hi(Rr);
        auto dem = [&](int j) {
            if (D.ptype[j] <= 1000) return;
            PairT<R> g = pair_test<R>(xi, yi, zi, D.x[j], D.y[j], D.z[j], Rr, 1e-20, r2l, r2h);
            if (!g.in) return;
            R r = g.r + (R)1e-20, ir = rcp(r);
            R w = kw(K, r);
            R dw = kdw(K, r);
            R rj = (R)D.rad[j];
            R v = dem_measure(P, rj);
            por += w * v;
            dfx += dw * g.dx * ir * (R)D.ux[j] * v;
            dfy += dw * g.dy * ir * (R)D.uy[j] * v;
            dfz += dw * g.dz * ir * (R)D.uz[j] * v;
        };
        const int cd = W.ncntd[i];
        if (cd <= P.nbd_cap) {
            for (int k = 0; k < cd; k++) dem(W.nbrd[(size_t)k * n + i]);
        } else {
            int ic, jc, kc;
            cell_ijk(P, xi, yi, zi, ic, jc, kc);
            for_stencil_j(P, ic, jc, kc, drows, make_cull(xi, yi, zi, Rr), dem);
        }
    }
    R isf = rcp(sflt + (R)1e-20);
    R pori = (R)1 - por * isf;
    W.DEMpor[i] = pori;
    S.dDEMpor[i] = (dfx + dfy + dfz) * isf;
    // prep_sph
    R hd = (R)P.h_over_dx;
    R v = sph_volume(P, th, hd);
    R mref;
    if (pt == 9) mref = (R)P.rho_liquid * v * pori;
    else if (pt == -3 || pt == 0 || pt == 3 || pt == 1) mref = (R)P.rho_gas * v * pori;
    else mref = (R)P.rho_liquid * v * pori;
    if (pt == 9 && zi < 0.05) mref = (R)P.rho_gas * v * pori;
    R rref = (P.dim == 2) ? mref / ((th / hd) * (th / hd)) : mref / v;
    W.rho_ref[i] = rref;
    R mn = mo, rn = ro;
    if (P.rho_type == 1) {
        rn = mref / v;
        mn = mref;
    }
    W.rho_new[i] = rn;
    W.m_new[i] = mn;
    rec.f1[i] = mk4<R>(mn, rn, S.temp[i], pori);
}

// contact history permutation, one thread per (slot, sphere): the writes of
// a slot plane are coalesced
__global__ void k_gather_history(int n, const int* __restrict__ perm, const int* __restrict__ hid_src,
                                 const double* __restrict__ hds_src, int* hid_dst, double* hds_dst) {
    grid_dep_wait();
    int q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= n * SPHDEM_NSLOT) return;
    int s = q / n, i = q - s * n;
    int p = perm[i];
    hid_dst[(size_t)s * n + i] = hid_src[(size_t)s * n + p];
#pragma unroll
    for (int c = 0; c < 3; c++) hds_dst[(size_t)(s * 3 + c) * n + i] = hds_src[(size_t)(s * 3 + c) * n + p];
}

// KERNEL_clc_prep3D_coupling_dem: functions_PREP2.cuh:3367-3523.
// One warp per DEM sphere; lanes stride over the candidate rows.
// G = 32: a warp per sphere; G = 1: a thread per sphere (2-D beds with many
// spheres); dem_thread_per_sphere in engine.cu.
template <typename R, int G>
__global__ void __launch_bounds__(128) k_dem_prep(DevParams P, SphState<R> S, SphRec<R> rec, DemState<double> D,
                                                  DemWork<double> DW, const int4* __restrict__ srows, const int4* __restrict__ drows) {
    static_assert(G == 32 || G == 1, "a warp or a thread per sphere");
    grid_dep_wait();
    const int i = G == 32 ? (int)((blockIdx.x * blockDim.x + threadIdx.x) >> 5)
                          : (int)(blockIdx.x * blockDim.x + threadIdx.x);
    const int lane = G == 32 ? (int)(threadIdx.x & 31) : 0;
    __shared__ int s_rows[4][20];   // 128 threads = 4 warps
    int* sm = s_rows[threadIdx.x >> 5];
    if (i >= P.nd) return;
    if (D.itype[i] > 2) return;
    int pti = D.ptype[i];
    double xi = D.x[i], yi = D.y[i], zi = D.z[i], hi = D.h[i];
    R th = (R)hi;
    Knl<R> K = knl_make<R>(P, th);
    double Rr = P.kappa * hi;
    Band bd = make_band(P, Rr);
    float r2l = r2_lo(Rr), r2h = r2_hi(Rr);
    PosRec<R> qp = make_pos<R>(P, xi, yi, zi, 0, 0, 0);
    int ic, jc, kc;
    cell_ijk(P, xi, yi, zi, ic, jc, kc);
    R f1 = 0, f3 = 0, por = 0;
    const Cull cu = make_cull(xi, yi, zi, Rr);
    // the sphere's SPH neighbours (p_type <= 1000, |x_i - x_j| < kappa h_i,
    // the add = 0 form that k_dem_coupling uses) into DW.nbs in visit order,
    // ranked by a ballot per round; the filter sums take their own subset
    // (p_type 1 or 3, the 1e-20 form)
    const unsigned lt = (1u << lane) - 1u;
    int cs = 0;
    auto dem_por = [&](int j) {
        if (D.ptype[j] <= 1000) return;
        PairT<R> g = pair_test<R>(xi, yi, zi, D.x[j], D.y[j], D.z[j], Rr, 1e-20, r2l, r2h);
        if (!g.in) return;
        R w = kw(K, g.r);
        R rj = (R)D.rad[j];
        por += w * dem_measure(P, rj);
    };
    if constexpr (G == 1) {
        // in visit order, one candidate after another
        for_stencil_j(P, ic, jc, kc, srows, cu, [&](int j) {
            const PosRec<R> qj = ldr(rec.pos + j);
            const int ptj = tag_ptype(qj.w);
            if (ptj > 1000) return;
            bool in = false, in20 = false;
            Disp<R> d;
            R r2 = 0;
            test_pair2(P, qp, qj, xi, yi, zi, S.x, S.y, S.z, j, Rr, bd, d, r2, in, in20);
            if (in) {
                if (cs < DEM_SPH_CAP) DW.nbs[(size_t)i * DEM_SPH_CAP + cs] = j;
                cs++;
            }
            if (!in20 || (ptj != 1 && ptj != 3)) return;
            R r, rinv;
            rdist(r2, r, rinv);
            V2<R> mr = ldr(rec.mr0 + j);
            R c = mr.x * rcp(mr.y) * kw(K, r);
            if (ptj == 1) f1 += c;
            else f3 += c;
        });
        DW.ncs[i] = cs;
        for_stencil_j(P, ic, jc, kc, drows, cu, dem_por);
    } else {
    for_rows_warp_all(P, ic, jc, kc, srows, cu, sm, lane, [&](int j) {
        bool in = false, in20 = false;
        int ptj = 0;
        Disp<R> d;
        R r2 = 0;
        if (j >= 0) {
            const PosRec<R> qj = ldr(rec.pos + j);
            ptj = tag_ptype(qj.w);
            if (ptj <= 1000) test_pair2(P, qp, qj, xi, yi, zi, S.x, S.y, S.z, j, Rr, bd, d, r2, in, in20);
        }
        const unsigned m = __ballot_sync(0xffffffffu, in);
        if (in) {
            const int pos = cs + __popc(m & lt);
            if (pos < DEM_SPH_CAP) DW.nbs[(size_t)i * DEM_SPH_CAP + pos] = j;
        }
        cs += __popc(m);
        if (!in20 || (ptj != 1 && ptj != 3)) return;
        R r, rinv;
        rdist(r2, r, rinv);
        V2<R> mr = ldr(rec.mr0 + j);
        R c = mr.x * rcp(mr.y) * kw(K, r);
        if (ptj == 1) f1 += c;
        else f3 += c;
    });
    if (lane == 0) DW.ncs[i] = cs;
    for_rows_warp(P, ic, jc, kc, drows, cu, sm, lane, dem_por);
    f1 = warp_sum(f1);
    f3 = warp_sum(f3);
    por = warp_sum(por);
    }
    if (lane == 0 && pti > 1000) {
        DW.flt_s[i] = f3;
        DW.flt_sd[i] = f1;
        DW.flt_sd2[i] = f1;
        DW.DEMpor[i] = (R)1 - (por / (f3 + f1 + (R)1.0e-20));
    }
}

// ---------------------------------------------------------------------------
// Sub-particle-scale eddy viscosity, the strain-rate branch of
// KERNEL_clc_prep3D_sph (functions_PREP2.cuh:2113-2118, 2166-2171), run
// with fv_solve and the SPS turbulence model only:
//   S_i = sum_j -m_j (rho_i + rho_j) |u_i - u_j|^2 / (2 rho_i rho_j r^2) (x_ij . grad W_ij)
// with the uncorrected kernel slope, and vis_t_i = (C_s L h_i)^2 max(S_i, 1e-20) rho_i
// (C_s = 0.12, L = 0.01, Parameters.cuh:102-104).  Pass B's viscous term
// reads vis_t of both particles of a pair, so this runs as its own pass
// just before it.
// ---------------------------------------------------------------------------
template <typename R, int KT>
__global__ void __launch_bounds__(128) k_sps(DevParams P, SphState<R> S, SphWork<R> W) {
    grid_dep_wait();
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    int n = P.ns;
    if (i >= n) return;
    if (S.itype[i] > 2 || S.ptype[i] > 1000) {
        W.vist[i] = 0;
        return;
    }
    const SphRec<R> rec = W.rec;
    R th = (R)S.h[i];
    Knl<R, KT> K = knl_make<R, KT>(P, th);
    PosRec<R> qi = ldr(rec.pos + i);
    V4<R> upi = rec.up[i];
    V4<R> fi = rec.f1[i];
    R uxi = upi.x, uyi = upi.y, uzi = upi.z, rhoi = fi.y;
    R irhoi = rcp(rhoi);
    int cnt = min(W.ncnt[i], P.nb_cap);
    R sr = 0;
    nb_walk<4, NbQ44<R>>(
        cnt, W.nbr, n, i,
        [&](int j) {
            NbQ44<R> t;
            t.q = ldr(rec.pos + j);
            t.a = ldr(rec.f1 + j);
            t.b = ldr(rec.up + j);
            return t;
        },
        [&](int j, const NbQ44<R>& t) {
            Disp<R> g = disp(P, qi, t.q, S.x, S.y, S.z, i, j);
            R r2 = g.dx * g.dx + g.dy * g.dy + g.dz * g.dz, r, rinv;
            rdist(r2, r, rinv);
            R dw = kdw(K, r) * rinv;
            R ux = uxi - t.b.x, uy = uyi - t.b.y, uz = uzi - t.b.z;
            R v = (R)-0.5 * t.a.x * (rhoi + t.a.y) * (ux * ux + uy * uy + uz * uz) * irhoi * rcp(t.a.y) * rinv * rinv;
            sr += v * r2 * dw;   // v (x_ij . x_ij) W'/r
        });
    sr = sr > (R)1e-20 ? sr : (R)1e-20;
    R cl = (R)0.12 * (th * (R)0.01);
    W.vist[i] = cl * cl * sr * rhoi;
}

// ---------------------------------------------------------------------------
// pass B: KERNEL_clc_prep3D_sph (functions_PREP2.cuh:1985-2227, Shepard
// filter) + KERNEL_advection_force3D_sph (functions_PPE2.cuh:1251-1607).
// The delta-SPH density gradient of prep3D is not formed: no kernel of the
// ISPH step reads it.
// ---------------------------------------------------------------------------
// FORCES: one of the interface-sharpness force, the repulsive boundary
// force, the SPS eddy viscosity or the inter-particle surface tension is on
// (a separate instantiation, so that the default pass keeps its registers)
template <typename R, bool FORCES, int KT, int SW>
__global__ void __launch_bounds__(128) k_passB(DevParams P, SphState<R> S, SphWork<R> W, const DevFlags* F) {
    grid_dep_wait();
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    int n = P.ns;
    if (i >= n) return;
    const SphRec<R> rec = W.rec;
    // Shepard filter every freq_filt*decouple_stride steps (functions_PREP2.cuh:2120)
    const int filt = (F->step_count % P.filt_period) == 0;
    int it = S.itype[i], pt = S.ptype[i], bt = S.btype[i];
    W.ftx[i] = 0; W.fty[i] = 0; W.ftz[i] = 0; W.ftot[i] = 0;
    W.pgfx[i] = 0; W.pgfy[i] = 0; W.pgfz[i] = 0;
    W.dtemp[i] = 0;
    if (it > 2 || pt > 1000) return;
    bool adv = !(P.open_bc > 0 && bt > 0) && pt < 1000 && pt > 0;
    if (!filt && !adv) return;
    R th = (R)S.h[i];
    Knl<R, KT> K = knl_make<R, KT>(P, th);
    PosRec<R> qi = ldr(rec.pos + i);
    V4<R> upi = rec.up[i];
    V4<R> fi = rec.f1[i];
    R uxi = upi.x, uyi = upi.y, uzi = upi.z, pi = upi.w;
    R rhoi = fi.y, tempi = fi.z, pori = fi.w, mi = fi.x;
    R irhoi = rcp(rhoi);
    const bool kgc = sw_on<SW>(SW_KGC, P.kgc == 1);
    Cm9<R> Cm = cm_load(W.Cm, n, i, kgc);
    R vis = (R)P.mu_gas, vis_h = (vis * vis) / (vis + vis);
    R kc = (R)P.k_sph;
    R eli = sw_on<SW>(SW_LAGR, P.sph_lagrangian != 0) ? (R)1 : (R)0;
    // per-particle factors of the pair terms
    R cp_i = -pori * irhoi * (rhoi / pori);      // rho_i/eps_i * (-eps_i / rho_i)
    R cv_i = vis_h * (R)4 * pori * irhoi;
    R visi = vis;
    if (FORCES && P.sps) visi += W.vist[i];   // viscosity + P3.vis_t (functions_PPE2.cuh:1323)
    R ch_i = (R)4 * pori * kc * kc * irhoi / (kc + kc);
    int cnt = min(W.ncnt[i], P.nb_cap);
    R flt = 0, tx = 0, ty = 0, tz = 0, px = 0, py = 0, pz = 0, Rc = 0, ex = 0, ey = 0, ez = 0, et = 0;
    const int* __restrict__ nb = W.nbr;
    nb_walk<4, NbQ44<R>>(
        cnt, nb, n, i,
        [&](int j) {
            NbQ44<R> t;
            t.q = ldr(rec.pos + j);
            t.a = ldr(rec.f1 + j);
            t.b = ldr(rec.up + j);
            return t;
        },
        [&](int j, const NbQ44<R>& t) {
            const V4<R>& fj = t.a;
            const V4<R>& uj = t.b;
            Disp<R> g = disp(P, qi, t.q, S.x, S.y, S.z, i, j);
            R r2 = g.dx * g.dx + g.dy * g.dy + g.dz * g.dz, r, rinv;
            rdist(r2, r, rinv);
            R mj = fj.x, irj = rcp(fj.y);
            if (filt) flt += mj * irj * kw(K, r);
            if (!adv || tag_ptype(t.q.w) >= 1000) return;
            R dw = kdw(K, r);
            R gx = dw * g.dx * rinv, gy = dw * g.dy * rinv, gz = dw * g.dz * rinv;
            cm_apply(Cm, kgc, gx, gy, gz);
            R tj = fj.z;
            if (sw_on<SW>(SW_FP, P.fp != 0)) {
                R s = cp_i * mj * (pi + uj.w) * irj;
                px += s * gx;
                py += s * gy;
                pz += s * gz;
            }
            if (sw_on<SW>(SW_FV, P.fv != 0)) {
                R cv = cv_i;
                if (FORCES && P.sps) {
                    // harmonic mean of the two particles' viscosity + vis_t
                    const R visj = vis + W.vist[j];
                    cv = visi * visj / (visi + visj) * (R)4 * pori * irhoi;
                }
                R Cv = (g.dx * gx + g.dy * gy + g.dz * gz) * cv * mj * irj * rinv * rinv;
                tx += Cv * (uxi - uj.x);
                ty += Cv * (uyi - uj.y);
                tz += Cv * (uzi - uj.z);
            }
            if (sw_on<SW>(SW_FVA, P.fva != 0)) {
                R uij = (uxi - uj.x) * g.dx + (uyi - uj.y) * g.dy + (uzi - uj.z) * g.dz;
                if (uij < (R)0) {
                    R hij = (th + th) * (R)0.5;
                    R phi = hij * uij / (r * r + (R)0.01 * hij * hij);
                    R Pij = mi * phi * ((R)-0.1 * (R)P.soundspeed + (R)0.02 * phi) / (rhoi + fj.y) * (R)0.5;
                    tx += -Pij * gx;
                    ty += -Pij * gy;
                    tz += -Pij * gz;
                }
            }
            if (FORCES) {
                const int ptj = tag_ptype(t.q.w);
                if (P.iface) {
                    // interface sharpness force (functions_PPE2.cuh:1450-1464): raw
                    // kernel slope; the neighbour's pressure only across a fluid-fluid
                    // interface (wall 0 and moving 9 excluded)
                    const bool flag = (pt != 0) && (pt != 9) && (ptj != 0) && (ptj != 9) && (pt != ptj);
                    const R mri = mi * irhoi, mrj = mj * irj;
                    R Ci = fabs(pi) * mri * mri + fabs(uj.w) * mrj * mrj * (R)flag;
                    Ci *= ((R)0.08 / mi) * dw * rinv;
                    tx += Ci * -g.dx;
                    ty += Ci * -g.dy;
                    tz += Ci * -g.dz;
                }
                if (P.fb && pt == 1 && ptj != 1) {
                    // repulsive force of non-fluid neighbours (functions_PPE2.cuh:1465-1472)
                    const R rr = r + (R)1e-10;
                    const R fb = (R)P.c_repulsive / rr / rr * kw(K, r) * ((R)2 * mj / (mi + mj));
                    tx += fb * g.dx;
                    ty += fb * g.dy;
                    tz += fb * g.dz;
                }
                if (P.ipf && pt == 1 && ptj == 1) {
                    // inter-particle surface tension (functions_PPE2.cuh:1490-1542): of the
                    // pair strengths of Parameters.cuh:134-148 only fluid-fluid (s_ff1 =
                    // 1.1e-6) is non-zero and every A is zero, so
                    // Cs = -s_ff1 w_ipf / (m_i (r + 1e-10)) with the cosine kernel
                    // w_ipf = -cos(3 pi / 4 r / h) for r < 2h (functions_INTERACTION.cuh:1-33)
                    const R tR = r * rcp(th);
                    const R wipf = tR < (R)2 ? -cos((R)(3.0 * 3.141592653 / 4.0) * tR) : (R)0;
                    const R Cs = -((R)1.1e-6 * (wipf / (mi * (r + (R)1e-10))));
                    tx += Cs * g.dx;
                    ty += Cs * g.dy;
                    tz += Cs * g.dz;
                }
            }
            if (eli < (R)1) {
                R mr = mj * irj * ((R)1 - eli);
                R ug = uxi * gx + uyi * gy + uzi * gz;
                ex += (uj.x - uxi) * ug * mr;
                ey += (uj.y - uyi) * ug * mr;
                ez += (uj.z - uzi) * ug * mr;
                if (sw_on<SW>(SW_CON, P.con != 0)) et += (tj - tempi) * ug * mr;
            }
            if (sw_on<SW>(SW_CON, P.con != 0)) Rc += ch_i * mj * (tempi - tj) * dw * irj * rcp(r + (R)1e-10);
        });
    if (filt) S.flt_s[i] = flt;
    if (!adv) return;
    if (P.fg) tz += -(R)P.g_sph;
    W.ftx[i] = tx - ex;
    W.fty[i] = ty - ey;
    W.ftz[i] = tz - ez;
    W.ftot[i] = sqrt(tx * tx + ty * ty + tz * tz);
    W.pgfx[i] = px;
    W.pgfy[i] = py;
    W.pgfz[i] = pz;
    if (sw_on<SW>(SW_CON, P.con != 0)) W.dtemp[i] = Rc / (R)P.cp_sph * (R)(pt != -1) - et;
}

// ---------------------------------------------------------------------------
// DEM contact: KERNEL_DEM_interaction3D_dem (functions_DEM_INTERACTION2.cuh:
// 888-1766).  The history lookup compares against the start-of-step slot
// ids held in registers; inserts pick the first slot that was free at the
// start of the step (so two new partners in one step share a slot, as in
// the reference).  Spring increments and overlap are FP64.
// ---------------------------------------------------------------------------
// G = 32: one warp per sphere (3-D beds: ~160 stencil candidates each);
// G = 1: one thread per sphere over its candidates in visit order (2-D beds
// with many spheres: a few candidates, which a warp would leave mostly
// idle).  The launch picks G from the configuration (dem_thread_per_sphere
// in engine.cu), so a bed always runs one form.
template <typename R, int G>
// 4 blocks of 128 per SM (128 registers, a few spilled): 0.145 -> 0.124 ms on
// the bench bed against the unbounded 162-register build
__global__ void __launch_bounds__(128, 4) k_dem_contact(DevParams P, DemState<double> D, DemWork<double> DW,
                                                     const int4* __restrict__ drows,
                                                     DevFlags* F) {
    static_assert(G == 32 || G == 1, "a warp or a thread per sphere");
    grid_dep_wait();
    // G = 32: lanes take candidates l, l+32, ... of the stencil in visit
    // order (for_rows_warp) and the pair terms are reduced with shuffles.
    // History writes keep the sequential semantics: lookups use the
    // start-of-step ids, a release clears only the partner's own slot, and
    // every new contact targets the first slot free at the start of the
    // step, so the new contact visited last wins that slot.
    const int i = G == 32 ? (int)((blockIdx.x * blockDim.x + threadIdx.x) >> 5)
                          : (int)(blockIdx.x * blockDim.x + threadIdx.x);
    const int lane = G == 32 ? (int)(threadIdx.x & 31) : 0;
    __shared__ int s_rows[4][20];
    int* sm = s_rows[threadIdx.x >> 5];
    const int n = P.nd;
    if (i >= n) return;
    if (lane == 0) {
        DW.ftx[i] = 0; DW.fty[i] = 0; DW.ftz[i] = 0;
        DW.tqx[i] = 0; DW.tqy[i] = 0; DW.tqz[i] = 0;
        DW.dtemp[i] = 0; DW.dtemp1[i] = 0; DW.dtemp2[i] = 0; DW.dtemp3[i] = 0;
    }
    if (D.itype[i] != 1 || D.ptype[i] <= 1000) return;
    // the contact mechanics run in FP64 in both builds (the state is FP64 and
    // stiff colliding contacts amplify rounding; 0.01 ms per step against R);
    // the radiation heat rate below is formed in R
    using Q = double;
    double xi = D.x[i], yi = D.y[i], zi = D.z[i], radi = D.rad[i];
    Q uxi = D.ux[i], uyi = D.uy[i], uzi = D.uz[i], wxi = D.wx[i], wyi = D.wy[i], wzi = D.wz[i];
    Q mi = D.m[i], rii = D.ri[i], rhoi = D.rho[i], tempi = D.temp[i];
    Q pri = (Q)P.nu_p, Gi = (Q)P.G, ymi = Gi * ((Q)2 * ((Q)1 + pri));
    Q ymij = (Q)1 / ((((Q)1 - pri * pri) / ymi) + (((Q)1 - pri * pri) / ymi));
    Q Gij = (Q)1 / ((((Q)2 - pri) / Gi) + (((Q)2 - pri) / Gi));
    Q cdamp = sqrt((Q)3.333333333) * (Q)P.damp;
    Q kci = (Q)P.k_dem, cpi = (Q)P.cp_dem;
    const R tiR = (R)tempi;
    const R emiR = (tiR >= (R)700) ? ((R)0.505586 + (R)7.92943e-4 * tiR - (R)5.228643e-7 * tiR * tiR +
                                      (R)1.10479e-10 * tiR * tiR * tiR)
                                   : (R)0.842337;
    Q radiR = (Q)radi;
    const Q imi = (Q)1 / mi, iradi = (Q)1 / radiR;   // hoisted reciprocals of the sphere's own terms
    Q dr2 = ((Q)1 / (Q)6) * radiR;
    Q volm = ((Q)4 / (Q)3) * (Q)3.141592 * (radiR * radiR * radiR - (radiR - dr2) * (radiR - dr2) * (radiR - dr2));
    int oid[SPHDEM_NSLOT];
    int free_slot = -1;
#pragma unroll
    for (int s = 0; s < SPHDEM_NSLOT; s++) {
        oid[s] = D.hid[s * n + i];
        if (free_slot < 0 && oid[s] < 1) free_slot = s;
    }
    int ic, jc, kc;
    cell_ijk(P, xi, yi, zi, ic, jc, kc);
    Q tx = 0, ty = 0, tz = 0, tqx = 0, tqy = 0, tqz = 0, dtr = 0, dtc = 0;
    const double kdt = P.dt;
    // this lane's last new contact (visit order t) and its spring
    int new_t = -1, new_id = 0;
    double new_dx = 0, new_dy = 0, new_dz = 0;
    int t_visit = lane - G;
    const Cull cu = make_cull(xi, yi, zi, P.r_search * radi);
    auto pair = [&](int j) {
        t_visit += G;
        if (D.ptype[j] <= 1000) return;
        double xj = D.x[j], yj = D.y[j], zj = D.z[j], radj = D.rad[j];
        double td = pair_dist(xi, yi, zi, xj, yj, zj);
        if (!(td < P.r_search * radi && td > 0.0)) return;
        double ovlp = radi + radj - td;
        int demj = D.dem_idx[j];
        Q radjR = (Q)radj;
        Q radij = (Q)1 / (iradi + (Q)1 / radjR);
        Q tdR = (Q)td;
        if (P.con) {
            // radiation between spheres within the search range (functions_DEM_INTERACTION2.cuh:
            // 1080-1194): a heat rate, formed in the field precision R
            const R ti = (R)tempi, tj = (R)D.temp[j];
            const R riR = (R)radiR, rjR = (R)radjR, rijR = (R)radij, tdF = (R)tdR;
            R emj = (tj >= (R)700) ? ((R)0.505586 + (R)7.92943e-4 * tj - (R)5.228643e-7 * tj * tj +
                                      (R)1.10479e-10 * tj * tj * tj)
                                   : (R)0.842337;
            const R itdF = rcp(tdF);
            R ai = riR * itdF, aj = rjR * itdF, dij = aj - ai;
            R dc_r = (R)0.56 * ((R)2 * rijR);
            R dc_ar = (R)3.14159 * dc_r * dc_r;
            R dmax = (R)0.5 * (sqrt((R)1 + (R)4 * dc_ar / ((R)3.14159 * tdF * tdF * ((R)1 - dij * dij))) - dij);
            R ci = ((R)1 - dij * dij) / ((R)2 * dmax) - dij;
            R cj = ((R)1 - dij * dij) / ((R)2 * (dmax + dij)) + dij;
            R si = sqrt((R)1 - ci * ci), sj = sqrt((R)1 - cj * cj);
            R ri_cr = riR * si, rj_cr = rjR * sj;
            R td_cr = tdF - riR * ci - rjR * cj;
            R z_cr = (R)1 + ((R)4 * rj_cr * rj_cr + td_cr * td_cr) / (ri_cr * ri_cr);
            R F_cr = (R)0.5 * (z_cr - sqrt(z_cr * z_cr - (R)4 * rj_cr * rj_cr / (ri_cr * ri_cr)));
            R F_ij = ((R)1 + ci) * F_cr * (R)0.5;
            R ar_i = (R)2 * (R)3.14159 * riR * riR * ((R)1 - ci);
            R ar_j = (R)2 * (R)3.14159 * rjR * rjR * ((R)1 - cj);
            R arr = ar_j / ar_i;
            R Y = F_ij + ((R)1 - F_ij) * (arr / ((R)1 + arr));
            R einv = ((R)1 - emiR) / (emiR * ar_i) + ((R)1 - emj) / (emj * ar_j) + (R)1 / (Y * ar_i);
            // Ti^4 - Tj^4; in FP32 as (Ti - Tj)(Ti + Tj)(Ti^2 + Tj^2), which keeps the
            // relative precision of a difference of nearly equal temperatures
            R d4;
            if constexpr (sizeof(R) == 4) d4 = (ti - tj) * (ti + tj) * (ti * ti + tj * tj);
            else d4 = ti * ti * ti * ti - tj * tj * tj * tj;
            dtr += (Q)(-(R)5.6704e-8 * d4 / (einv * ((R)rhoi * (R)volm) * (R)cpi));
        }
        if (!(td < P.r_contact * radi)) return;
        int slot = -1;
#pragma unroll
        for (int s = 0; s < SPHDEM_NSLOT; s++)
            if (slot < 0 && oid[s] == demj) slot = s;
        if (td > 0 && ovlp > 0) {
            Q tov = (Q)ovlp;
            if (P.con) {
                Q kij = (Q)1 / ((Q)1 / kci + (Q)1 / kci);
                dtc += -(Q)4 * kij * sqrt(((Q)2 * tov) * (radij - (Q)0.5 * tov)) * (tempi - D.temp[j]) /
                       ((rhoi * volm) * cpi);
            }
            double dsx = 0, dsy = 0, dsz = 0;
            if (slot >= 0) {
                dsx = D.hds[(slot * 3 + 0) * n + i];
                dsy = D.hds[(slot * 3 + 1) * n + i];
                dsz = D.hds[(slot * 3 + 2) * n + i];
            }
            Q mj = D.m[j];
            const Q itd = (Q)1 / (Q)td;
            Q nx = (Q)(xj - xi) * itd, ny = (Q)(yj - yi) * itd, nz = (Q)(zj - zi) * itd;
            Q li = radiR - (Q)0.5 * tov, lj = radjR - (Q)0.5 * tov;
            Q rcxi = li * nx, rcyi = li * ny, rczi = li * nz;
            Q rcxj = -lj * nx, rcyj = -lj * ny, rczj = -lj * nz;
            Q wxj = D.wx[j], wyj = D.wy[j], wzj = D.wz[j];
            Q urxi = wyi * rczi - wzi * rcyi, uryi = wzi * rcxi - wxi * rczi, urzi = wxi * rcyi - wyi * rcxi;
            Q urxj = wyj * rczj - wzj * rcyj, uryj = wzj * rcxj - wxj * rczj, urzj = wxj * rcyj - wyj * rcxj;
            Q urx = (D.ux[j] + urxj) - (uxi + urxi);
            Q ury = (D.uy[j] + uryj) - (uyi + uryi);
            Q urz = (D.uz[j] + urzj) - (uzi + urzi);
            Q unm = nx * urx + ny * ury + nz * urz;
            Q unx = unm * nx, uny = unm * ny, unz = unm * nz;
            Q usx = urx - unx, usy = ury - uny, usz = urz - unz;
            dsx += (double)usx * kdt;
            dsy += (double)usy * kdt;
            dsz += (double)usz * kdt;
            const Q iusm = (Q)1 / (sqrt(usx * usx + usy * usy + usz * usz) + (Q)1e-20);
            Q sx = usx * iusm, sy = usy * iusm, sz = usz * iusm;
            Q mij = (Q)1 / (imi + (Q)1 / mj);
            Q sq = sqrt(radij * tov);   // sqrt(R* delta): also stands for sqrt(R*) sqrt(delta)
            Q Cspr = (Q)1.33333 * ymij * sq * tov * imi;
            Q Cspr_s = (Q)8 * Gij * sq * imi;
            Q Kn = (Q)2 * ymij * sq;
            Q Cd = cdamp * sqrt(mij * Kn) * imi;
            Q Cds = cdamp * sqrt(mij * Cspr_s * mi) * imi;
            tx += Cspr * -nx;
            ty += Cspr * -ny;
            tz += Cspr * -nz;
            tx += Cd * unx;
            ty += Cd * uny;
            tz += Cd * unz;
            Q fssx = Cspr_s * (Q)dsx + Cds * usx;
            Q fssy = Cspr_s * (Q)dsy + Cds * usy;
            Q fssz = Cspr_s * (Q)dsz + Cds * usz;
            Q sgx = (fssx >= (Q)0) ? (Q)1 : (Q)-1;
            Q sgy = (fssy >= (Q)0) ? (Q)1 : (Q)-1;
            Q sgz = (fssz >= (Q)0) ? (Q)1 : (Q)-1;
            // stick while |f_spring| < |f_friction| (the squares compare the same way)
            Q mfss2 = fssx * fssx + fssy * fssy + fssz * fssz;
            Q fr = (Q)P.fric * Cspr;
            Q ffx = fr * sx, ffy = fr * sy, ffz = fr * sz;
            Q mfsf2 = ffx * ffx + ffy * ffy + ffz * ffz;
            bool stick = mfss2 < mfsf2;
            Q fsx = stick ? fssx : sgx * fabs(ffx);
            Q fsy = stick ? fssy : sgy * fabs(ffy);
            Q fsz = stick ? fssz : sgz * fabs(ffz);
            tx += fsx;
            ty += fsy;
            tz += fsz;
            tqx += mi * (rcyi * fsz - rczi * fsy);
            tqy += mi * (rczi * fsx - rcxi * fsz);
            tqz += mi * (rcxi * fsy - rcyi * fsx);
            if (slot >= 0) {
                // existing partner: its own slot, no other pair touches it
                D.hid[slot * n + i] = demj;
                D.hds[(slot * 3 + 0) * n + i] = dsx;
                D.hds[(slot * 3 + 1) * n + i] = dsy;
                D.hds[(slot * 3 + 2) * n + i] = dsz;
            } else {
                new_t = t_visit;
                new_id = demj;
                new_dx = dsx;
                new_dy = dsy;
                new_dz = dsz;
            }
        } else if (slot >= 0) {
            D.hds[(slot * 3 + 0) * n + i] = 0.0;
            D.hds[(slot * 3 + 1) * n + i] = 0.0;
            D.hds[(slot * 3 + 2) * n + i] = 0.0;
            D.hid[slot * n + i] = 0;
        }
    };
    if constexpr (G == 32) for_rows_warp(P, ic, jc, kc, drows, cu, sm, lane, pair);
    else for_stencil_j(P, ic, jc, kc, drows, cu, pair);
    // the new contact visited last takes the first slot free at the start
    int last_t = new_t;
    if constexpr (G == 32) {
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) last_t = max(last_t, __shfl_xor_sync(0xffffffffu, last_t, o));
    }
    if (last_t >= 0 && new_t == last_t) {
        // no free slot (a 17th partner): flag it; the new contact acted this
        // step and is not recorded (the reference writes through an unset
        // slot index here, functions_DEM_INTERACTION2.cuh:1567)
        const int slot = free_slot;
        if (slot < 0) {
            atomicOr(&F->overflow, 2);
        } else {
            D.hid[slot * n + i] = new_id;
            D.hds[(slot * 3 + 0) * n + i] = new_dx;
            D.hds[(slot * 3 + 1) * n + i] = new_dy;
            D.hds[(slot * 3 + 2) * n + i] = new_dz;
        }
    }
    if constexpr (G == 32) {
        tx = warp_sum(tx); ty = warp_sum(ty); tz = warp_sum(tz);
        tqx = warp_sum(tqx); tqy = warp_sum(tqy); tqz = warp_sum(tqz);
        dtr = warp_sum(dtr); dtc = warp_sum(dtc);
    }
    if (lane != 0) return;
    if (P.fg) tz += -(Q)P.g_dem;
    if (P.con) {
        Q temp1i = D.temp1[i], temp2i = D.temp2[i], temp3i = D.temp3[i];
        Q a0 = kci / (rhoi * cpi);
        Q dr1 = ((Q)5 / (Q)6) * radiR / (Q)3;
        Q A = ((Q)2 * kci / dr1) / ((Q)2 * kci / dr1 + kci / dr2), B = (Q)1 - A;
        Q ts = A * temp1i + B * tempi;
        Q d0 = (Q)2 * (a0 / radiR) * (tempi - ts) / ((Q)2 * dr2) + a0 * (tempi - (Q)2 * tempi + ts) / (dr2 * dr2);
        Q d1 = ((Q)2 * a0 / ((Q)2.5 * dr1)) * ((Q)2 * ts - temp1i - temp2i) / ((Q)2 * dr1) +
               a0 * ((Q)2 * ts - (Q)3 * temp1i + temp2i) / (dr1 * dr1);
        Q d2 = (Q)2 * (a0 / ((Q)1.5 * dr1)) * (temp1i - temp3i) / ((Q)2 * dr1) +
               a0 * (temp1i - (Q)2 * temp2i + temp3i) / (dr1 * dr1);
        Q d3 = (Q)2 * (a0 / ((Q)0.5 * dr1)) * ((temp2i - temp3i) / ((Q)2 * dr1)) + a0 * (temp2i - temp3i) / (dr1 * dr1);
        DW.dtemp[i] = d0 + dtr + dtc;
        DW.dtemp1[i] = d1;
        DW.dtemp2[i] = d2;
        DW.dtemp3[i] = d3;
    }
    DW.ftx[i] = tx;
    DW.fty[i] = ty;
    DW.ftz[i] = tz;
    DW.tqx[i] = tqx / rii;
    DW.tqy[i] = tqy / rii;
    DW.tqz[i] = tqz / rii;
}

// ---------------------------------------------------------------------------
// KERNEL_DEM_coupling3D_dem (functions_SPH_DEM_COUPLING2.cuh:627-1129) with
// KERNEL_clc_projection_dem (functions_TIME_ISPH2.cuh:206-308) fused into its
// epilogue (the predictor only needs this particle's force).  The pair sums
// of one sphere over its SPH neighbours (dc_pair) are formed by a warp --
// lanes over the candidates, partial sums reduced with shuffles -- and one
// lane runs the drag closure and the predictor (dem_coupling_finish).
// ---------------------------------------------------------------------------
template <typename R>
struct DcSums {
    R tx, ty, tz, ufx, ufy, ufz, uax, uay, uaz, por, ttf, tta;
    R wtf, wta;   // the weights of ttf/tta: their SPH temperatures are stored as T - t_ref
    int has_f, has_a;
};

// one SPH neighbour j of sphere i at distance r (the pair already passed the
// kappa h_i test): Shepard sums of fluid/air velocity, temperature and
// porosity, and the pressure-gradient force
template <typename R, int KT>
__device__ __forceinline__ void dc_pair(const SphWork<R>& W, const Knl<R, KT>& K, R ff, R fa, R pgc, int j, int ptj, R r,
                                        DcSums<R>& a) {
    const V4<R> fj = ldr(W.rec.f1 + j);
    const R porj = fj.w;
    if (!(porj < (R)1)) return;
    R w = kw(K, r);
    R mj = fj.x, rhoj = fj.y, c = mj * w * rcp(rhoj);
    if ((ptj == 1 && ff > (R)0.000001) || (ptj == 3 && fa > (R)0.000001)) {
        V4<R> uj = ldr(W.rec.up + j);
        if (ptj == 1) {
            a.has_f = 1;
            a.ufx += uj.x * c; a.ufy += uj.y * c; a.ufz += uj.z * c;
            a.ttf += fj.z * c;
            a.wtf += c;
        } else {
            a.has_a = 1;
            a.uax += uj.x * c; a.uay += uj.y * c; a.uaz += uj.z * c;
            a.tta += fj.z * c;
            a.wta += c;
        }
        a.por += porj * c;
    }
    if (ptj != 0 && ptj != 9 && ptj != -3 && ptj != 3 && ff > (R)0.01) {
        R q = c * pgc;
        a.tx += W.pgfx[j] * q;
        a.ty += W.pgfy[j] * q;
        a.tz += W.pgfz[j] * q;
    }
}

template <typename R>
__device__ __forceinline__ void dc_warp_sum(DcSums<R>& a) {
    a.tx = warp_sum(a.tx); a.ty = warp_sum(a.ty); a.tz = warp_sum(a.tz);
    a.ufx = warp_sum(a.ufx); a.ufy = warp_sum(a.ufy); a.ufz = warp_sum(a.ufz);
    a.uax = warp_sum(a.uax); a.uay = warp_sum(a.uay); a.uaz = warp_sum(a.uaz);
    a.por = warp_sum(a.por); a.ttf = warp_sum(a.ttf); a.tta = warp_sum(a.tta);
    a.wtf = warp_sum(a.wtf); a.wta = warp_sum(a.wta);
    a.has_f = __any_sync(0xffffffffu, a.has_f);
    a.has_a = __any_sync(0xffffffffu, a.has_a);
}

// drag closure on the reduced sums (when coupled) and the DEM predictor
template <typename R>
__device__ void dem_coupling_finish(const DevParams& P, DemState<double>& D, DemWork<double>& DW, int i, bool coupled,
                                    const DcSums<R>& a) {
    using Q = double;   // the DEM set is FP64: the closure and the predictor run in FP64
    const int pt = D.ptype[i];
    Q uxi = D.ux[i], uyi = D.uy[i], uzi = D.uz[i];
    Q ftx = DW.ftx[i], fty = DW.fty[i], ftz = DW.ftz[i];
    if (coupled) {
        Q radi = (Q)D.rad[i], di = (Q)2 * radi;
        Q mi = D.m[i], rhoi = D.rho[i], tempi = D.temp[i];
        Q fa = DW.flt_s[i], ff = DW.flt_sd[i];
        const Q tx = a.tx, ty = a.ty, tz = a.tz, ufx = a.ufx, ufy = a.ufy, ufz = a.ufz;
        const Q uax = a.uax, uay = a.uay, uaz = a.uaz, por = a.por, ttf = a.ttf, tta = a.tta;
        const int has_f = a.has_f, has_a = a.has_a;
        Q rho_f = has_f ? (Q)P.rho_gas : (Q)0, rho_a = has_a ? (Q)P.rho_gas : (Q)0;
        Q ki = (radi < (Q)0.0012) ? (Q)55.0 : (Q)0.84;
        Q ali = (radi < (Q)0.0012) ? (Q)1.77e-5 : (Q)2.5e-6;
        Q cpi = ki / (ali * rhoi);
        Q eps = (Q)1.0e-15;
        Q pori = por / (ff + eps);
        Q ux_f = ufx / (ff + eps) - uxi, uy_f = ufy / (ff + eps) - uyi, uz_f = ufz / (ff + eps) - uzi;
        // the SPH temperatures in ttf/tta are stored as T - t_ref: absolute sums
        const Q tr = (Q)P.t_ref;
        const Q ttfa = ttf + tr * (Q)a.wtf, ttaa = tta + tr * (Q)a.wta;
        Q tf = ttfa / (ff + eps) - tempi;
        Q ux_a = uax / (fa + eps) - uxi, uy_a = uay / (fa + eps) - uyi, uz_a = uaz / (fa + eps) - uzi;
        Q ta = ttaa / (fa + eps) - tempi;
        Q ux_fa = (ufx + uax) / (ff + fa + eps) - uxi, uy_fa = (ufy + uay) / (ff + fa + eps) - uyi,
          uz_fa = (ufz + uaz) / (ff + fa + eps) - uzi;
        Q tfa = (ttfa + ttaa) / (ff + fa + eps) - tempi;
        Q f_fluid = ff / (ff + fa + eps), f_air = fa / (ff + fa + eps);
        Q mf = sqrt(ux_f * ux_f + uy_f * uy_f + uz_f * uz_f);
        DW.magf[i] = mf;
        Q ma = sqrt(ux_a * ux_a + uy_a * uy_a + uz_a * uz_a);
        Q mfa = sqrt(ux_fa * ux_fa + uy_fa * uy_fa + uz_fa * uz_fa);
        Q dfx = 0, dfy = 0, dfz = 0, dax = 0, day = 0, daz = 0, dq = 0;
        Q a_ht = (Q)6 / di;
        Q nu = (Q)P.nu_gas;
        DW.DEMpor[i] = pori;
        // the Di Felice closure (functions_SPH_DEM_COUPLING2.cuh:979-1009) in the
        // field precision R: an empirical coefficient, applied to the FP64 slip
        const R diR = (R)di, poriR = (R)pori, miR = (R)mi, nuR = (R)nu, epsR = (R)1.0e-15;
        const R mfR = (R)mf, maR = (R)ma, mfaR = (R)mfa, kiR = (R)ki, ahtR = (R)a_ht;
        if (mf > (Q)1.0e-8 && (ff + fa) > (Q)0.00001 && f_fluid > (Q)0.65) {
            R Re = diR * mfR * poriR / (nuR + epsR);
            R q = (R)0.63 + (R)4.8 / sqrt(Re);
            R Cdf = q * q;
            R lr = (R)1.5 - log10(Re);
            R bf = (R)3.7 - (R)0.65 * exp(-lr * lr / (R)2);
            R c = ((R)1 / (R)8) * Cdf * (R)rho_f * (R)3.14159 * diR * diR * mfR * pow(poriR, (R)2 - bf) / miR;
            dfx = c * ux_f; dfy = c * uy_f; dfz = c * uz_f;
            dq = (Q)(((R)2 + (R)0.6 * sqrt(Re)) * (R)0.0518 / diR * ahtR) * tf;
            D.Fdx_df[i] = dfx;
            D.Fdy_df[i] = dfy;
            D.Fdz_df[i] = dfz;
        }
        if (ma > (Q)1.0e-8 && (ff + fa) > (Q)0.00001 && f_air > (Q)0.65) {
            R Re = diR * poriR * maR / (nuR + epsR);
            R q = (R)0.63 + (R)4.8 / sqrt(Re);
            R lr = (R)1.5 - log10(Re);
            R b = (R)2.65 * ((R)1 + poriR) - ((R)5.3 - (R)3.5 * poriR) * poriR * poriR * exp(-lr * lr / (R)2);
            R c = ((R)1 / (R)8) * q * q * (R)rho_a * (R)3.14159 * diR * diR * maR * pow(poriR, (R)-1 - b) / miR;
            dax = c * ux_a; day = c * uy_a; daz = c * uz_a;
            dq = (Q)(((R)2 + (R)0.6 * sqrt(Re)) * kiR / diR * ahtR) * ta;
        }
        if ((ma > (Q)1.0e-8 || mf > (Q)1.0e-8) && (ff + fa) > (Q)0.00001 && f_air <= (Q)0.65 && f_fluid <= (Q)0.65) {
            R rfa = (R)P.rho_gas * (R)f_air + (R)P.rho_liquid * (R)f_fluid;
            R vfa = (R)P.mu_gas * (R)f_air + (R)P.mu_liquid * (R)f_fluid;
            R vk = vfa / (rfa + epsR);
            R Re = diR * poriR * mfaR / (vk + epsR);
            R q = (R)0.63 + (R)4.8 / sqrt(Re);
            R lr = (R)1.5 - log10(Re);
            R b = (R)2.65 * ((R)1 + poriR) - ((R)5.3 - (R)3.5 * poriR) * poriR * poriR * exp(-lr * lr / (R)2);
            R c = ((R)1 / (R)8) * q * q * rfa * (R)3.14159 * diR * diR * mfaR * pow(poriR, (R)-1 - b) / miR;
            dax = c * ux_fa; day = c * uy_fa; daz = c * uz_fa;
            dq = (Q)(((R)2 + (R)0.6 * sqrt(Re)) * kiR / diR * ahtR) * tfa;
        }
        ftx = ftx + dfx / pori + tx;
        fty = fty + dfy / pori + ty;
        ftz = ftz + dfz / pori + tz;
        DW.ftx[i] = ftx;
        DW.fty[i] = fty;
        DW.ftz[i] = ftz;
        if (P.con) {
            DW.dtemp[i] = dq / (rhoi * cpi);
            D.Q_sd[i] = dq * mi / rhoi;
        }
        DW.Fdx_da[i] = dax; DW.Fdy_da[i] = day; DW.Fdz_da[i] = daz;
        DW.Fdx_b[i] = tx; DW.Fdy_b[i] = ty; DW.Fdz_b[i] = tz;
    }
    // predictor (DEM): u* = u + f dt
    DW.ux0[i] = uxi; DW.uy0[i] = uyi; DW.uz0[i] = uzi;
    if (pt == 9) {
        D.ux[i] = (Q)P.ball_vel; D.uy[i] = (Q)0; D.uz[i] = (Q)0;
        DW.ux0[i] = (Q)P.ball_vel; DW.uy0[i] = (Q)0; DW.uz0[i] = (Q)0;
    } else if (pt >= 0) {
        Q b = (Q)(D.btype[i] == 0);
        Q dt = (Q)P.dt;
        D.ux[i] = uxi + ftx * b * dt;
        D.uy[i] = uyi + fty * b * dt;
        D.uz[i] = uzi + ftz * b * dt;
    }
    if (P.con && pt > 0) DW.temp0[i] = D.temp[i];
}

// G = 32: a warp per sphere; G = 1: a thread per sphere (2-D beds with many
// spheres, ~20 SPH neighbours each); dem_thread_per_sphere in engine.cu.
template <typename R, int KT, int G>
__global__ void __launch_bounds__(128) k_dem_coupling(DevParams P, SphState<R> S, SphWork<R> W, DemState<double> D,
                                                      DemWork<double> DW, const int4* __restrict__ srows) {
    static_assert(G == 32 || G == 1, "a warp or a thread per sphere");
    grid_dep_wait();
    const int i = G == 32 ? (int)((blockIdx.x * blockDim.x + threadIdx.x) >> 5)
                          : (int)(blockIdx.x * blockDim.x + threadIdx.x);
    const int lane = G == 32 ? (int)(threadIdx.x & 31) : 0;
    __shared__ int s_rows[4][20];   // 128 threads = 4 warps
    int* sm = s_rows[threadIdx.x >> 5];
    if (i >= P.nd) return;
    int it = D.itype[i], pt = D.ptype[i];
    if (it > 2) {
        if (lane == 0) DW.dcf[i] = -1;   // k_dem_finish skips it
        return;
    }
    DcSums<R> a{};
    const bool coupled = it == 1 && pt > 1000;
    if (coupled) {
        const SphRec<R> rec = W.rec;
        double xi = D.x[i], yi = D.y[i], zi = D.z[i], hi = D.h[i];
        R radi = (R)D.rad[i], voli = ((R)4 / (R)3) * (R)3.14159 * radi * radi * radi;
        R mi = D.m[i];
        R fa = DW.flt_s[i], ff = DW.flt_sd[i];
        R th = (R)hi;
        Knl<R, KT> K = knl_make<R, KT>(P, th);
        double Rr = P.kappa * hi;
        Band bd = make_band(P, Rr);
        PosRec<R> qp = make_pos<R>(P, xi, yi, zi, 0, 0, 0);
        int ic, jc, kc;
        cell_ijk(P, xi, yi, zi, ic, jc, kc);
        R pgc = voli / (mi * ff + (R)1.0e-15);
        auto pair = [&](int j) {
            PosRec<R> qj = ldr(rec.pos + j);
            int ptj = tag_ptype(qj.w);
            if (ptj > 1000) return;
            Disp<R> d;
            R r2;
            if (!test_pair(P, qp, qj, xi, yi, zi, S.x, S.y, S.z, j, Rr, 0.0, bd, d, r2)) return;
            R r, rinv;
            rdist(r2, r, rinv);
            dc_pair(W, K, ff, fa, pgc, j, ptj, r, a);
        };
        // the neighbours k_dem_prep listed (same positions, same predicate);
        // a sphere with more than the list holds walks its stencil
        const int cs = DW.ncs[i];
        if (cs <= DEM_SPH_CAP) {
            const int* __restrict__ nbs = DW.nbs + (size_t)i * DEM_SPH_CAP;
            for (int k = lane; k < cs; k += G) pair(__ldg(nbs + k));
        } else {
            const Cull cu = make_cull(xi, yi, zi, Rr);
            if constexpr (G == 32) for_rows_warp(P, ic, jc, kc, srows, cu, sm, lane, pair);
            else for_stencil_j(P, ic, jc, kc, srows, cu, pair);
        }
        if constexpr (G == 32) dc_warp_sum(a);
    }
    if (lane != 0) return;
    // the closure and the predictor run in k_dem_finish (thread per sphere),
    // so this pair pass keeps the registers of the FP32 sums only
    const int nd = P.nd;
    double* o = DW.dcs;
    o[0 * nd + i] = a.tx; o[1 * nd + i] = a.ty; o[2 * nd + i] = a.tz;
    o[3 * nd + i] = a.ufx; o[4 * nd + i] = a.ufy; o[5 * nd + i] = a.ufz;
    o[6 * nd + i] = a.uax; o[7 * nd + i] = a.uay; o[8 * nd + i] = a.uaz;
    o[9 * nd + i] = a.por; o[10 * nd + i] = a.ttf; o[11 * nd + i] = a.tta;
    o[12 * nd + i] = a.wtf; o[13 * nd + i] = a.wta;
    DW.dcf[i] = (coupled ? 1 : 0) | (a.has_f ? 2 : 0) | (a.has_a ? 4 : 0);
}

// the drag closure and the DEM predictor of every sphere the pair pass
// reached (dcf >= 0), on the sums it left in DW.dcs
template <typename R>
__global__ void __launch_bounds__(128) k_dem_finish(DevParams P, DemState<double> D, DemWork<double> DW) {
    grid_dep_wait();
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int nd = P.nd;
    if (i >= nd) return;
    const int f = DW.dcf[i];
    if (f < 0) return;
    const double* o = DW.dcs;
    DcSums<R> a;
    a.tx = (R)o[0 * nd + i]; a.ty = (R)o[1 * nd + i]; a.tz = (R)o[2 * nd + i];
    a.ufx = (R)o[3 * nd + i]; a.ufy = (R)o[4 * nd + i]; a.ufz = (R)o[5 * nd + i];
    a.uax = (R)o[6 * nd + i]; a.uay = (R)o[7 * nd + i]; a.uaz = (R)o[8 * nd + i];
    a.por = (R)o[9 * nd + i]; a.ttf = (R)o[10 * nd + i]; a.tta = (R)o[11 * nd + i];
    a.wtf = (R)o[12 * nd + i]; a.wta = (R)o[13 * nd + i];
    a.has_f = (f >> 1) & 1;
    a.has_a = (f >> 2) & 1;
    dem_coupling_finish(P, D, DW, i, (f & 1) != 0, a);
}

// ---------------------------------------------------------------------------
// KERNEL_SPH_coupling3D_sph (functions_SPH_DEM_COUPLING2.cuh:1815-2019) +
// KERNEL_clc_projection_sph (functions_TIME_ISPH2.cuh:104-204).
// ---------------------------------------------------------------------------
template <typename R, int KT>
__global__ void __launch_bounds__(128) k_sph_coupling(DevParams P, SphState<R> S, SphWork<R> W, DemState<double> D,
                                                      DemWork<double> DW, const int4* __restrict__ drows, int time_zero) {
    grid_dep_wait();
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    int n = P.ns;
    if (i >= n) return;
    int it = S.itype[i], pt = S.ptype[i];
    if (it > 2) return;
    R ftx = W.ftx[i], fty = W.fty[i], ftz = W.ftz[i];
    if (it == 1 && pt <= 1000) {
        double xi = S.x[i], yi = S.y[i], zi = S.z[i], hi = S.h[i];
        R rhoi = W.rho_new[i], tempi = S.temp[i];
        // heat_capacity(ptypei, tempi): the reference passes the arguments
        // swapped (functions_SPH_DEM_COUPLING2.cuh:1860)
        R cpi = (abs((int)(tempi + (R)P.t_ref)) > 1000) ? (R)P.cp_dem : (R)P.cp_sph;   // stored T - t_ref
        R th = (R)hi;
        Knl<R, KT> K = knl_make<R, KT>(P, th);
        double Rr = P.kappa * hi;
        R tx = 0, ty = 0, tz = 0, tt = 0;
        if (P.nd > 0 && (pt == 1 || pt == 3)) {
            float r2l = r2_lo(Rr), r2h = r2_hi(Rr);
            auto dem = [&](int j) {
                if (D.ptype[j] <= 1000) return;
                PairT<R> g = pair_test<R>(xi, yi, zi, D.x[j], D.y[j], D.z[j], Rr, 0.0, r2l, r2h);
                if (!g.in) return;
                R ffj = (R)DW.flt_sd2[j] + (R)DW.flt_s[j];
                if (!(ffj > (R)0)) return;
                R w = kw(K, g.r);
                if (P.dim == 2) w *= (R)0.75 / (R)D.rad[j];   // per unit depth (depth 4 r / 3)
                R c = w / (ffj + (R)1.0e-20);
                R mr = (R)D.m[j] / rhoi;
                tx += -mr * (R)D.Fdx_df[j] * c;
                ty += -mr * (R)D.Fdy_df[j] * c;
                tz += -mr * (R)D.Fdz_df[j] * c;
                tt += -(R)D.Q_sd[j] / (rhoi * cpi) * c;
            };
            const int cd = W.ncntd[i];
            if (cd <= P.nbd_cap) {
                for (int k = 0; k < cd; k++) dem(W.nbrd[(size_t)k * n + i]);
            } else {
                int ic, jc, kc;
                cell_ijk(P, xi, yi, zi, ic, jc, kc);
                for_stencil_j(P, ic, jc, kc, drows, make_cull(xi, yi, zi, Rr), dem);
            }
        }
        ftx += tx;
        fty += ty;
        ftz += tz;
        W.ftx[i] = ftx;
        W.fty[i] = fty;
        W.ftz[i] = ftz;
        W.ftot[i] = sqrt(ftx * ftx + fty * fty + ftz * ftz);
        if (P.con) W.dtemp[i] += tt;
    }
    // predictor (SPH), KERNEL_clc_projection_sph; u* also goes to the
    // {u, p} record the PPE reads
    R uxi = S.ux[i], uyi = S.uy[i], uzi = S.uz[i];
    W.ux0[i] = uxi; W.uy0[i] = uyi; W.uz0[i] = uzi;
    R usx = uxi, usy = uyi, usz = uzi;
    if (pt == 9) {
        usx = (R)P.ball_vel; usy = (R)0; usz = (R)0;
        W.ux0[i] = (R)P.ball_vel; W.uy0[i] = (R)0; W.uz0[i] = (R)0;
    } else if (pt >= 0) {
        R b = (R)(S.btype[i] == 0);
        R dt = (R)P.sdt;
        usx = uxi + ftx * b * dt;
        usy = uyi + fty * b * dt;
        usz = uzi + ftz * b * dt;
    }
    S.ux[i] = usx; S.uy[i] = usy; S.uz[i] = usz;
    W.rec.up[i] = mk4<R>(usx, usy, usz, S.pres[i]);
    if (time_zero) W.rho_ref[i] = W.rho_new[i];
    if (P.con && pt > 0) W.temp0[i] = S.temp[i];
}

// ---------------------------------------------------------------------------
// KERNEL_Neumann_boundary3D_sph (functions_BC.cuh:139-274): wall particles
// take the Shepard average over fluid within 2*kappa*h (W evaluated with
// 2h) inside the 27-cell stencil.  pres is the array the walls write into.
// One warp per wall particle (W.wall_idx lists the walls of this step).
// ---------------------------------------------------------------------------
template <typename R>
__global__ void __launch_bounds__(128) k_neumann(DevParams P, SphState<R> S, SphWork<R> W, R* pres,
                                                 const int4* __restrict__ rows,
                                                 int patch_up) {
    grid_dep_wait();
    int w = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
    __shared__ int s_rows[4][20];   // 128 threads = 4 warps
    int* sm = s_rows[threadIdx.x >> 5];
    if (w >= P.nwall || w >= W.counters[0]) return;
    const SphRec<R> rec = W.rec;
    int i = W.wall_idx[w];
    double xi = S.x[i], yi = S.y[i], zi = S.z[i], hi = S.h[i];
    R th2 = (R)2 * (R)hi;
    Knl<R> K = knl_make<R>(P, (R)hi);
    K.ih = rcp(th2);
    K.th = th2;
    double R2 = 2.0 * (P.kappa * hi);
    Band bd = make_band(P, R2);
    PosRec<R> qi = ldr(rec.pos + i);
    int ic, jc, kc;
    cell_ijk(P, xi, yi, zi, ic, jc, kc);
    R tp = 0, flt = 0, tt = 0, tr = 0;
    const Cull cu = make_cull(xi, yi, zi, R2);
    for_rows_warp(P, ic, jc, kc, rows, cu, sm, lane, [&](int j) {
        PosRec<R> qj = ldr(rec.pos + j);
        int ptj = tag_ptype(qj.w);
        if (ptj < 1 || ptj >= 1000) return;
        Disp<R> d;
        R r2;
        if (!test_pair(P, qi, qj, xi, yi, zi, S.x, S.y, S.z, j, R2, 1e-20, bd, d, r2)) return;
        R r, rinv;
        rdist(r2, r, rinv);
        R wk = kw(K, r);
        V4<R> fj = ldr(rec.f1 + j);
        R mj = fj.x, rj = fj.y;
        R mr = mj * rcp(rj) * wk;
        tp += mr * pres[j];
        flt += mr;
        tt += mr * fj.z;
        tr += rj * rcp(fj.w) * wk * mj * rcp(rj);
    });
    tp = warp_sum(tp);
    flt = warp_sum(flt);
    tt = warp_sum(tt);
    tr = warp_sum(tr);
    if (lane != 0) return;
    R pw, rw;
    if (flt < (R)1e-6) {
        rw = W.rho_ref[i];
        pw = (R)0;
    } else {
        pw = tp / flt;
        S.temp[i] = tt / flt;
        rw = rec.f1[i].w * tr / flt;
    }
    pres[i] = pw;
    W.rho_new[i] = rw;
    *comp<R>(rec.f1, i, 1) = rw;
    if (patch_up) *comp<R>(rec.up, i, 3) = pw;
}

// Cell-tiled Neumann pass (FP32 build): one warp per cell that holds wall
// particles.  The fluid candidates of the cell's 9 stencil rows are staged
// (compacted in order) in shared memory with the factors the sums need
// ({x, y, z relative to a particle of the cell, slot} and {m/rho, p, T,
// m/eps}); each lane -- one wall particle of the cell -- runs over them in
// order with its own 2 kappa h radius, FP32 prefilter and the FP64
// reference predicate inside the band.  Same sums as k_neumann in candidate
// order per wall, so the FP32 results differ from it by rounding only.
constexpr int NT_WARPS = 4, NT_CH = 128;
// one cell of k_neumann_tiled (saw, sbw, srw: the warp's shared staging)
__device__ __forceinline__ void neumann_cell(int c, DevParams P, SphState<float> S, SphWork<float> W,
                                                                   float* pres, const int* __restrict__ gs,
                                                                   const int* __restrict__ ge,
                                                                   const int4* __restrict__ rows, int patch_up, float4* saw, float4* sbw, int* srw, int lane) {    const int a0 = __ldg(gs + c);
    if (a0 < 0) return;
    const int e0 = __ldg(ge + c);
    const SphRec<float> rec = W.rec;
    bool any_wall = false;
    for (int i = a0 + lane; i < e0; i += 32) any_wall |= S.ptype[i] <= 0;
    if (!__any_sync(0xffffffffu, any_wall)) return;
    const int ic = c % P.NI, jc = (c / P.NI) % P.NJ, kc = c / (P.NI * P.NJ);
    const int tot = stage_rows(P, ic, jc, kc, rows, srw, lane);
    const RelFrame Fr = rel_frame(P, ldr(rec.pos + a0));
    const unsigned lt = (1u << lane) - 1u;
    for (int p0 = a0; p0 < e0; p0 += 32) {
        const int i = p0 + lane;
        const bool act = i < e0 && S.ptype[i] <= 0;
        if (!__any_sync(0xffffffffu, act)) continue;
        double xi = 0, yi = 0, zi = 0, R2 = 0;
        float lo2 = 0, hi2 = 0, fx = 0, fy = 0, fz = 0;
        Knl<float> K{};
        bool slow = false;
        if (act) {
            xi = S.x[i];
            yi = S.y[i];
            zi = S.z[i];
            const double hi = S.h[i];
            const float th2 = 2.f * (float)hi;
            K = knl_make<float>(P, (float)hi);
            K.ih = rcp(th2);
            K.th = th2;
            R2 = 2.0 * (P.kappa * hi);
            const double b = rel_band(P, Fr, R2), r2 = R2 * R2;
            lo2 = (float)(r2 * (1.0 - b));
            hi2 = (float)(r2 * (1.0 + b));
            const int4 qi = ldr(rec.pos + i);
            slow = Fr.o_oor || rel_slow(Fr, qi);
            const float4 f = rel_coord(Fr, qi, 0);
            fx = f.x;
            fy = f.y;
            fz = f.z;
        }
        const bool lanes_slow = __any_sync(0xffffffffu, act && slow);
        float tp = 0.f, flt = 0.f, tt = 0.f, tr = 0.f;
        float scale = 1.f;   // the sums times scale are the normalised sums
        int t = 0;   // next raw candidate
        while (t < tot) {
            // stage fluid candidates in order until the chunk is full
            int ns = 0;
            bool any_oor = false;
            while (t < tot && ns <= NT_CH - 32) {
                const int tl = t + lane;
                bool keep = false;
                int4 qj = make_int4(0, 0, 0, 0);
                int j = 0;
                if (tl < tot) {
                    j = row_slot(srw, tl);
                    qj = ldr(rec.pos + j);
                    const int ptj = tag_ptype(qj.w);
                    keep = ptj >= 1 && ptj < 1000;
                }
                const unsigned m = __ballot_sync(0xffffffffu, keep);
                if (keep) {
                    const int pos = ns + __popc(m & lt);
                    const bool oor = rel_slow(Fr, qj);
                    any_oor |= oor;
                    const float4 fj = ldr(rec.f1 + j);
                    const float mr = fj.x * rcp(fj.y);
                    saw[pos] = rel_coord(Fr, qj, j | (oor ? (int)0x80000000 : 0));
                    sbw[pos] = make_float4(mr, pres[j], fj.z, fj.x * rcp(fj.w));
                }
                ns += __popc(m);
                t += 32;
            }
            const bool slow_chunk = lanes_slow || __any_sync(0xffffffffu, any_oor);
            __syncwarp();
            if (act && !slow_chunk && K.kt == 3) {
                // every candidate on the FP32 frame: the kernel is evaluated
                // for all of them and the pairs outside the radius add
                // nothing, so the lanes do not diverge (only a pair in the
                // rounding band takes the FP64 predicate).  Wendland C2 in
                // line without its normalisation tA, which cancels in the
                // ratios below (only the empty-support test scales by it).
                const float hq = 0.5f * K.ih;
#pragma unroll 4
                for (int u = 0; u < ns; u++) {
                    const float4 cj = saw[u];
                    const float dx = fx - cj.x, dy = fy - cj.y, dz = fz - cj.z;
                    const float r2 = dx * dx + dy * dy + dz * dz;
                    bool in = r2 < lo2;
                    if (!in && r2 <= hi2) {
                        const int j = __float_as_int(cj.w);
                        in = __dadd_rn(pair_dist(xi, yi, zi, S.x[j], S.y[j], S.z[j]), 1e-20) < R2;
                    }
                    const float q = r2 * rsqrtf(fmaxf(r2, 1e-30f)) * hq;
                    const float a = 1.f - q, a2 = a * a;
                    const float wk = a2 * a2 * (1.f + 4.f * q);
                    const float4 bj = sbw[u];
                    if (in && q < 1.f) {
                        const float mr = bj.x * wk;
                        tp += mr * bj.y;
                        flt += mr;
                        tt += mr * bj.z;
                        tr += bj.w * wk;
                    }
                }
                scale = K.tA;
            } else if (act && !slow_chunk) {
                // as above, any kernel
#pragma unroll 2
                for (int u = 0; u < ns; u++) {
                    const float4 cj = saw[u];
                    const float dx = fx - cj.x, dy = fy - cj.y, dz = fz - cj.z;
                    const float r2 = dx * dx + dy * dy + dz * dz;
                    bool in = r2 < lo2;
                    if (!in && r2 <= hi2) {
                        const int j = __float_as_int(cj.w);
                        in = __dadd_rn(pair_dist(xi, yi, zi, S.x[j], S.y[j], S.z[j]), 1e-20) < R2;
                    }
                    float r, rinv;
                    rdist(r2, r, rinv);
                    const float wk = kw(K, r);
                    const float4 bj = sbw[u];
                    if (in) {
                        const float mr = bj.x * wk;
                        tp += mr * bj.y;
                        flt += mr;
                        tt += mr * bj.z;
                        tr += bj.w * wk;
                    }
                }
            } else if (act) {
                for (int u = 0; u < ns; u++) {
                    const float4 cj = saw[u];
                    const float dx = fx - cj.x, dy = fy - cj.y, dz = fz - cj.z;
                    const float r2 = dx * dx + dy * dy + dz * dz;
                    bool in;
                    if (!slow_chunk) {
                        if (r2 > hi2) continue;
                        in = r2 < lo2;
                        if (!in) {
                            const int j = __float_as_int(cj.w);
                            in = __dadd_rn(pair_dist(xi, yi, zi, S.x[j], S.y[j], S.z[j]), 1e-20) < R2;
                        }
                    } else {
                        const int jb = __float_as_int(cj.w), j = jb & 0x7fffffff;
                        if (!slow && jb >= 0) {
                            if (r2 > hi2) continue;
                            in = r2 < lo2 ||
                                 __dadd_rn(pair_dist(xi, yi, zi, S.x[j], S.y[j], S.z[j]), 1e-20) < R2;
                        } else {
                            in = __dadd_rn(pair_dist(xi, yi, zi, S.x[j], S.y[j], S.z[j]), 1e-20) < R2;
                        }
                    }
                    if (!in) continue;
                    float r, rinv;
                    if (!slow_chunk || (!slow && __float_as_int(cj.w) >= 0)) {
                        rdist(r2, r, rinv);
                    } else {
                        const int j = __float_as_int(cj.w) & 0x7fffffff;
                        const float ex = (float)(xi - S.x[j]), ey = (float)(yi - S.y[j]), ez = (float)(zi - S.z[j]);
                        rdist(ex * ex + ey * ey + ez * ez, r, rinv);
                    }
                    const float wk = kw(K, r);
                    const float4 bj = sbw[u];
                    const float mr = bj.x * wk;
                    tp += mr * bj.y;
                    flt += mr;
                    tt += mr * bj.z;
                    tr += bj.w * wk;
                }
            }
            __syncwarp();
        }
        if (!act) continue;
        float pw, rw;
        if (flt * scale < 1e-6f) {
            rw = W.rho_ref[i];
            pw = 0.f;
        } else {
            pw = tp / flt;
            S.temp[i] = tt / flt;
            rw = rec.f1[i].w * tr / flt;
        }
        pres[i] = pw;
        W.rho_new[i] = rw;
        *comp<float>(rec.f1, i, 1) = rw;
        if (patch_up) *comp<float>(rec.up, i, 3) = pw;
    }
}

template <bool OCC>
__global__ void __launch_bounds__(NT_WARPS * 32, 8) k_neumann_tiled(DevParams P, SphState<float> S, SphWork<float> W,
                                                                   float* pres, const int* __restrict__ gs,
                                                                   const int* __restrict__ ge,
                                                                   const int4* __restrict__ rows, int patch_up,
                                                                   const int* __restrict__ occ, const int* __restrict__ occ_n) {
    grid_dep_wait();
    __shared__ float4 sa[NT_WARPS][NT_CH + 32];
    __shared__ float4 sb[NT_WARPS][NT_CH + 32];
    __shared__ int srow[NT_WARPS][20];
    const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
    if constexpr (OCC) {   // a sparse grid: the occupied cells, grid-stride
        const int no = *occ_n;
        for (int q = blockIdx.x * NT_WARPS + w; q < no; q += gridDim.x * NT_WARPS) {
            neumann_cell(occ[q], P, S, W, pres, gs, ge, rows, patch_up, sa[w], sb[w], srow[w], lane);
            __syncwarp();
        }
    } else {
        const int c = blockIdx.x * NT_WARPS + w;
        if (c < P.NI * P.NJ * P.NK) neumann_cell(c, P, S, W, pres, gs, ge, rows, patch_up, sa[w], sb[w], srow[w], lane);
    }
}

// ---------------------------------------------------------------------------
// KERNEL_PPE3D_sph + KERNEL_PPE3D_calc_sph (functions_PPE2.cuh:542-698,
// 868-878): one Jacobi sweep; p_new = (b + sum A_ij p_j) / sum A_ij for
// fluid, every other particle keeps its pressure.
// ---------------------------------------------------------------------------
template <typename R, int KT, int SW>
__global__ void __launch_bounds__(128) k_ppe(DevParams P, SphState<R> S, SphWork<R> W) {
    grid_dep_wait();
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    int n = P.ns;
    if (i >= n) return;
    const SphRec<R> rec = W.rec;
    int it = S.itype[i], pt = S.ptype[i], bt = S.btype[i];
    V4<R> upi = rec.up[i];
    bool solve = it <= 2 && !(P.open_bc > 0 && bt > 0) && pt < 1000 && pt > 0;
    if (!solve) {
        W.p_new[i] = upi.w;
        return;
    }
    R th = (R)S.h[i];
    Knl<R, KT> K = knl_make<R, KT>(P, th);
    PosRec<R> qi = ldr(rec.pos + i);
    V4<R> fi = rec.f1[i];
    R uxi = upi.x, uyi = upi.y, uzi = upi.z, rhoi = fi.y, pori = fi.w;
    R irhoi = rcp(rhoi), prhoi = pori * rhoi;
    R pux = pori * uxi, puy = pori * uyi, puz = pori * uzi;
    const bool kgc = sw_on<SW>(SW_KGC, P.kgc == 1);
    Cm9<R> Cm = cm_load(W.Cm, n, i, kgc);
    int cnt = min(W.ncnt[i], P.nb_cap);
    R bx = 0, by = 0, bz = 0, A = 0, AP = 0;
    const int* __restrict__ nb = W.nbr;
    nb_walk<4, NbQ44<R>>(
        cnt, nb, n, i,
        [&](int j) {
            NbQ44<R> t;
            t.q = ldr(rec.pos + j);
            t.a = ldr(rec.f1 + j);
            t.b = ldr(rec.up + j);
            return t;
        },
        [&](int j, const NbQ44<R>& t) {
            int tj = t.q.w;
            if (tag_ptype(tj) >= 1000 || tag_itype(tj) == 4) return;
            const V4<R>& fj = t.a;
            const V4<R>& uj = t.b;
            Disp<R> g = disp(P, qi, t.q, S.x, S.y, S.z, i, j);
            R r2 = g.dx * g.dx + g.dy * g.dy + g.dz * g.dz, r, rinv;
            rdist(r2, r, rinv);
            R mj = fj.x, rhoj = fj.y, porj = fj.w, irj = rcp(rhoj);
            R dw = kdw(K, r);
            R gx = dw * g.dx * rinv, gy = dw * g.dy * rinv, gz = dw * g.dz * rinv;
            cm_apply(Cm, kgc, gx, gy, gz);
            R mr = mj * irj;
            bx += mr * (pux - porj * uj.x) * gx;
            by += mr * (puy - porj * uj.y) * gy;
            bz += mr * (puz - porj * uj.z) * gz;
            R c = -(g.dx * gx + g.dy * gy + g.dz * gz) * rinv * rinv;
            R a = mj * ((prhoi + porj * rhoj) * irj * irhoi) * c;
            A += a;
            AP += a * uj.w;
        });
    R b = (R)P.rho_gas * (bx + by + bz + (R)2 * S.dDEMpor[i] - W.dDEMpor_prev[i]) / (R)P.sdt;
    W.p_new[i] = (b + AP) / A;
}

// ---------------------------------------------------------------------------
// pass C: KERNEL_pressureforce3D_sph (functions_PPE2.cuh:2154-2335) and
// KERNEL_time_update_projection_sph (functions_TIME_ISPH2.cuh:467-620).
// ---------------------------------------------------------------------------
template <typename R, int KT, int SW>
__global__ void __launch_bounds__(128) k_passC(DevParams P, SphState<R> S, SphWork<R> W) {
    grid_dep_wait();
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    int n = P.ns;
    if (i >= n) return;
    const SphRec<R> rec = W.rec;
    int it = S.itype[i], pt = S.ptype[i], bt = S.btype[i];
    W.fpx[i] = 0; W.fpy[i] = 0; W.fpz[i] = 0;
    if (it > 2) {
        rec.ut[i] = mk4<R>(S.ux[i], S.uy[i], S.uz[i], S.temp[i]);
        return;
    }
    R fx = 0, fy = 0, fz = 0;
    bool pf = !(P.open_bc > 0 && bt > 0) && pt < 1000 && pt > 0;
    if (pf && sw_on<SW>(SW_FP, P.fp != 0)) {
        R th = (R)S.h[i];
        Knl<R, KT> K = knl_make<R, KT>(P, th);
        PosRec<R> qi = ldr(rec.pos + i);
        R pi = W.p_new[i], rhoi = W.rho_new[i], pori = rec.f1[i].w;
        R cpi = -pori * rcp(rhoi);
        const bool kgc = sw_on<SW>(SW_KGC, P.kgc == 1);
        Cm9<R> Cm = cm_load(W.Cm, n, i, kgc);
        int cnt = min(W.ncnt[i], P.nb_cap);
        const int* __restrict__ nb = W.nbr;
        const R* __restrict__ pn = W.p_new;
        nb_walk<4, NbQ2S<R>>(
            cnt, nb, n, i,
            [&](int j) {
                NbQ2S<R> t;
                t.q = ldr(rec.pos + j);
                t.a = ldr(reinterpret_cast<const V2<R>*>(rec.f1 + j));
                t.s = __ldg(pn + j);
                return t;
            },
            [&](int j, const NbQ2S<R>& t) {
                if (tag_ptype(t.q.w) >= 1000) return;
                Disp<R> g = disp(P, qi, t.q, S.x, S.y, S.z, i, j);
                R r2 = g.dx * g.dx + g.dy * g.dy + g.dz * g.dz, r, rinv;
                rdist(r2, r, rinv);
                R dw = kdw(K, r);
                R gx = dw * g.dx * rinv, gy = dw * g.dy * rinv, gz = dw * g.dz * rinv;
                cm_apply(Cm, kgc, gx, gy, gz);
                R Cp = cpi * t.a.x * (pi + t.s) * rcp(t.a.y);
                fx += Cp * gx;
                fy += Cp * gy;
                fz += Cp * gz;
            });
        W.fpx[i] = fx; W.fpy[i] = fy; W.fpz[i] = fz;
    }
    if (pt == 9) {
        rec.ut[i] = mk4<R>(S.ux[i], S.uy[i], S.uz[i], S.temp[i]);
        return;
    }
    R ux0, uy0, uz0, ax, ay, az;
    if (pt > 0) {
        ux0 = S.ux[i]; uy0 = S.uy[i]; uz0 = S.uz[i];
        R b = (R)(bt == 0);
        ax = fx * b; ay = fy * b; az = fz * b;
    } else {
        ux0 = W.ux0[i]; uy0 = W.uy0[i]; uz0 = W.uz0[i];
        ax = ay = az = (R)0;
    }
    R dt = (R)P.sdt;
    R uxc = ux0 + ax * dt, uyc = uy0 + ay * dt, uzc = uz0 + az * dt;
    R lim = (R)P.u_limit;
    if ((uxc * uxc + uyc * uyc + uzc * uzc) >= lim * lim) {
        uxc = ux0; uyc = uy0; uzc = uz0;
    }
    if (!P.xsph && sw_on<SW>(SW_LAGR, P.sph_lagrangian != 0) && pt > 0) {
        S.x[i] += ((double)W.ux0[i] + (double)uxc) / 2.0 * P.sdt;
        S.y[i] += ((double)W.uy0[i] + (double)uyc) / 2.0 * P.sdt;
        S.z[i] += ((double)W.uz0[i] + (double)uzc) / 2.0 * P.sdt;
    }
    S.ux[i] = uxc; S.uy[i] = uyc; S.uz[i] = uzc;
    R tn = S.temp[i];
    if (sw_on<SW>(SW_CON, P.con != 0) && pt > 0) {
        tn = W.temp0[i] + W.dtemp[i] * dt * (R)(pt != -1);
        S.temp[i] = tn;
    }
    rec.ut[i] = mk4<R>(uxc, uyc, uzc, tn);
}

// ---------------------------------------------------------------------------
// DEM corrector (KERNEL_time_update_projection_dem, functions_TIME_ISPH2.cuh:
// 622-776) followed by KERNEL_treat_DEM_{cylinder_z,box_z,truncated_cone_z}_dem
// (functions_DEM_BC.cuh:491-718, 1770-2027, 4485-4722) on the same particle.
// ---------------------------------------------------------------------------
template <typename R>
__device__ void dem_wall_response(const DevParams& P, DemState<R>& D, DemWork<R>& DW, int i, R nx, R ny, R nz) {
    R kdt = (R)P.dt;
    R ux = D.ux[i], uy = D.uy[i], uz = D.uz[i], wx = D.wx[i], wy = D.wy[i], wz = D.wz[i];
    R m = D.m[i], ri = D.ri[i], rad = (R)D.rad[i];
    R ftx = DW.ftx[i], fty = DW.fty[i], ftz = DW.ftz[i];
    R ucx = ux - rad * (wy * nz - wz * ny), ucy = uy - rad * (wz * nx - wx * nz), ucz = uz - rad * (wx * ny - wy * nx);
    R cwx = -rad * (wy * nz - wz * ny), cwy = -rad * (wz * nx - wx * nz), cwz = -rad * (wx * ny - wy * nx);
    R unm = ux * nx + uy * ny + uz * nz;
    R ucn = ucx * nx + ucy * ny + ucz * nz, cwn = cwx * nx + cwy * ny + cwz * nz;
    R usx = ucx - ucn * nx, usy = ucy - ucn * ny, usz = ucz - ucn * nz;
    R uwx = cwx - cwn * nx, uwy = cwy - cwn * ny, uwz = cwz - cwn * nz;
    const R tiny = (R)1e-10;
    if (fabs(usx) < tiny) usx = 0;
    if (fabs(usy) < tiny) usy = 0;
    if (fabs(usz) < tiny) usz = 0;
    if (fabs(uwx) < tiny) uwx = 0;
    if (fabs(uwy) < tiny) uwy = 0;
    if (fabs(uwz) < tiny) uwz = 0;
    R usm = sqrt(usx * usx + usy * usy + usz * usz), uwm = sqrt(uwx * uwx + uwy * uwy + uwz * uwz);
    R sx = usx / (usm + (R)1e-20), sy = usy / (usm + (R)1e-20), sz = usz / (usm + (R)1e-20);
    R swx = uwx / (uwm + (R)1e-20), swy = uwy / (uwm + (R)1e-20), swz = uwz / (uwm + (R)1e-20);
    if (fabs(unm) < (R)50 * kdt) {
        R fn = ftx * nx + fty * ny + ftz * nz;
        R a = (R)P.mu_s * m * fn, b = (R)P.mu_rs * m * fn;
        R ffx = a * sx, ffy = a * sy, ffz = a * sz, frx = b * swx, fry = b * swy, frz = b * swz;
        if (fn > (R)0) { ffx = ffy = ffz = frx = fry = frz = 0; }
        DW.ftx[i] = ftx + ffx / m;
        DW.fty[i] = fty + ffy / m;
        DW.ftz[i] = ftz + ffz / m;
        R q = rad / ri;
        DW.tqx[i] += -q * (ny * (ffz + frz) - nz * (ffy + fry));
        DW.tqy[i] += -q * (nz * (ffx + frx) - nx * (ffz + frz));
        DW.tqz[i] += -q * (nx * (ffy + fry) - ny * (ffx + frx));
        R uxc = ux + (ffx / m) * kdt, uyc = uy + (ffy / m) * kdt, uzc = uz + (ffz / m) * kdt;
        R ucn2 = uxc * nx + uyc * ny + uzc * nz;
        D.ux[i] = uxc - ucn2 * nx;
        D.uy[i] = uyc - ucn2 * ny;
        D.uz[i] = uzc - ucn2 * nz;
        D.wx[i] = wx - q * (ny * (ffz + frz) - nz * (ffy + fry)) * kdt;
        D.wy[i] = wy - q * (nz * (ffx + frx) - nx * (ffz + frz)) * kdt;
        D.wz[i] = wz - q * (nx * (ffy + fry) - ny * (ffx + frx)) * kdt;
    } else {
        R cn = -m * ((R)1 + (R)P.rest_n) * ucn;
        R cs = -(R)1 / (((R)1 / m) + (rad * rad / ri)) * ((R)1 + (R)P.rest_s) * usm;
        R Jx = cn * nx + cs * sx, Jy = cn * ny + cs * sy, Jz = cn * nz + cs * sz;
        R q = rad / ri;
        D.ux[i] = ux + ((R)1 / m) * Jx;
        D.uy[i] = uy + ((R)1 / m) * Jy;
        D.uz[i] = uz + ((R)1 / m) * Jz;
        D.wx[i] = wx - q * (ny * Jz - nz * Jy);
        D.wy[i] = wy - q * (nz * Jx - nx * Jz);
        D.wz[i] = wz - q * (nx * Jy - ny * Jx);
    }
}

template <typename R>
__global__ void __launch_bounds__(128) k_dem_update(DevParams P, DemState<R> D, DemWork<R> DW) {
    grid_dep_wait();
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= P.nd) return;
    int it = D.itype[i], pt = D.ptype[i];
    if (it > 2) return;
    if (pt != 9) {
        R ux0, uy0, uz0;
        if (pt > 0) { ux0 = D.ux[i]; uy0 = D.uy[i]; uz0 = D.uz[i]; }
        else { ux0 = DW.ux0[i]; uy0 = DW.uy0[i]; uz0 = DW.uz0[i]; }
        // fp and fb are zero for DEM particles: the corrector keeps u*
        R lim = (R)P.u_limit;
        R uxc = ux0, uyc = uy0, uzc = uz0;
        if ((uxc * uxc + uyc * uyc + uzc * uzc) >= lim * lim) { uxc = ux0; uyc = uy0; uzc = uz0; }
        if (pt > 0) {
            D.x[i] += ((double)DW.ux0[i] + (double)uxc) / 2.0 * P.dt;
            D.y[i] += ((double)DW.uy0[i] + (double)uyc) / 2.0 * P.dt;
            D.z[i] += ((double)DW.uz0[i] + (double)uzc) / 2.0 * P.dt;
        }
        D.ux[i] = uxc; D.uy[i] = uyc; D.uz[i] = uzc;
    }
    if (P.con && pt > 0) D.temp[i] = DW.temp0[i] + DW.dtemp[i] * (R)P.dt * (R)(pt != -1);
    if (it != 1 || pt <= 1000) return;
    // cylinder_z
    if (P.wall_mask & 1) {
        double xc = P.cyl_cx, yc = P.cyl_cy, Rc = P.cyl_r;
        double x = D.x[i], y = D.y[i], z = D.z[i], rad = D.rad[i];
        double F = (x - xc) * (x - xc) + (y - yc) * (y - yc) - (Rc - rad) * (Rc - rad);
        if (F > 0) {
            double rr = sqrt((x - xc) * (x - xc) + (y - yc) * (y - yc));
            double cpx = xc + (Rc - rad) * (x - xc) / rr, cpy = yc + (Rc - rad) * (y - yc) / rr;
            D.x[i] = cpx; D.y[i] = cpy; D.z[i] = z;
            double nx = -(cpx - xc) / (Rc - rad), ny = -(cpy - yc) / (Rc - rad);
            if (!(sqrt(nx * nx + ny * ny) < 0.5)) dem_wall_response<R>(P, D, DW, i, (R)nx, (R)ny, (R)0);
        }
    }
    // box_z
    if (P.wall_mask & 2) {
        double xc = P.box_c[0], yc = P.box_c[1], zc = P.box_c[2];
        double hx = 0.5 * P.box_L[0], hy = 0.5 * P.box_L[1], hz = 0.5 * P.box_L[2];
        double x = D.x[i], y = D.y[i], z = D.z[i], rad = D.rad[i];
        double F = fmax(fmax(fabs(x - xc) - (hx - rad), fabs(y - yc) - (hy - rad)), fabs(z - zc) - (hz - rad));
        if (F > 0) {
            double cpx = xc + fmin(hx - rad, fmax(-(hx - rad), x - xc));
            double cpy = yc + fmin(hy - rad, fmax(-(hy - rad), y - yc));
            double cpz = zc + fmin(hz - rad, fmax(-(hz - rad), z - zc));
            D.x[i] = cpx; D.y[i] = cpy; D.z[i] = cpz;
            double sgx = (cpx - x) / (fabs(cpx - x) + 1e-20);
            double sgy = (cpy - y) / (fabs(cpy - y) + 1e-20);
            double sgz = (cpz - z) / (fabs(cpz - z) + 1e-20);
            if (fabs(cpy - y) < 1e-12) sgy = 0.0;
            if (fabs(cpy - x) < 1e-12) sgx = 0.0;  // the reference tests cpy-x here (functions_DEM_BC.cuh:1846)
            if (fabs(cpz - z) < 1e-12) sgz = 0.0;
            double nn = sqrt(sgx * sgx + sgy * sgy + sgz * sgz) + 1e-20;
            double nx = sgx / nn, ny = sgy / nn, nz = sgz / nn;
            if (!(sqrt(nx * nx + ny * ny + nz * nz) < 0.5)) dem_wall_response<R>(P, D, DW, i, (R)nx, (R)ny, (R)nz);
        }
    }
    // truncated_cone_z
    if (P.wall_mask & 4) {
        double xc = P.cone_c[0], yc = P.cone_c[1], r1 = P.cone_r1, r2 = P.cone_r2, hc = P.cone_h;
        double x = D.x[i], y = D.y[i], z = D.z[i], rad = D.rad[i];
        if (!(z <= -hc + rad)) {
            double L = sqrt((r1 - r2) * (r1 - r2) + hc * hc);
            double st = hc / L, ct = fabs(r1 - r2) / L, tt = st / ct;
            double rr = r2 + (hc + z) / tt - rad / st;
            double rxy = sqrt((x - xc) * (x - xc) + (y - yc) * (y - yc));
            double F = (x - xc) * (x - xc) + (y - yc) * (y - yc) - rr * rr;
            if (F > 0) {
                double cpz = tt * (rxy + rad / st - r2) - hc;
                D.z[i] = cpz;
                double nx = -st * (x - xc) / rxy, ny = -st * (y - yc) / rxy, nz = ct;
                dem_wall_response<R>(P, D, DW, i, (R)nx, (R)ny, (R)nz);
            }
        }
    }
}

// ---------------------------------------------------------------------------
// KERNEL_open_boundary_extrapolation3D_1{,_calc}_sph (functions_BC.cuh:
// 787-984, 1204-1218): buffer particles take Shepard averages of the fluid
// around their mirror point.  Only non-buffer fluid is read, so the update
// is done in place.  One warp per buffer particle (W.buf_idx).
// ---------------------------------------------------------------------------
template <typename R, int KT>
__global__ void __launch_bounds__(128) k_open_bc(DevParams P, SphState<R> S, SphWork<R> W, const int4* __restrict__ rows) {
    grid_dep_wait();
    int w = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
    __shared__ int s_rows[4][20];   // 128 threads = 4 warps
    int* sm = s_rows[threadIdx.x >> 5];
    if (w >= P.nbuf || w >= W.counters[1]) return;
    int i = W.buf_idx[w];
    int bt = S.btype[i];
    double xi = S.x[i], yi = S.y[i], zi = S.z[i], hi = S.h[i];
    const BedObc ob = bed_obc(P, yi);
    double zg = zi;
    if (bt == 1) zg = 2 * ob.L2 - zi;
    else if (bt == 2) zg = 2 * ob.L3 - zi;
    R th = (R)hi;
    Knl<R, KT> K = knl_make<R, KT>(P, th);
    double Rr = P.kappa * hi;
    const Band bd = make_band(P, Rr);
    const PosRec<R> qp = make_pos<R>(P, xi, yi, zg, 0, 0, 0);   // the mirror point
    int ic, jc, kc;
    cell_ijk(P, xi, yi, zg, ic, jc, kc);
    R hd = (R)P.h_over_dx;
    R trho = 0, tp = 0, tux = 0, tuy = 0, tuz = 0, tt = 0, flt = 0;
    const Cull cu = make_cull(xi, yi, zg, Rr);
    // the candidate's type and the prefilter from its packed record (one
    // load); the FP64 predicate only inside the band
    for_rows_warp(P, ic, jc, kc, rows, cu, sm, lane, [&](int j) {
        const PosRec<R> qj = ldr(W.rec.pos + j);
        if (tag_ptype(qj.w) != 1 || tag_btype(qj.w) != 0) return;
        Disp<R> d;
        R r2;
        if (!test_pair(P, qp, qj, xi, yi, zg, S.x, S.y, S.z, j, Rr, 1e-20, bd, d, r2)) return;
        R r, rinv;
        rdist(r2, r, rinv);
        R wk = kw(K, r);
        R hj = (R)S.h[j];
        R volj = sph_volume(P, hj, hd);
        R vw = volj * wk;
        trho += W.rho_new[j] / W.DEMpor[j] * wk * volj;
        tp += vw * W.p_new[j];
        tuz += vw * S.uz[j];
        tux += vw * S.ux[j];
        tuy += vw * S.uy[j];
        tt += vw * S.temp[j];
        flt += vw;
    });
    trho = warp_sum(trho); tp = warp_sum(tp); tux = warp_sum(tux); tuy = warp_sum(tuy);
    tuz = warp_sum(tuz); tt = warp_sum(tt); flt = warp_sum(flt);
    if (lane != 0 || P.open_bc != 1) return;
    R pori = W.DEMpor[i];
    R vol0 = sph_volume(P, th, hd);
    R rho_old = W.rho_new[i];
    R pn, rn, ux, uy, uz, tn;
    if (bt == 1) {
        pn = tp / flt;
        rn = pori * (R)P.rho_gas;
        uz = (R)ob.inlet_uz * (R)2 - tuz / flt;
        ux = (R)0 - tux / flt;
        uy = (R)0 - tuy / flt;
        tn = (R)(ob.inlet_temp - P.t_ref);   // stored T - t_ref
    } else {
        pn = (R)0;
        rn = pori * (trho / flt);
        uz = tuz / flt;
        ux = tux / flt;
        uy = tuy / flt;
        tn = tt / flt;
    }
    R mn = rho_old * vol0;
    W.p_new[i] = pn;
    W.rho_new[i] = rn;
    W.m_new[i] = mn;
    S.ux[i] = ux; S.uy[i] = uy; S.uz[i] = uz;
    S.temp[i] = tn;
    // the XSPH pass reads buffer particles through the records
    *comp<R>(W.rec.f1, i, 0) = mn;
    *comp<R>(W.rec.f1, i, 1) = rn;
    W.rec.ut[i] = mk4<R>(ux, uy, uz, tn);
}

// ---------------------------------------------------------------------------
// KERNEL_xsph3D_sph + KERNEL_xsph3D_calc_sph (functions_TIME.cuh:1735-1997).
// Writes the smoothed velocity/temperature of every particle (or a copy)
// into u_tmp/temp_tmp; the next reorder reads them.
// ---------------------------------------------------------------------------
template <typename R, int KT>
__global__ void __launch_bounds__(128, sizeof(R) == 4 ? 6 : 1) k_xsph(DevParams P, SphState<R> S, SphWork<R> W) {
    grid_dep_wait();
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    int n = P.ns;
    if (i >= n) return;
    const SphRec<R> rec = W.rec;
    int it = S.itype[i], pt = S.ptype[i];
    V4<R> ui = rec.ut[i];
    R uxi = ui.x, uyi = ui.y, uzi = ui.z, ti = ui.w;
    if (it != 1 || pt > 1000 || pt == 0 || pt == 9) {
        W.u_tmpx[i] = uxi; W.u_tmpy[i] = uyi; W.u_tmpz[i] = uzi; W.temp_tmp[i] = ti;
        return;
    }
    R th = (R)S.h[i];
    Knl<R, KT> K = knl_make<R, KT>(P, th);
    PosRec<R> qi = ldr(rec.pos + i);
    R c = (R)P.c_xsph;
    int cnt = min(W.ncnt[i], P.nb_cap);
    R tx = 0, ty = 0, tz = 0, tt = 0, flt = 0;
    const int* __restrict__ nb = W.nbr;
    nb_walk<4, NbQ24<R>>(
        cnt, nb, n, i,
        [&](int j) {
            NbQ24<R> t;
            t.q = ldr(rec.pos + j);
            t.a = ldr(reinterpret_cast<const V2<R>*>(rec.f1 + j));
            t.b = ldr(rec.ut + j);
            return t;
        },
        [&](int j, const NbQ24<R>& t) {
            int ptj = tag_ptype(t.q.w);
            if (ptj != 1 && ptj != 3) return;
            Disp<R> g = disp(P, qi, t.q, S.x, S.y, S.z, i, j);
            R r2 = g.dx * g.dx + g.dy * g.dy + g.dz * g.dz, r, rinv;
            rdist(r2, r, rinv);
            R w = kw(K, r);
            R m = t.a.x * rcp(t.a.y) * w;
            R cm = c * m;
            tx += cm * (t.b.x - uxi);
            ty += cm * (t.b.y - uyi);
            tz += cm * (t.b.z - uzi);
            tt += (R)0.01 * cm * (t.b.w - ti);
            flt += m;
        });
    R on = (R)(pt > 0);
    R iflt = rcp(flt);
    W.u_tmpx[i] = (uxi + tx * iflt) * on;
    W.u_tmpy[i] = (uyi + ty * iflt) * on;
    W.u_tmpz[i] = (uzi + tz * iflt) * on;
    W.temp_tmp[i] = (ti + tt * iflt) * on;
}

// end of a step: the host loop's count++ (ISPH_Calc_seperate.cuh:925)
__global__ void k_tick(DevFlags* F) {
    grid_dep_wait(); F->step_count += 1; }

// ---------------------------------------------------------------------------
// printed maxima (kernel_copy_max_*, functions_OUTPUT.cuh:19-65 + cub max)
// out[0..2] = rho, |u|, ftotal over p_type!=0 && i_type<2 (zeroed by the
// caller).  Grid-stride blocks; block maxima are combined with an integer
// atomicMax on the bit patterns, which orders non-negative doubles.
// ---------------------------------------------------------------------------
template <typename R, typename RR = R>
__global__ void __launch_bounds__(256) k_stats(int n, const RR* __restrict__ rho, const R* __restrict__ ux,
                                               const R* __restrict__ uy, const R* __restrict__ uz,
                                               const R* __restrict__ ft, const int* __restrict__ ptype,
                                               const int* __restrict__ itype, double* out, DevFlags* F) {
    __shared__ double sm[3][256];
    double a = 0, b = 0, c = 0;
    int bad = 0;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        double uzi = uz ? (double)uz[i] : 0.0;   // 2-D sets pass no uz
        double u = sqrt((double)ux[i] * ux[i] + (double)uy[i] * uy[i] + uzi * uzi);
        if (!isfinite(u) || !isfinite((double)rho[i])) bad = 1;
        if (ptype[i] == 0 || itype[i] >= 2) continue;
        a = fmax(a, (double)rho[i]);
        b = fmax(b, u);
        c = fmax(c, ft ? (double)ft[i] : 0.0);
    }
    sm[0][threadIdx.x] = a; sm[1][threadIdx.x] = b; sm[2][threadIdx.x] = c;
    if (bad) atomicOr(&F->nan, 1);
    __syncthreads();
    for (int s = blockDim.x / 2; s > 0; s >>= 1) {
        if (threadIdx.x < s)
            for (int q = 0; q < 3; q++) sm[q][threadIdx.x] = fmax(sm[q][threadIdx.x], sm[q][threadIdx.x + s]);
        __syncthreads();
    }
    if (threadIdx.x == 0)
        for (int q = 0; q < 3; q++)
            atomicMax(reinterpret_cast<unsigned long long*>(out + q), (unsigned long long)__double_as_longlong(sm[q][0]));
}

}  // namespace sphdem
